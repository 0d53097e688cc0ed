"""bench.py's launch contract, on CPU: `--gpus N` starts N ranks itself (one
process per GPU, the RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* environment of
torchrun) and rank 0 alone prints one JSON line with n_gpus = N. The
`--dry-run` switch runs that protocol over gloo without a device."""
from __future__ import annotations

import importlib.util
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(ROOT, "bench.py")


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_module", BENCH)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def run(*args, env=None):
    e = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        e.pop(k, None)
    e.update(env or {})
    return subprocess.run([sys.executable, BENCH, *args], capture_output=True, text=True,
                          timeout=240, env=e, cwd=ROOT)


def test_gpus_two_starts_two_ranks_and_rank_zero_reports_them():
    out = run("--gpus", "2", "--dry-run")
    assert out.returncode == 0, out.stderr
    assert "rank 0 of 2 started" in out.stderr
    assert "rank 1 of 2 started" in out.stderr
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["dry_run"] is True
    assert line["max_over_ranks"] == 2.0  # the max over both ranks' values


def test_one_gpu_runs_in_process_and_a_launcher_is_respected():
    out = run("--dry-run")
    assert out.returncode == 0 and json.loads(out.stdout.strip())["n_gpus"] == 1
    # under a launcher (WORLD_SIZE set) bench.py does not spawn again
    out = run("--gpus", "2", "--dry-run", env={"WORLD_SIZE": "1", "RANK": "0",
                                               "LOCAL_RANK": "0"})
    assert out.returncode == 0
    assert json.loads(out.stdout.strip())["n_gpus"] == 1
    assert "rank 1 of" not in out.stderr


def test_bench_workloads_are_the_package_workloads():
    from parallax_b200.scenes import WORKLOADS

    bench = load_bench()
    for name, w in bench.BENCH_WORKLOADS.items():
        assert w == WORKLOADS[name]


def test_both_arms_schedule_the_same_views():
    bench = load_bench()
    assert bench.view_ids(0, 8, 64) == list(range(8))
    assert bench.view_ids(9, 8, 64) == [8, 9, 10, 11, 12, 13, 14, 15]
    assert bench.view_ids(0, 8, 64, rank=1) == list(range(7, 15))

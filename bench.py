#!/usr/bin/env python
"""Gaussian-splat training step benchmark on B200.

Workload (default "c4"): 1M gaussians, SH degree 3, a 64-camera pool at
1920x1440 (Fibonacci sphere, radius 3, 60 degree FOV), 8 views per step
rendered, differentiated and accumulated, then one Adam step. Synthetic data:
truth cloud seed 1 (targets rendered from it and quantised to 8-bit frames),
start cloud seed 2, cameras seed 3; inputs are larger than L2 (1M gaussians x
236 B of parameters, 8 x 33 MB of targets per step), so no L2 flush is needed
between steps.

Arms:
  ours (default)  the batched, CUDA-graph-captured step; also the plain
                  per-view form, the end-to-end step through the C ABI with the
                  step's 8-bit target frames copied from pinned host memory and
                  converted on the device (and, beside it, FP32 images), per-stage
                  device timing, the roofline of the dominant kernel and, on
                  rank 0 at N=1, one full step of the reference's CPU trainer.
  reference       the reference's own CPU trainer (compiled from its sources into
                  oracle/_ref with its release flags) on the same workload and
                  view schedule: every step renders, scores and differentiates
                  the step's views, one view per host thread, adds the
                  gradients and takes the reference's Adam step
                  (oracle/ref_bench.py). It never loads the product library.

Multi-GPU: `--gpus N` starts N ranks itself (one process per GPU, RANK /
LOCAL_RANK / WORLD_SIZE / MASTER_ADDR=127.0.0.1 in their environment) unless
a launcher (torchrun) already set WORLD_SIZE. Data parallel over views: each
rank renders and differentiates its own 8 views per step (weak scaling), the
gradient block is summed with one NCCL all-reduce, and every rank applies the
same Adam step. `--dry-run` runs the same launch and rank protocol on CPU
(gloo) without a device, for tests.
"""
from __future__ import annotations

import argparse
import ctypes as ct
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STAGES = ["project", "bin", "forward", "loss", "backward", "param_grads", "adam"]
DATA = ("synthetic (seeded: truth cloud 1, start cloud 2, cameras 3; targets rendered from the "
        "truth cloud, quantised to 8-bit frames)")
METRIC = "train steps/s (fwd+bwd+Adam, 8 views of 1920x1440, 1M gaussians SH3), batched graph-captured step"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", default="c4")
    p.add_argument("--views", type=int, default=0,
                   help="views per step (default: the workload's); a smaller case for profiling")
    p.add_argument("--pool", type=int, default=0,
                   help="use only the first N cameras of the pool (smaller device footprint, "
                        "for profiler captures); 0 = the workload's pool")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--px", default="",
                   help="pixels per thread 'F,B' for compositing and its adjoint "
                        "(default: the autotuner picks)")
    p.add_argument("--quality", action="store_true",
                   help="train the batched and the plain form side by side for --steps steps "
                        "and report their PSNR (c4, or c3 for the phone-shape schedule)")
    p.add_argument("--dry-run", action="store_true",
                   help="launch and rank protocol only, on CPU over gloo (no device)")
    return p.parse_args()


# The benchmark workloads; "c4" is the headline. They equal
# parallax_b200.scenes.WORKLOADS (tests/test_bench_names.py), restated here so
# the reference arm never imports the product package.
BENCH_WORKLOADS = {
    "c4": dict(gaussians=1_000_000, sh_degree=3, views_per_step=8, pool=64, width=1920,
               height=1440, layout=0),
}


def workload_config(name, w, V, pool):
    """The `config` of the JSON line; both arms print the same one."""
    return {"workload": f"{name}: {w['gaussians']} gaussians SH{w['sh_degree']}, {V} views/step "
                        f"at {w['width']}x{w['height']} from a {pool}-camera pool, "
                        "fwd+L1/SSIM+bwd+Adam",
            "gaussians": w["gaussians"], "sh_degree": w["sh_degree"], "views_per_step": V,
            "pool": pool, "width": w["width"], "height": w["height"],
            "l2": "inputs larger than L2 (no flush)"}


def view_ids(step, V, pool, rank=0):
    """The views of `step` on `rank`: V consecutive cameras of the pool."""
    base = (step * V + rank * 7) % pool
    return [(base + i) % pool for i in range(V)]


def free_port():
    import socket

    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def spawn_ranks(args) -> int:
    """Starts args.gpus ranks of this script (one per GPU) and waits for them.
    Rank 0 prints the JSON line. If a rank fails, the others get the process
    group's timeout to end on their own, then are stopped."""
    port = free_port()
    procs = []
    for r in range(args.gpus):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(args.gpus),
                   LOCAL_WORLD_SIZE=str(args.gpus), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.abspath(__file__)] + sys.argv[1:],
                                      env=env))
    rc, failed_at = 0, None
    while any(p.poll() is None for p in procs):
        for p in procs:
            if p.poll() not in (None, 0) and failed_at is None:
                failed_at = time.time()
        if failed_at is not None and time.time() - failed_at > 240:
            for p in procs:
                if p.poll() is None:
                    p.kill()
        time.sleep(0.2)
    for p in procs:
        rc = rc or p.returncode
    return rc


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ------------------------------------------------------------- clocks


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples every 50 ms. `start` waits
    for the first sample, so that the sampler is running before the timed
    region opens; `mark` brackets the timed region, and `stop` keeps the
    samples whose timestamps fall inside it (the nearest one when the region
    is shorter than the interval)."""
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None
        self.window = None

    def start(self, wait_s: float = 10.0):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.file,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        deadline = time.time() + wait_s
        while time.time() < deadline and self.proc.poll() is None:
            if os.path.getsize(self.file.name) > 0:
                break
            time.sleep(0.02)

    def mark(self, t_begin: float, t_end: float):
        self.window = (t_begin, t_end)

    @staticmethod
    def _time_of(stamp: str):
        for fmt in ("%Y/%m/%d %H:%M:%S.%f", "%Y/%m/%d %H:%M:%S"):
            try:
                return datetime.datetime.strptime(stamp, fmt).timestamp()
            except ValueError:
                pass
        return None

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 10:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        kept = rows
        if self.window is not None:
            t0, t1 = self.window
            stamped = [(self._time_of(r[0]), r) for r in rows]
            inside = [r for t, r in stamped if t is not None and t0 <= t <= t1]
            if inside:
                kept = inside
            else:
                timed = [(abs(t - 0.5 * (t0 + t1)), r) for t, r in stamped if t is not None]
                kept = [min(timed, key=lambda x: x[0])[1]] if timed else rows[-1:]
        sm = [float(r[2]) for r in kept if r[2].replace(".", "").isdigit()]
        smax = [float(r[3]) for r in kept if r[3].replace(".", "").isdigit()]
        reasons = sorted({self.REASONS[i] for r in kept for i in range(4) if r[6 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(kept), "interval_ms": 50}


# ------------------------------------------------------ reference CPU trainer


def reference_step(workload, V, pool, threads, steps_needed):
    """The reference's own CPU trainer on the workload (oracle/ref_bench.py),
    with targets rendered for the views of the first `steps_needed` steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_bench

    w = BENCH_WORKLOADS[workload]
    needed = sorted({i for s in range(steps_needed) for i in view_ids(s, V, pool)})
    return ref_bench.ReferenceBatchStep(
        w["gaussians"], w["sh_degree"], pool, w["width"], w["height"], threads,
        target_views=needed, log=lambda m: print(m, file=sys.stderr, flush=True))


def reference_sample(w, V, threads):
    return (f"whole steps of the reference's CPU trainer (oracle/_ref/libpxref_fast.so, its "
            f"-O3 -ffast-math release flags): per step {V} views of {w['width']}x{w['height']}, "
            f"each projectSplats + rasterizeSplats + photometricLoss + rasterizeSplatsBackward "
            f"(CpuSplatBackend::renderAndAccumulate) on its own host thread ({threads} threads), "
            f"gradients added, then SplatTrainer's own Adam step over {w['gaussians']} gaussians "
            f"SH{w['sh_degree']}; nothing extrapolated")


# ------------------------------------------------------------ our arm


def stage_work(w, P, N, V, K, E, Q, pixels):
    """Algorithmic work per stage: (bytes, flops)."""
    return {
        "project": (N * (4 * P + 52 * V), 0),
        "bin": (K * 24, 0),
        "forward": (0, 17 * E + 10 * Q),
        "loss": (0, 480 * 3 * pixels),
        "backward": (0, 17 * E + 58 * Q),
        "param_grads": (N * (4 * P * 2 + 92 * V), 0),
        "adam": (28 * N * P, 0),
    }


def run_ours(args):
    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import parallax_b200 as px
    from parallax_b200.scenes import WORKLOADS, workload_scene

    w = WORKLOADS[args.workload]
    V = args.views or w["views_per_step"]
    truth, start, views = workload_scene(args.workload)
    if args.pool > 0:
        views = views[:args.pool]
    P = px.param_count(start.rest_per_channel)
    N = start.count

    # targets: the truth cloud rendered on the device, kept in pinned host memory
    opts = px.RasterOptions(sh_degree=w["sh_degree"])
    lib = px.lib()
    renderer = px.SplatTrainer(truth, [], px.TrainConfig(iterations=1))
    pinned = []
    for view in views:
        buf = torch.empty(view.width * view.height * 3, dtype=torch.float32, pin_memory=True)
        arr = buf.numpy()
        cam = view.camera()
        renderer._check(lib.pxs_trainer_render(renderer.handle, ct.byref(cam), ct.byref(opts),
                                               arr.ctypes.data, None))
        pinned.append((buf, arr))
    renderer.close()
    del renderer
    # the same targets as 8-bit frames, the reference's image format before
    # downscaleToWidth; the trainer trains on frame / 255 (ingested on the device)
    frames = []
    for _, arr in pinned:
        fbuf = torch.empty(arr.size, dtype=torch.uint8, pin_memory=True)
        fbuf.numpy()[:] = np.rint(np.clip(arr, 0.0, 1.0) * 255.0).astype(np.uint8)
        frames.append(fbuf)

    cfg = px.TrainConfig(iterations=100000, sh_degree=w["sh_degree"], sh_increase_interval=0,
                         densify_from_iteration=10 ** 9, densify_until_iteration=10 ** 9,
                         opacity_reset_interval=0, max_gaussians=max(600000, N))
    trainer = px.SplatTrainer(start, [(v.camera(), arr) for v, (_, arr) in zip(views, pinned)],
                              cfg, device=local)
    def ingest(ids):
        id_arr = (ct.c_int32 * len(ids))(*ids)
        ptrs = (ct.c_void_p * len(ids))(*[frames[i].data_ptr() for i in ids])
        ws = (ct.c_int32 * len(ids))(*[views[i].width for i in ids])
        hs = (ct.c_int32 * len(ids))(*[views[i].height for i in ids])
        trainer._check(lib.pxs_trainer_ingest_images(trainer.handle, len(ids), id_arr, ptrs,
                                                     ws, hs))

    ingest(list(range(len(views))))
    sp = ct.c_void_p()
    trainer._check(lib.pxs_trainer_stream(trainer.handle, ct.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value)
    pool = len(views)

    def ids_for(step):
        return view_ids(step, V, pool, rank)

    if world > 1:
        # data parallel over views: each rank renders its own V views, the
        # gradient buffers are summed over the ranks, every rank takes the
        # same Adam step
        from parallax_b200.data_parallel import DataParallelStep
        dp_step = DataParallelStep(trainer, device="cuda")

        def batch_step(step, graph=True):
            return dp_step(ids_for(step))
    else:
        def batch_step(step, graph=True):
            return trainer.step_batch(V, ids_for(step), graph=graph)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def timed(fn, steps):
        barrier()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for s in range(steps):
            fn(s)
        b.record(stream)
        b.synchronize()
        torch.cuda.synchronize()
        barrier()
        ms = a.elapsed_time(b) / steps
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    step_counter = [0]

    def next_batch(_):
        step_counter[0] += 1
        batch_step(step_counter[0])

    # the autotuner picks pixels per thread for compositing and its adjoint
    fpx, bpx = ct.c_int32(), ct.c_int32()
    if args.px:
        f_, b_ = (int(x) for x in args.px.split(","))
        trainer._check(lib.pxs_set_raster_config(f_, b_))
        lib.pxs_get_raster_config(ct.byref(fpx), ct.byref(bpx))
    else:
        ids0 = (ct.c_int32 * V)(*ids_for(0))
        trainer._check(lib.pxs_trainer_autotune(trainer.handle, V, ids0, ct.byref(fpx),
                                                ct.byref(bpx)))

    sched = [ct.c_int32() for _ in range(4)]
    lib.pxs_get_raster_schedule(*[ct.byref(x) for x in sched])
    tuning = {"pixels_per_thread": {"forward": fpx.value, "backward": bpx.value},
              "entry_batch": {"forward": sched[0].value, "backward": sched[1].value},
              "tile_schedule": {"forward": sched[2].value, "backward": sched[3].value},
              "schedules": "0 one CTA per tile, 1 heaviest tiles first, 2 persistent"}
    if not args.px:
        report = ct.create_string_buffer(8192)
        trainer._check(lib.pxs_trainer_autotune_report(trainer.handle, report, 8192))
        tuning["measured"] = [ln for ln in report.value.decode().splitlines() if ln]

    # warm-up: capture the graph, then once more with stage timing on
    for _ in range(max(args.warmup, 3)):
        next_batch(0)
    trainer._check(lib.pxs_trainer_set_timing(trainer.handle, 1))
    next_batch(0)
    trainer._check(lib.pxs_trainer_set_timing(trainer.handle, 1))  # reset the totals

    clocks = ClockSampler(local)
    clocks.start()
    t_begin = time.time()
    ms_batched = timed(next_batch, args.steps)
    clocks.mark(t_begin, time.time())
    clock_info = clocks.stop()

    stage_ms = (ct.c_float * len(STAGES))()
    n_stages, n_steps = ct.c_int32(), ct.c_int32()
    trainer._check(lib.pxs_trainer_stage_times(trainer.handle, stage_ms, len(STAGES),
                                               ct.byref(n_stages), ct.byref(n_steps)))
    per_stage = {s: stage_ms[i] / max(n_steps.value, 1) for i, s in enumerate(STAGES)}
    pairs, launches = ct.c_int64(), ct.c_int64()
    trainer._check(lib.pxs_trainer_step_info(trainer.handle, ct.byref(pairs), ct.byref(launches)))
    kernels_per_step = launches.value
    evaluated, contributing = ct.c_int64(), ct.c_int64()
    trainer._check(lib.pxs_trainer_pair_stats(trainer.handle, ct.byref(evaluated),
                                              ct.byref(contributing)))
    trainer._check(lib.pxs_trainer_set_timing(trainer.handle, 0))
    next_batch(0)  # re-capture without the timing events

    result = {}
    ms_plain = None
    if not args.no_plain and world == 1:
        def plain_step(_):
            step_counter[0] += 1
            trainer.step_views(V, ids_for(step_counter[0]))
        plain_step(0)
        ms_plain = timed(plain_step, max(3, args.steps // 2))

    e2e = None
    if not args.no_e2e:
        def stage(ids):
            id_arr = (ct.c_int32 * len(ids))(*ids)
            ptrs = (ct.c_void_p * len(ids))(*[frames[i].data_ptr() for i in ids])
            ws = (ct.c_int32 * len(ids))(*[views[i].width for i in ids])
            hs = (ct.c_int32 * len(ids))(*[views[i].height for i in ids])
            trainer._check(lib.pxs_trainer_stage_images(trainer.handle, len(ids), id_arr, ptrs,
                                                        ws, hs))

        # The feeding loop of a training job: every step's 8-bit frames cross
        # from pinned host memory, staged one step ahead so the copy overlaps
        # the step before (pxs_trainer_stage_images), are converted on the
        # device, the step runs and its loss is read back. Exactly `steps`
        # frame sets are copied inside the timed region, one per step.
        def timed_e2e(steps):
            barrier()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            first = step_counter[0] + 1
            stage(ids_for(first))
            for k in range(steps):
                if k + 1 < steps:
                    stage(ids_for(first + k + 1))
                batch_step(first + k)  # reads the loss back to the host
            step_counter[0] = first + steps - 1
            b.record(stream)
            b.synchronize()
            torch.cuda.synchronize()
            barrier()
            ms = a.elapsed_time(b) / steps
            if world > 1:
                import torch.distributed as dist
                t = torch.tensor([ms], device="cuda")
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                ms = float(t.item())
            return ms

        # the same without overlap: ingest (synchronous), then the step
        def e2e_serial_step(_):
            step_counter[0] += 1
            ingest(ids_for(step_counter[0]))
            batch_step(step_counter[0])

        # the same with the targets uploaded as FP32 images (pxs_trainer_set_images)
        def e2e_float_step(_):
            step_counter[0] += 1
            ids = ids_for(step_counter[0])
            id_arr = (ct.c_int32 * V)(*ids)
            ptrs = (ct.c_void_p * V)(*[pinned[i][1].ctypes.data for i in ids])
            trainer._check(lib.pxs_trainer_set_images(trainer.handle, V, id_arr, ptrs))
            batch_step(step_counter[0])

        timed_e2e(2)  # warm the staging buffers and the graph
        ms_e2e = timed_e2e(args.steps)
        h2d = sum(views[i].width * views[i].height * 3 for i in ids_for(0))
        e2e_serial_step(0)
        ms_e2e_serial = timed(e2e_serial_step, args.steps)
        e2e_float_step(0)
        ms_e2e_float = timed(e2e_float_step, args.steps)
        # restore the 8-bit targets of the views the float leg replaced
        ingest(list(range(len(views))))
        e2e = {"value": world * 1000.0 / ms_e2e, "unit": "steps/s", "ms_per_step": ms_e2e,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 4 + 4,
               "inputs": "8-bit RGB frames at the view size from pinned host memory, staged "
                         "one step ahead on a copy stream and converted on the device",
               "serial": {"value": world * 1000.0 / ms_e2e_serial,
                          "ms_per_step": ms_e2e_serial, "h2d_bytes_per_step": h2d,
                          "inputs": "the same frames ingested synchronously before each step"},
               "fp32_targets": {"value": world * 1000.0 / ms_e2e_float,
                                "ms_per_step": ms_e2e_float, "h2d_bytes_per_step": 4 * h2d,
                                "inputs": "FP32 RGB images (pxs_trainer_set_images)"}}

    # roofline of the dominant kernel and of the whole step
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    hbm_source = "measured" if "hbm_gbs" in peaks else "fallback"
    fp32 = ct.c_float()
    if lib.pxs_measure_fp32_peak(local, ct.byref(fp32)) != 0:
        fp32.value = 74.0
    pixels = sum(views[i].width * views[i].height for i in ids_for(0))
    work = stage_work(w, P, N, V, pairs.value, evaluated.value, contributing.value, pixels)
    dominant = max(per_stage, key=per_stage.get)
    bytes_, flops = work[dominant]
    dom_ms = per_stage[dominant]
    if flops > 0:
        achieved = flops / (dom_ms * 1e-3) / 1e12
        roofline = {"kernel": dominant, "bound": "fp32", "achieved": achieved,
                    "peak": fp32.value, "unit": "TFLOP/s", "frac": achieved / fp32.value,
                    "peak_source": "measured FP32 FMA microkernel (pxs_measure_fp32_peak)"}
    else:
        achieved = bytes_ / (dom_ms * 1e-3) / 1e9
        roofline = {"kernel": dominant, "bound": "hbm", "achieved": achieved, "peak": hbm,
                    "unit": "GB/s", "frac": achieved / hbm,
                    "peak_source": f"{hbm_source} MEASURED_PEAKS.json hbm_gbs"}
    roofline["traffic"] = traffic_from_profiles(dominant)
    roofline["launch_ms"] = dom_ms
    t_roof = 0.0
    for s, (b_, f_) in work.items():
        t_roof += max(b_ / (hbm * 1e9), f_ / (fp32.value * 1e12))
    step_roofline = {"t_roofline_ms": t_roof * 1e3, "t_measured_ms": ms_batched,
                     "frac": t_roof * 1e3 / ms_batched}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload in BENCH_WORKLOADS:
        # one whole step of the reference's CPU trainer on this workload: a
        # bounded sample (about half a minute on the host cores)
        try:
            threads = min(V, os.cpu_count() or 1)
            ref = reference_step(args.workload, V, pool, threads, 1)
            t0 = time.perf_counter()
            ref.step(view_ids(0, V, pool))
            seconds = time.perf_counter() - t0
            ref.close()
            cpu = {"value": 1.0 / seconds, "unit": "steps/s", "cores": threads,
                   "kind": "reference", "sample": "one " + reference_sample(w, V, threads)[6:],
                   "seconds_per_step": seconds, "host_cores": os.cpu_count()}
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "steps/s", "cores": 0, "kind": "unavailable",
                   "sample": f"failed: {exc}"}

    line = {
        "metric": METRIC,
        "value": world * 1000.0 / ms_batched,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_batched,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": DATA,
        "config": workload_config(args.workload, w, V, pool),
        "parallelism": f"dp{world} over views, one GPU per rank",
        "tuning": tuning,
        "plain": {"ms_per_step": ms_plain,
                  "value": world * 1000.0 / ms_plain if ms_plain else None,
                  "batched_over_plain": (ms_plain / ms_batched) if ms_plain else None,
                  "form": "per-view kernel sequences, host-synchronised pair counts, no graph"},
        "e2e": e2e,
        "gpu_launches": kernels_per_step * args.steps,
        "kernels_per_step": kernels_per_step,
        "stage_ms": per_stage,
        "pairs_per_step": pairs.value,
        "evaluated_pairs": evaluated.value,
        "contributing_pairs": contributing.value,
        "roofline": roofline,
        "step_roofline": step_roofline,
        "cpu_baseline": cpu,
        "clocks": clock_info,
    }
    trainer.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def run_multi_scene(args):
    """The uneven batch of independent scans: 32 scenes (5k-150k gaussians SH3,
    320x240 / 640x480 / 1280x720), 4 views each; one step renders and
    differentiates all 128 views in one pass of each kernel and takes every
    scene's Adam step (a multi-scene trainer, pxs_trainer_create_scenes)."""
    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    import parallax_b200 as px
    from parallax_b200.scenes import MULTI_SCENE, multi_scene_workload

    scenes = multi_scene_workload(5)
    lib = px.lib()
    opts = px.RasterOptions(sh_degree=MULTI_SCENE["sh_degree"])
    scene_views, starts = [], []
    for truth, start, views in scenes:
        renderer = px.SplatTrainer(truth, [], px.TrainConfig(iterations=1))
        pairs = []
        for view in views:
            arr = np.empty(view.width * view.height * 3, dtype=np.float32)
            cam = view.camera()
            renderer._check(lib.pxs_trainer_render(renderer.handle, ct.byref(cam),
                                                   ct.byref(opts), arr.ctypes.data, None))
            pairs.append((cam, arr))
        renderer.close()
        scene_views.append(pairs)
        starts.append(start)
    cfg = px.TrainConfig(iterations=100000, sh_degree=MULTI_SCENE["sh_degree"],
                         sh_increase_interval=0, densify_from_iteration=10 ** 9,
                         densify_until_iteration=10 ** 9, opacity_reset_interval=0)
    trainer = px.SplatTrainer.from_scenes(starts, scene_views, cfg, device=local)
    n_views = sum(len(v) for v in scene_views)
    ids = list(range(n_views))
    sp = ct.c_void_p()
    trainer._check(lib.pxs_trainer_stream(trainer.handle, ct.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value)
    fpx, bpx = ct.c_int32(), ct.c_int32()
    id_arr = (ct.c_int32 * n_views)(*ids)
    trainer._check(lib.pxs_trainer_autotune(trainer.handle, n_views, id_arr, ct.byref(fpx),
                                            ct.byref(bpx)))
    for _ in range(max(args.warmup, 3)):
        trainer.step_batch(n_views, ids)
    trainer._check(lib.pxs_trainer_set_timing(trainer.handle, 1))
    trainer.step_batch(n_views, ids)
    trainer._check(lib.pxs_trainer_set_timing(trainer.handle, 1))
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.steps):
        trainer.step_batch(n_views, ids)
    b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b) / args.steps
    stage_ms = (ct.c_float * len(STAGES))()
    n_stages, n_steps = ct.c_int32(), ct.c_int32()
    trainer._check(lib.pxs_trainer_stage_times(trainer.handle, stage_ms, len(STAGES),
                                               ct.byref(n_stages), ct.byref(n_steps)))
    pairs, launches = ct.c_int64(), ct.c_int64()
    trainer._check(lib.pxs_trainer_step_info(trainer.handle, ct.byref(pairs), ct.byref(launches)))
    counts = [c.count for c in starts]
    line = {
        "metric": "train steps/s (fwd+bwd+Adam), 32 independent scenes x 4 views in one "
                  "batched graph-captured step",
        "value": 1000.0 / ms, "unit": "steps/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic (seeded: scene s truth cloud 1000+2s, start 1001+2s, cameras 3000+s)",
        "config": {"workload": f"c5: {len(starts)} scenes, {sum(counts)} gaussians "
                               f"({min(counts)}..{max(counts)}) SH{MULTI_SCENE['sh_degree']}, "
                               f"{n_views} views of 320x240 / 640x480 / 1280x720",
                   "pixels_per_thread": {"forward": fpx.value, "backward": bpx.value}},
        "gpu_launches": launches.value * args.steps, "kernels_per_step": launches.value,
        "pairs_per_step": pairs.value,
        "stage_ms": {s: stage_ms[i] / max(n_steps.value, 1) for i, s in enumerate(STAGES)},
    }
    trainer.close()
    print(json.dumps(line))


def psnr(rendered, target):
    """10 log10(1 / MSE) over linear RGB clamped to [0, 1]."""
    mse = float(np.mean((np.clip(rendered, 0.0, 1.0) - target) ** 2))
    return 10.0 * np.log10(1.0 / max(mse, 1e-20))


def run_quality(args):
    """Equal quality of the batched (graph-captured) form and the plain form.

    c4: both forms train the C4 scene for `--steps` steps (8 views per step, the
        benchmark's view schedule) from the same start; PSNR over the 64 pool
        views.
    c3: the phone-shape schedule (200k gaussians SH3, 64 cameras at 1280x720,
        7000 iterations, densify/prune every 100 steps in [500, 5000], opacity
        reset, SH bands unlocked every 1000): one trainer steps with
        pxs_trainer_step_views over one view (per-view kernels, host-
        synchronised), the other with one-view graph-captured batched steps on
        the same schedule; final gaussian counts and PSNR over the 64 training
        views.
    """
    import torch

    import parallax_b200 as px
    from parallax_b200.scenes import WORKLOADS, workload_scene

    torch.cuda.set_device(0)
    w = WORKLOADS[args.workload]
    truth, start, views = workload_scene(args.workload)
    lib = px.lib()
    opts = px.RasterOptions(sh_degree=w["sh_degree"])
    renderer = px.SplatTrainer(truth, [], px.TrainConfig(iterations=1))
    targets = []
    for view in views:
        arr = np.empty(view.width * view.height * 3, dtype=np.float32)
        cam = view.camera()
        renderer._check(lib.pxs_trainer_render(renderer.handle, ct.byref(cam), ct.byref(opts),
                                               arr.ctypes.data, None))
        targets.append(np.rint(np.clip(arr, 0, 1) * 255.0).astype(np.float32) / np.float32(255))
    renderer.close()
    pairs = [(v.camera(), t) for v, t in zip(views, targets)]
    if args.workload == "c4":
        cfg = px.TrainConfig(iterations=100000, sh_degree=w["sh_degree"], sh_increase_interval=0,
                             densify_from_iteration=10 ** 9, densify_until_iteration=10 ** 9,
                             opacity_reset_interval=0, max_gaussians=max(600000, start.count))
    else:
        cfg = px.TrainConfig(iterations=args.steps, sh_degree=w["sh_degree"])
    forms = {"batched": px.SplatTrainer(start, pairs, cfg), "plain": px.SplatTrainer(start, pairs, cfg)}
    V, pool = w["views_per_step"], len(views)
    t0 = time.perf_counter()
    losses = {k: [] for k in forms}
    for s in range(args.steps):
        if args.workload == "c4":
            ids = view_ids(s, V, pool)
            losses["batched"].append(forms["batched"].step_batch(V, ids, graph=True))
            losses["plain"].append(forms["plain"].step_views(V, ids))
        else:
            if forms["plain"].state()["iteration"] >= cfg.iterations:
                break
            losses["plain"].append(forms["plain"].step_views(1))
            losses["batched"].append(forms["batched"].step_batch(1, None, graph=True))
    seconds = time.perf_counter() - t0
    result = {"quality": args.workload, "steps": args.steps, "seconds": seconds,
              "psnr_definition": "10 log10(1/MSE), linear RGB clamped to [0,1], mean over "
                                 f"the {pool} training views"}
    for name, t in forms.items():
        values = []
        for view, target in zip(views, targets):
            arr = np.empty(view.width * view.height * 3, dtype=np.float32)
            cam = view.camera()
            t._check(lib.pxs_trainer_render(t.handle, ct.byref(cam), None, arr.ctypes.data, None))
            values.append(psnr(arr, target))
        st = t.state()
        result[name] = {"psnr_db": float(np.mean(values)), "gaussians": st["count"],
                        "iteration": st["iteration"], "last_loss": st["last_loss"],
                        "smoothed_loss": st["smoothed_loss"]}
        t.close()
    result["psnr_delta_db"] = result["batched"]["psnr_db"] - result["plain"]["psnr_db"]
    print(json.dumps(result))


def traffic_from_profiles(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    try:
        return json.load(open(path)).get(kernel)
    except (OSError, ValueError):
        return None


# ------------------------------------------------------- reference arm


def run_reference(args):
    """The reference's CPU trainer on the workload and view schedule of our arm
    (rank 0 only; other ranks exit at once). Never imports the product."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    n_gpus = world if "WORLD_SIZE" in os.environ else args.gpus
    if args.workload not in BENCH_WORKLOADS:
        print(json.dumps({"impl": "reference",
                          "unavailable": f"no reference arm for workload {args.workload}"}))
        return
    w = BENCH_WORKLOADS[args.workload]
    V = args.views or w["views_per_step"]
    pool = args.pool or w["pool"]
    threads = min(V, os.cpu_count() or 1)
    try:
        ref = reference_step(args.workload, V, pool, threads, args.warmup + args.steps)
    except Exception as exc:
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU build: {exc}"}))
        return
    for s in range(args.warmup):
        ref.step(view_ids(s, V, pool))
        print(f"reference warm-up step {s + 1}/{args.warmup}", file=sys.stderr, flush=True)
    t0 = time.perf_counter()
    for s in range(args.steps):
        ref.step(view_ids(args.warmup + s, V, pool))
    seconds = (time.perf_counter() - t0) / max(args.steps, 1)
    ref.close()
    value = 1.0 / seconds
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "steps/s",
        "n_gpus": n_gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": seconds * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": DATA,
        "config": workload_config(args.workload, w, V, pool),
        "parallelism": f"host threads, one view each ({threads} threads)",
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads,
                         "kind": "reference", "sample": reference_sample(w, V, threads),
                         "host_cores": os.cpu_count()},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "final_loss": ref.loss,
    }
    print(json.dumps(line))


def run_dry(args):
    """The launch and rank protocol of the multi-GPU run without a device:
    every rank joins a gloo group, reports, and the ranks agree on a maximum
    time the way the timed region does."""
    import datetime

    import torch
    import torch.distributed as dist

    world, rank, local = dist_env()
    print(f"rank {rank} of {world} started (local rank {local})", file=sys.stderr, flush=True)
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    t = torch.tensor([float(rank + 1)])
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": None, "unit": "steps/s", "n_gpus": world,
                          "dry_run": True, "max_over_ranks": float(t.item())}))


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args))
    if args.dry_run:
        run_dry(args)
    elif args.quality:
        run_quality(args)
    elif args.workload == "c5":
        run_multi_scene(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

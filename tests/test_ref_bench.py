"""The benchmark's reference arm (oracle/ref_bench.py) runs the same scene as
the product arm and the reference's own trainer arithmetic.

CPU only: the reference compiled from its sources (oracle/_ref) and the C
restatement.
"""
from __future__ import annotations

import ctypes as ct
import os
import sys

import numpy as np
import pytest

import oracle_lib as O
import parallax_b200 as px
from parallax_b200._abi import RasterOptions, TrainConfig, as_ptr
from parallax_b200.scenes import orbit_views

sys.path.insert(0, O.ORACLE_DIR)
import ref_bench  # noqa: E402

needs_ref = pytest.mark.skipif(not O.ref_available("fast") or not O.ref_available("ieee"),
                               reason="oracle/_ref not built")


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@needs_ref
@pytest.mark.parametrize("kind", ["fast", "ieee"])
def test_reference_arm_clouds_are_the_product_clouds(kind):
    lib = ref_bench.library(kind)
    for seed, count, sh in [(1, 3000, 3), (2, 2000, 0), (5, 1000, 1)]:
        ours = px.synthetic_cloud(seed, count, sh).params
        theirs = ref_bench.synthetic_cloud(lib, seed, count, sh)
        assert np.array_equal(bits(ours), bits(theirs)), (seed, count, sh)


def test_reference_arm_cameras_are_the_product_cameras():
    for count, w, h in [(64, 1920, 1440), (7, 320, 240)]:
        K, R, t = ref_bench.orbit_cameras(3, count, w, h)
        views = orbit_views(3, count, w, h)
        for i, v in enumerate(views):
            assert tuple(K[i]) == tuple(v.K)
            assert np.array_equal(R[i], np.asarray(v.R).reshape(9))
            assert np.array_equal(t[i], np.asarray(v.t).reshape(3))


@needs_ref
def test_reference_batch_step_is_summed_views_then_the_reference_adam():
    """One step of the batched reference trainer equals the reference's
    renderAndAccumulate over each view of the batch, summed in view order,
    followed by the reference's Adam step (its oracle restatement is pinned to
    SplatTrainer::step bit for bit in test_oracle.py)."""
    n, sh, pool, w, h = 1500, 3, 5, 64, 48
    batch = [3, 0, 4]
    step = ref_bench.ReferenceBatchStep(n, sh, pool, w, h, threads=2, kind="ieee")
    loss = step.step(batch)
    after = step.cloud()
    step.close()

    lib = ref_bench.library("ieee")
    truth = ref_bench.synthetic_cloud(lib, 1, n, sh)
    start = ref_bench.synthetic_cloud(lib, 2, n, sh)
    rest = ref_bench.rest_per_channel(sh)
    K, R, t = ref_bench.orbit_cameras(3, pool, w, h)
    views = [O.View(tuple(K[i]), w, h, R[i].reshape(3, 3), t[i]) for i in range(pool)]
    opt = RasterOptions(sh_degree=sh)
    grads = np.zeros_like(start)
    losses = []
    for v in batch:
        rgb, _ = O.ref_render(truth, rest, sh, views[v], opt)
        target = np.rint(np.clip(rgb, 0, 1) * 255.0).astype(np.uint8).astype(np.float32)
        target /= np.float32(255.0)
        lv, g, _, _ = O.oracle_render_and_accumulate(start, rest, sh, views[v].camera(), opt,
                                                     target, 0.2)
        grads += g
        losses.append(lv)
    assert abs(loss - np.float32(sum(losses)) / np.float32(len(losses))) <= 1e-6 * loss

    cfg = TrainConfig(iterations=100000, sh_degree=sh, sh_increase_interval=0,
                      densify_from_iteration=10 ** 9, densify_until_iteration=10 ** 9,
                      opacity_reset_interval=0, max_gaussians=600000)
    extent = np.float32(O.RefTrainer(start, rest, sh, views, [np.zeros(w * h * 3, np.float32)]
                                     * pool, cfg).state()["extent"])
    libm = ct.CDLL("libm.so.6")
    libm.powf.restype = ct.c_float
    libm.powf.argtypes = [ct.c_float, ct.c_float]
    f = np.float32
    ratio = f(cfg.position_lr_final) / f(cfg.position_lr_initial)
    lr = np.array([f(f(cfg.position_lr_initial) * f(libm.powf(ratio, 0.0))) * extent,
                   cfg.scale_lr, cfg.rotation_lr, cfg.opacity_lr, cfg.dc_lr,
                   f(cfg.dc_lr) / f(cfg.sh_rest_lr_divider)], dtype=np.float32)
    c1 = f(1) - f(libm.powf(cfg.adam_beta1, 1.0))
    c2 = f(1) - f(libm.powf(cfg.adam_beta2, 1.0))
    p, m, v = start.copy(), np.zeros_like(start), np.zeros_like(start)
    O.pxo().pxo_adam_f32(as_ptr(p), as_ptr(grads), as_ptr(m), as_ptr(v), n, rest, as_ptr(lr),
                         ct.c_float(cfg.adam_beta1), ct.c_float(cfg.adam_beta2),
                         ct.c_float(cfg.adam_epsilon), ct.c_float(c1), ct.c_float(c2))
    assert np.array_equal(bits(p), bits(after))


def test_reference_arm_does_not_load_the_product_library():
    """bench.py --impl reference runs in a process that never maps libpxs.so."""
    import subprocess

    code = ("import sys; sys.path.insert(0, %r); import ref_bench; "
            "print(open('/proc/self/maps').read().count('libpxs.so'))" % O.ORACLE_DIR)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         check=True)
    assert out.stdout.strip() == "0"
    src = open(os.path.join(O.ROOT, "bench.py")).read()
    body = src[src.index("def run_reference"):]
    body = body[:body.index("\ndef ", 1)]
    assert "parallax_b200" not in body

"""Quality checks on whole workloads, beyond the per-kernel parity tests.

* The adjoint check at the C2 shape: 4000 gaussians, SH degree 3 (coefficients
  N(0, 0.1)), 4 views at 128x128, loss L1 + 0.2 D-SSIM summed over the views.
  The device's FP32 gradient is compared with FP64 central differences
  (relative step 1e-4) of the oracle's double instantiation on every parameter
  type, and with the reference's own CPU gradient. The reference's gradient
  check (SplatRasterTest.cpp:341-415) turns the alpha floor and the
  transmittance cutoff off, since a pixel crossing either makes the loss jump;
  so does this one. Tolerance: 1e-4, normwise per parameter group.
* Training quality: the batched graph-captured step and the plain per-view
  step train the same scene to the same PSNR (within 0.05 dB), PSNR being
  10 log10(1 / MSE) over linear RGB clamped to [0, 1], averaged over the views.

Each test prints the errors it measured.
"""
from __future__ import annotations

import math
import multiprocessing as mp
import os

import numpy as np
import pytest

import oracle_lib as O
import parallax_b200 as px
from parallax_b200._abi import RasterOptions, TrainConfig

pytestmark = pytest.mark.gpu

GROUPS = {"position": slice(0, 3), "log_scale": slice(3, 6), "rotation": slice(6, 10),
          "opacity": slice(10, 11), "dc": slice(11, 14), "sh_rest": slice(14, None)}


_FD = {}


def _fd_init(params, rest, cams, opt, targets, tests_dir):
    import sys
    sys.path.insert(0, tests_dir)
    _FD.update(p64=params.astype(np.float64), rest=rest, cams=cams, opt=opt,
               targets=[t.astype(np.float64) for t in targets])


def _fd_task(item):
    """Central difference of the summed FP64 loss in parameter (c, g), or NaN
    when the loss jumps inside the step.

    The loss is smooth in every parameter except where the depth order of two
    overlapping splats changes: moving a position can swap it with a neighbour
    and make the composited colour jump. For positions the difference at the
    relative step 1e-4 is checked against steps ten and a hundred times
    smaller; the largest step that agrees with the next one (1e-5 relative)
    is used, and NaN marks a parameter where none agree."""
    import oracle_lib as OL
    c, g = item
    p64 = _FD["p64"]

    def objective(q):
        return sum(OL.oracle_objective_f64(q, _FD["rest"], 3, cam, _FD["opt"], t, 0.2)
                   for cam, t in zip(_FD["cams"], _FD["targets"]))

    def central(h):
        q = p64.copy()
        q[c, g] += h
        plus = objective(q)
        q[c, g] -= 2 * h
        minus = objective(q)
        return (plus - minus) / (2 * h)

    scale = max(abs(p64[c, g]), 1.0)
    first = central(1e-4 * scale)
    if c >= 3:  # not a position
        return first
    values = [first, central(1e-5 * scale), central(1e-6 * scale)]
    for a, b in zip(values, values[1:]):
        if abs(a - b) <= 1e-5 * max(abs(a), abs(b), 1e-12):
            return a
    return float("nan")


def c2_scene():
    params, rest = O.random_cloud(31, 4000, 3, log_scale_mean=-3.0)
    truth, _ = O.random_cloud(32, 4000, 3, log_scale_mean=-3.0)
    views = O.orbit_views(4, 128, 128, seed=33)
    opt = RasterOptions(sh_degree=3, min_alpha=0.0, transmittance_cutoff=0.0)
    targets = [O.oracle_rasterize(O.oracle_project(truth, rest, 3, v.camera(), opt), v.camera(),
                                  opt)[0] for v in views]
    return params, rest, views, opt, targets


def test_c2_gradients_match_fp64_differences_and_the_reference():
    params, rest, views, opt, targets = c2_scene()
    cloud = px.GaussianCloud(params, 3, rest)
    grads = px.SplatGradients.zeros(cloud)
    for v, t in zip(views, targets):
        px.render_and_accumulate(cloud, v.camera(), opt, t, 0.2, grads)
    # the reference's own CPU gradient (SplatTrainer.cpp:104-113), summed over the views
    ref = np.zeros_like(params)
    for v, t in zip(views, targets):
        ref += O.ref_render_and_accumulate(params, rest, 3, v, opt, t, 0.2)[1]
    ref_err = {name: float(np.linalg.norm(grads.params[sl] - ref[sl]) /
                           max(np.linalg.norm(ref[sl]), 1e-30))
               for name, sl in GROUPS.items()}
    print("C2 device vs reference gradient (normwise):", ref_err)
    assert max(ref_err.values()) <= 1e-4, ref_err

    # FP64 central differences on every parameter of a sample of gaussians:
    # the 6 with the largest gradients and 2 more at random among the visible;
    # each difference is two renders of the four views in double precision,
    # spread over the host's cores (a pool started with spawn)
    norms = np.linalg.norm(grads.params, axis=0)
    order = np.argsort(-norms)
    visible = np.nonzero(grads.visible_count > 0)[0]
    rs = np.random.default_rng(7)
    sample = list(order[:6]) + list(rs.choice(np.setdiff1d(visible, order[:6]), 2,
                                               replace=False))
    tasks = [(c, int(g)) for g in sample for c in range(params.shape[0])]
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(16, os.cpu_count() or 1), initializer=_fd_init,
                  initargs=(params, rest, [v.camera() for v in views], opt, targets,
                            os.path.dirname(os.path.abspath(__file__)))) as pool:
        values = pool.map(_fd_task, tasks, chunksize=4)
    fd = np.array(values, dtype=np.float64).reshape(len(sample), params.shape[0]).T
    dev = grads.params[:, sample].astype(np.float64)
    jumps = np.isnan(fd)
    fd_err = {}
    for name, sl in GROUPS.items():
        ok = ~jumps[sl]
        a, b = dev[sl][ok], fd[sl][ok]
        fd_err[name] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))
    print(f"C2 device vs FP64 central differences on {len(sample)} gaussians x "
          f"{params.shape[0]} parameters (normwise):", fd_err,
          f"; {int(jumps.sum())} position parameters excluded (depth-order jump in the step)")
    assert int(jumps.sum()) <= 3 * len(sample) // 2  # most positions are differentiable
    assert max(fd_err.values()) <= 1e-4, fd_err


def psnr(rgb, target):
    mse = float(np.mean((np.clip(rgb, 0, 1) - np.clip(target, 0, 1)) ** 2))
    return 10.0 * math.log10(1.0 / max(mse, 1e-20))


def test_batched_and_plain_training_reach_the_same_psnr():
    params, rest = O.random_cloud(41, 20000, 3, log_scale_mean=-4.0)
    truth, _ = O.random_cloud(42, 20000, 3, log_scale_mean=-4.0)
    views = O.orbit_views(8, 160, 120, seed=43)
    opt = RasterOptions(sh_degree=3)
    images = [px.render_splats(px.GaussianCloud(truth, 3, rest), v.camera(), opt)[0]
              for v in views]
    cfg = TrainConfig(iterations=1000, sh_degree=3, sh_increase_interval=0,
                      densify_from_iteration=10 ** 6, densify_until_iteration=10 ** 6)
    pairs = [(v.camera(), im) for v, im in zip(views, images)]
    scores = {}
    for mode in ("plain", "batched"):
        t = px.SplatTrainer(px.GaussianCloud(params, 3, rest), pairs, cfg)
        for s in range(60):
            ids = [(s * 4 + i) % 8 for i in range(4)]
            if mode == "plain":
                t.step_views(4, ids)
            else:
                t.step_batch(4, ids, graph=True)
        trained = px.GaussianCloud(t.cloud_params(), 3, rest)
        t.close()
        scores[mode] = float(np.mean([psnr(px.render_splats(trained, v.camera(), opt)[0], im)
                                      for v, im in zip(views, images)]))
    start = float(np.mean([psnr(px.render_splats(px.GaussianCloud(params, 3, rest),
                                                 v.camera(), opt)[0], im)
                           for v, im in zip(views, images)]))
    print(f"PSNR start {start:.3f} dB; after 60 steps plain {scores['plain']:.4f} dB, "
          f"batched {scores['batched']:.4f} dB")
    assert scores["batched"] > start + 0.2  # it trained
    assert abs(scores["batched"] - scores["plain"]) <= 0.05


def _c1_run():
    d = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                  "c1_run.npz")))
    n = int(d["n_views"])
    views = [O.View(tuple(d[f"view{i}_K"]), int(d[f"view{i}_size"][0]),
                    int(d[f"view{i}_size"][1]), d[f"view{i}_R"], d[f"view{i}_t"])
             for i in range(n)]
    images = [f.astype(np.float32) / np.float32(255.0) for f in d["frames"]]
    return d, views, images


def _psnr_of(params, views, images):
    cloud = px.GaussianCloud(params, 0, 0)
    out = []
    for v, im in zip(views, images):
        rgb, _ = px.render_splats(cloud, v.camera(), RasterOptions(sh_degree=0))
        mse = float(np.mean((np.clip(rgb, 0, 1).astype(np.float64) - im) ** 2))
        out.append(10.0 * math.log10(1.0 / mse))
    return np.array(out)


def test_c1_trains_like_the_reference_trainer():
    """The plain CPU-runnable configuration end to end (20k gaussians SH0, 16
    views at 320x240, 200 iterations of one view, the reference's default
    schedule) against the reference's own SplatTrainer run stored in
    tests/golden/c1_run.npz: the same view order, the first step's loss
    within 1e-4 (the reference's own float-summation drift), the whole loss
    curve within 1e-3, and the final PSNR within 0.05 dB of the reference's,
    view by view and on average. The engine's SplatTrainer on the CUDA
    backend (the shim) is held to the same."""
    d, views, images = _c1_run()
    start = px.synthetic_cloud(2, 20000, 0)
    cfg = TrainConfig(iterations=200, sh_degree=0)
    runs = {}
    trainer = px.SplatTrainer(start, [(v.camera(), im) for v, im in zip(views, images)], cfg)
    losses = []
    while trainer.step():
        losses.append(trainer.last_loss())
    runs["pxs trainer"] = (np.array(losses), trainer.cloud_params())
    trainer.close()
    if O.ref_available("shim"):
        shim = O.RefTrainer(start.params, 0, 0, views, images, cfg, kind="shim")
        losses = []
        while shim.step():
            losses.append(shim.state()["last_loss"])
        runs["engine trainer on the CUDA backend"] = (np.array(losses), shim.cloud())
    ref_losses = d["losses"].astype(np.float64)
    ref_psnr = d["psnr"]
    for name, (losses, params) in runs.items():
        assert len(losses) == len(ref_losses) == 200
        rel = np.abs(losses - ref_losses) / np.abs(ref_losses)
        psnr = _psnr_of(params, views, images)
        print(f"C1 {name}: loss drift first {rel[0]:.2e}, worst {rel.max():.2e} "
              f"(iteration {int(rel.argmax()) + 1}), final loss {losses[-1]:.6f} "
              f"(reference {ref_losses[-1]:.6f}); PSNR {psnr.mean():.4f} dB "
              f"(reference {ref_psnr.mean():.4f} dB), worst view difference "
              f"{np.abs(psnr - ref_psnr).max():.4f} dB")
        # The reference adds its 230,400 L1 terms and 76,800 SSIM terms into a
        # float one by one (photometricLoss); at this size that sum drifts by a
        # few 1e-5 from the exact one (2.7e-5 measured at the first step). The
        # device sums in double; its loss is held to 1e-5 of an FP64 evaluation
        # in the parity tests.
        assert rel[0] <= 1e-4, (name, rel[0])
        assert rel.max() <= 1e-3, (name, rel.max())
        assert abs(psnr.mean() - ref_psnr.mean()) <= 0.05, name
        assert np.abs(psnr - ref_psnr).max() <= 0.05, name

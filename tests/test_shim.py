"""The drop-in at the engine's own C++ interfaces.

parallax_b200/shim/CudaSplatTrainer.cpp defines parallax::trainSplatsOnGpu
and parallax::splatGpuAvailability with the signatures of the engine's
VulkanSplatTrainer.h:15-37, and parallax::makeCudaSplatBackend() for the
engine's SplatTrainer (SplatTrainer.h:114-135). oracle/Makefile builds it,
together with the engine's own splat sources, into oracle/_ref/libpxshim.so,
linked against parallax_b200/libpxs.so. These tests drive the engine's own
classes through it: the reference's SplatTrainer schedule running on the GPU
backend, and the production trainSplatsOnGpu call.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as O
from parallax_b200._abi import RasterOptions, TrainConfig

# Loss drift allowed over the 60-step trainer run (relative, worst step).
LOSS_DRIFT = 2e-5

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

needs_shim = pytest.mark.skipif(not O.ref_available("shim"),
                                reason="oracle/_ref/libpxshim.so not built")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


@needs_shim
def test_shim_defines_the_engine_symbols():
    out = subprocess.run(["nm", "-D", "-C", "--defined-only", O.ref_path("shim")],
                         capture_output=True, text=True, check=True).stdout
    assert "parallax::splatGpuAvailability()" in out
    assert "parallax::trainSplatsOnGpu(" in out
    assert "parallax::makeCudaSplatBackend(int)" in out


@needs_shim
@pytest.mark.gpu
def test_availability_through_the_engine_signature():
    lib = O.ref("shim")
    available = ct.c_int32()
    name = ct.create_string_buffer(256)
    reason = ct.create_string_buffer(256)
    lib.ref_shim_availability(ct.byref(available), name, 256, reason, 256)
    assert available.value == 1, reason.value
    assert name.value


@needs_shim
@pytest.mark.gpu
@pytest.mark.parametrize("name", ["raster_sh0.npz", "raster_sh3.npz"])
def test_cuda_backend_matches_the_reference_backend(name):
    """SplatBackend::renderAndAccumulate of makeCudaSplatBackend() against the
    reference's CPU backend on the golden case: loss 1e-5 relative, visible
    counts exact, gradients 1e-4 normwise."""
    d = load(name)
    view = O.View(tuple(d["K"]), int(d["size"][0]), int(d["size"][1]), d["R"], d["t"])
    opt = RasterOptions(background=tuple(d["background"]), sh_degree=int(d["sh_degree"]),
                        min_alpha=float(d["min_alpha"]),
                        transmittance_cutoff=float(d["transmittance_cutoff"]),
                        screen_dilation=float(d["screen_dilation"]))
    params, rest, sh = d["params"], int(d["rest"]), int(d["cloud_sh_degree"])
    n = params.shape[1]
    grads = np.zeros_like(params)
    screen = np.zeros(n, dtype=np.float32)
    visible = np.zeros(n, dtype=np.int32)
    loss = O.ref("shim").ref_shim_render_and_accumulate(
        O.as_ptr(params), n, rest, sh, *view.ref_args(), ct.byref(opt), O.as_ptr(d["target"]),
        ct.c_float(0.2), O.as_ptr(grads), O.as_ptr(screen), O.as_ptr(visible))
    r_loss, r_grads, r_screen, r_visible = O.ref_render_and_accumulate(
        params, rest, sh, view, opt, d["target"], 0.2)
    assert abs(loss - r_loss) <= 1e-5 * abs(r_loss)
    assert np.array_equal(visible, r_visible)
    err = np.linalg.norm(grads - r_grads) / np.linalg.norm(r_grads)
    assert err <= 1e-4, err
    assert np.linalg.norm(screen - r_screen) <= 1e-4 * np.linalg.norm(r_screen)


@needs_shim
@pytest.mark.gpu
def test_reference_trainer_runs_on_the_cuda_backend():
    """The engine's SplatTrainer with makeCudaSplatBackend() on the golden
    trainer scene (60 iterations, densify every 20): the densify counts are the
    reference run's and the losses stay within LOSS_DRIFT of it."""
    d = load("trainer_blobs.npz")
    n_views = int(d["n_views"])
    views, images = [], []
    for i in range(n_views):
        views.append(O.View(tuple(d[f"view{i}_K"]), int(d[f"view{i}_size"][0]),
                            int(d[f"view{i}_size"][1]), d[f"view{i}_R"], d[f"view{i}_t"]))
        images.append(d[f"image{i}"])
    cfg = TrainConfig(**{name: d[f"cfg_{name}"].item() for name, _ in TrainConfig._fields_})
    trainer = O.RefTrainer(d["start"], 0, 0, views, images, cfg, kind="shim")
    assert trainer.handle
    losses, counts = [], []
    while trainer.step():
        st = trainer.state()
        losses.append(st["last_loss"])
        counts.append(st["count"])
    assert counts == list(d["counts"])
    rel = np.abs(np.array(losses) - d["losses"]) / np.abs(d["losses"])
    # the first step differs only by the device's summation order; later steps
    # carry that difference forward through Adam and two densify steps
    print("loss drift against the reference run: first step %.2e, worst %.2e (step %d)"
          % (rel[0], rel.max(), int(rel.argmax()) + 1))
    assert rel[0] <= 1e-5, rel[0]
    assert rel.max() <= LOSS_DRIFT, rel.max()
    finished, sh_degree = trainer.finish()
    assert finished.shape == d["finished"].shape
    assert sh_degree == cfg.sh_degree
    assert (np.diff(finished[10]) <= 0).all()


def _views_arrays(views, images):
    K = np.ascontiguousarray(np.array([v.K for v in views], dtype=np.float64).reshape(-1))
    sizes = np.ascontiguousarray(np.array([[v.width, v.height] for v in views],
                                          dtype=np.int32).reshape(-1))
    R = np.ascontiguousarray(np.array([np.asarray(v.R).reshape(9) for v in views],
                                      dtype=np.float64).reshape(-1))
    t = np.ascontiguousarray(np.array([np.asarray(v.t).reshape(3) for v in views],
                                      dtype=np.float64).reshape(-1))
    imgs = [np.ascontiguousarray(im, dtype=np.float32) for im in images]
    ptrs = (ct.c_void_p * len(imgs))(*[im.ctypes.data for im in imgs])
    return K, sizes, R, t, imgs, ptrs


@needs_shim
@pytest.mark.gpu
@pytest.mark.parametrize("cancel_at", [0, 12])
def test_train_splats_on_gpu_through_the_engine_signature(cancel_at):
    """parallax::trainSplatsOnGpu: true, the cloud overwritten in place with
    the finished (pruned, opacity-sorted) cloud, the configured SH degree set;
    a cancelled run still writes back and returns true."""
    truth, _ = O.truth_cloud()
    views = O.ring_of_views(4, 1.6, 16, 16)
    images = [O.oracle_rasterize(O.oracle_project(truth, 0, 0, v.camera(), RasterOptions()),
                                 v.camera(), RasterOptions())[0] for v in views]
    start, _ = O.rough_start(10)
    start[10, 0] = -30.0  # transparent: pruned by finish()
    cfg = TrainConfig(iterations=30, sh_degree=0, sh_increase_interval=0,
                      densify_from_iteration=31, densify_until_iteration=31,
                      opacity_reset_interval=0, max_gaussians=64)
    P, n = start.shape
    buf = np.zeros(P * max(n, cfg.max_gaussians), dtype=np.float32)
    buf[: P * n] = start.reshape(-1)
    K, sizes, R, t, imgs, ptrs = _views_arrays(views, images)
    count, sh, seen = ct.c_int(), ct.c_int(), ct.c_int()
    err = ct.create_string_buffer(512)
    ok = O.ref("shim").ref_shim_train_splats_on_gpu(
        O.as_ptr(buf), n, 0, 0, len(views), O.as_ptr(K), O.as_ptr(sizes), O.as_ptr(R),
        O.as_ptr(t), ptrs, ct.byref(cfg), cancel_at, ct.byref(count), ct.byref(sh),
        ct.byref(seen), err, 512)
    assert ok == 1, err.value
    assert count.value == 9 and sh.value == 0
    out = buf[: P * count.value].reshape(P, count.value)
    assert (np.diff(out[10]) <= 0).all()
    assert np.isfinite(out).all()
    if cancel_at:
        assert seen.value == cancel_at
    else:
        assert seen.value == cfg.iterations


# ------------------------------------------------------ the pipeline's stage
#
# PipelineTest.cpp:704-801 runs the pipeline's splat stage
# (Pipeline::Impl::runSplatTraining, Pipeline.cpp:1844-2009) end to end; the
# pipeline itself needs the whole engine build. ref_shim_pipeline_splat_stage
# (oracle/ref_api.cpp) restates the stage from the coloured point cloud and the
# posed frames on, with trainSplatsOnGpu resolved to the CUDA shim; these
# tests are the PipelineTest cases on it, the field written and read back by
# the reference's own PLY writer and reader.


def capture_scene(frames=10, width=128, height=96):
    """A posed capture: a truth cloud rendered by the reference from an orbit
    as 8-bit frames, and its gaussian centres with their base colours as the
    coloured point cloud the stage seeds from."""
    truth, _ = O.random_cloud(91, 3000, 0, log_scale_mean=-3.5)
    views = O.orbit_views(frames, width, height, seed=9)
    images = []
    for v in views:
        rgb, _ = O.ref_render(truth, 0, 0, v, RasterOptions())
        images.append(np.rint(np.clip(rgb, 0, 1) * 255.0).astype(np.uint8))
    points = np.ascontiguousarray(truth[0:3].T)
    base = np.clip(0.5 + 0.28209479177387814 * truth[11:14].T, 0, 1)
    colors = np.ascontiguousarray(np.rint(base * 255.0).astype(np.uint8))
    return points, colors, views, images


def run_stage(points, colors, views, images, iterations, max_gaussians, sh_degree=0,
              image_width=64, max_views=6, budget_ms=0, cancel_at=0):
    lib = O.ref("shim")
    f = len(views)
    K = np.ascontiguousarray(np.array([v.K for v in views], dtype=np.float64))
    sizes = np.ascontiguousarray(np.array([[v.width, v.height] for v in views], np.int32))
    R = np.ascontiguousarray(np.array([np.asarray(v.R).reshape(9) for v in views], np.float64))
    t = np.ascontiguousarray(np.array([np.asarray(v.t).reshape(3) for v in views], np.float64))
    ptrs = (ct.c_void_p * f)(*[im.ctypes.data for im in images])
    settings = np.array([iterations, max_gaussians, sh_degree, image_width, max_views, budget_ms,
                         cancel_at], dtype=np.int32)
    rest_max = 15
    out = np.zeros((14 + 3 * rest_max) * max_gaussians, dtype=np.float32)
    count, rest, sh, cancelled = ct.c_int32(), ct.c_int32(), ct.c_int32(), ct.c_int32()
    backend, message = ct.create_string_buffer(32), ct.create_string_buffer(512)
    ok = lib.ref_shim_pipeline_splat_stage(
        O.as_ptr(points), O.as_ptr(colors), len(points), f, O.as_ptr(K), O.as_ptr(sizes),
        O.as_ptr(R), O.as_ptr(t), ptrs, O.as_ptr(settings), O.as_ptr(out), max_gaussians,
        ct.byref(count), ct.byref(rest), ct.byref(sh), ct.byref(cancelled), backend, 32,
        message, 512)
    n = max(count.value, 0)
    params = out[:(14 + 3 * rest.value) * n].reshape(14 + 3 * rest.value, n).copy() if n else None
    return dict(success=bool(ok), cancelled=bool(cancelled.value), count=n, rest=rest.value,
                sh=sh.value, backend=backend.value.decode(), message=message.value.decode(),
                params=params)


def reference_ply_roundtrip(params, rest, sh, tmp_path):
    """The field written by the reference's writeGaussianPly and read back by its
    readGaussianPly (both in their own process): (count, valid, least opacity)."""
    tool = os.path.join(os.path.dirname(O.ref_path("ieee")), "ref_writer")
    src, ply = str(tmp_path / "cloud.f32"), str(tmp_path / "splat.ply")
    np.ascontiguousarray(params, dtype=np.float32).tofile(src)
    subprocess.run([tool, src, str(params.shape[1]), str(rest), str(sh), "0", "12", ply],
                   check=True)
    out = subprocess.run([tool, "--read", ply], capture_output=True, text=True, check=True)
    count, valid, least = out.stdout.split()[:3]
    return int(count), int(valid), float(least)


@needs_shim
@pytest.mark.gpu
def test_pipeline_splat_stage_trains_a_field_on_the_cuda_backend(tmp_path):
    """TrainsASplatFieldWhenAskedTo (PipelineTest.cpp:704-748): 60 iterations,
    at most 4000 gaussians, SH 0, 64-pixel-wide views, at most 6 of them. The
    stage succeeds on the GPU path, the field is written and read back by the
    reference, it is valid, and every gaussian survived the final prune."""
    points, colors, views, images = capture_scene()
    r = run_stage(points, colors, views, images, iterations=60, max_gaussians=4000)
    assert r["success"], r["message"]
    assert r["backend"] == "gpu" and "(gpu)" in r["message"]
    assert r["count"] > 0
    count, valid, least = reference_ply_roundtrip(r["params"], r["rest"], r["sh"], tmp_path)
    assert count == r["count"]
    assert valid == 1
    assert least >= 0.0045


@needs_shim
@pytest.mark.gpu
def test_pipeline_splat_stage_stops_at_its_time_budget_and_keeps_the_field(tmp_path):
    """SplatTrainingStopsWhenItsTimeBudgetRunsOutAndKeepsTheField
    (PipelineTest.cpp:750-781): a 1 ms budget on a 100000-iteration schedule.
    Not a failure and not a cancellation: the note says the time budget ran out
    and the partly trained field is kept."""
    points, colors, views, images = capture_scene()
    r = run_stage(points, colors, views, images, iterations=100000, max_gaussians=20000,
                  budget_ms=1)
    assert r["success"], r["message"]
    assert not r["cancelled"]
    assert "time budget" in r["message"], r["message"]
    assert r["backend"] == "gpu"
    assert r["count"] > 0
    count, valid, _ = reference_ply_roundtrip(r["params"], r["rest"], r["sh"], tmp_path)
    assert count == r["count"] and valid == 1


@needs_shim
@pytest.mark.gpu
def test_pipeline_splat_stage_reports_a_cancellation():
    """The cancel token set during training (Pipeline.cpp:1935-1939, 1993): the
    stage ends cancelled, not failed and not out of time."""
    points, colors, views, images = capture_scene()
    r = run_stage(points, colors, views, images, iterations=200, max_gaussians=4000,
                  cancel_at=25)
    assert not r["success"]
    assert r["cancelled"] and r["message"] == "cancelled"

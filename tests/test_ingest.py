"""Image ingest: downscaleToWidth (ImageIo.cpp:300-337) and the /255 to the
float training image (Pipeline.cpp:1904-1913), run on the device, against the
reference's own function. Integer arithmetic: bit-exact."""
from __future__ import annotations

import ctypes as ct

import numpy as np
import pytest

import oracle_lib as O
import parallax_b200 as px


def reference_downscale(rgb, width, height, target):
    lib = O.ref()
    lib.ref_downscale.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p,
                                  ct.c_void_p, ct.c_void_p]
    w, h = ct.c_int(), ct.c_int()
    lib.ref_downscale(rgb.ctypes.data, width, height, target, None, ct.byref(w), ct.byref(h))
    out = np.zeros(w.value * h.value * 3, np.uint8)
    lib.ref_downscale(rgb.ctypes.data, width, height, target, out.ctypes.data, ct.byref(w),
                      ct.byref(h))
    return out, w.value, h.value


CASES = [(1920, 1080, 640), (1279, 719, 320), (640, 480, 640), (300, 200, 400), (7, 5, 3),
         (4032, 3024, 1280), (1, 1, 1), (513, 1, 100)]


@pytest.mark.gpu
@pytest.mark.parametrize("width,height,target", CASES)
def test_downscale_matches_the_reference(width, height, target):
    rgb = np.random.default_rng(width * 31 + height).integers(0, 256, width * height * 3,
                                                               dtype=np.uint8)
    ref, rw, rh = reference_downscale(rgb, width, height, target)
    out, lin, w, h = px.downscale_to_width(rgb, width, height, target)
    assert (w, h) == (rw, rh)
    assert np.array_equal(out, ref)
    assert np.array_equal(lin, ref.astype(np.float32) / np.float32(255.0))


@pytest.mark.gpu
def test_trainer_ingests_frames_at_its_view_size():
    params, rest = O.random_cloud(71, 500, 0)
    cloud = px.GaussianCloud(params, 0, rest)
    frames = [np.random.default_rng(k).integers(0, 256, 1280 * 720 * 3, dtype=np.uint8)
              for k in range(2)]
    expect = [reference_downscale(f, 1280, 720, 320) for f in frames]
    views = O.orbit_views(2, 320, 180, seed=3)
    t = px.SplatTrainer(cloud, [(v.camera(), np.zeros(320 * 180 * 3, np.float32))
                                for v in views], px.TrainConfig(iterations=2))
    t.ingest_images([0, 1], frames, [(1280, 720)] * 2)
    # the resident images are the floats: render-and-score through them is
    # the same as with the host-converted images
    a = px.SplatTrainer(cloud, [(v.camera(), e[0].astype(np.float32) / np.float32(255.0))
                                for v, e in zip(views, expect)], px.TrainConfig(iterations=2))
    assert t.step_batch(2, [0, 1]) == a.step_batch(2, [0, 1])
    with pytest.raises(px.PxsError):  # a 1280x800 frame at width 320 is 320x200, not 320x180
        t.ingest_images([0], [np.zeros(1280 * 800 * 3, np.uint8)], [(1280, 800)])
    for x in (t, a):
        x.close()


def reference_seed(points, colors, sh_degree, opacity):
    lib = O.ref()
    lib.ref_initialize_from_points.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_int,
                                               ct.c_float, ct.c_void_p]
    n = points.shape[0]
    rest = (min(3, max(0, sh_degree)) + 1) ** 2 - 1
    out = np.zeros(((14 + 3 * rest), n), np.float32)
    got = lib.ref_initialize_from_points(points.ctypes.data,
                                         None if colors is None else colors.ctypes.data, n,
                                         sh_degree, opacity, out.ctypes.data)
    assert got == n
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("n,sh,with_colors", [(3000, 0, True), (700, 3, True), (20000, 1, False),
                                               (2, 2, True), (1, 0, True)])
def test_seed_matches_the_reference(n, sh, with_colors):
    """initializeFromPointCloud (GaussianCloud.cpp:199-257): the spacing search
    on the device, bit-exact."""
    rs = np.random.default_rng(n + sh)
    points = np.ascontiguousarray(rs.normal(0, 1, (n, 3)).astype(np.float32))
    colors = np.ascontiguousarray(rs.integers(0, 256, (n, 3), dtype=np.uint8)) \
        if with_colors else None
    ours = px.initialize_from_points(points, colors, sh, 0.1)
    ref = reference_seed(points, colors, sh, 0.1)
    assert ours.params.shape == ref.shape
    assert np.array_equal(ours.params.view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("fw,fh", [(640, 480), (160, 120)])
def test_staged_frames_train_like_ingested_frames(fw, fh):
    """pxs_trainer_stage_images, pipelined the way a feeding loop uses it (the
    next step's frames staged before the current step runs), takes the same
    steps as ingesting each step's frames synchronously: same losses and the
    same cloud up to the order of the adjoint's atomic sums. Frames four times
    the view's width are downscaled one by one; frames at the view's size are
    converted together, one launch per staged set."""
    params, rest = O.random_cloud(72, 3000, 1)
    cloud = px.GaussianCloud(params, 1, rest)
    views = O.orbit_views(6, 160, 120, seed=4)
    blank = np.zeros(160 * 120 * 3, np.float32)
    rs = np.random.default_rng(9)
    frames = [rs.integers(0, 256, fw * fh * 3, dtype=np.uint8) for _ in range(6)]
    schedule = [[0, 1], [2, 3], [4, 5], [1, 4], [3, 0]]
    cfg = px.TrainConfig(iterations=50, sh_degree=1, sh_increase_interval=0)
    sync = px.SplatTrainer(cloud, [(v.camera(), blank) for v in views], cfg)
    staged = px.SplatTrainer(cloud, [(v.camera(), blank) for v in views], cfg)
    losses_sync, losses_staged = [], []
    for ids in schedule:
        sync.ingest_images(ids, [frames[i] for i in ids], [(fw, fh)] * len(ids))
        losses_sync.append(sync.step_batch(len(ids), ids))
    staged.stage_images(schedule[0], [frames[i] for i in schedule[0]], [(fw, fh)] * 2)
    for s, ids in enumerate(schedule):
        if s + 1 < len(schedule):
            nxt = schedule[s + 1]
            staged.stage_images(nxt, [frames[i] for i in nxt], [(fw, fh)] * len(nxt))
        losses_staged.append(staged.step_batch(len(ids), ids))
    assert np.allclose(losses_sync, losses_staged, rtol=1e-6, atol=0)
    # the adjoint sums with atomics in no fixed order: clouds agree to rounding
    a, b = sync.cloud_params(), staged.cloud_params()
    assert np.abs(a - b).max() <= 1e-5 * max(1.0, np.abs(a).max())
    with pytest.raises(px.PxsError):  # the wrong frame size is refused before any copy
        staged.stage_images([0], [np.zeros(640 * 400 * 3, np.uint8)], [(640, 400)])
    for t in (sync, staged):
        t.close()


@pytest.mark.gpu
@pytest.mark.parametrize("width,height", [(320, 240), (161, 97)])
def test_frames_at_the_view_size_convert_like_the_host(width, height):
    """Frames already at the view's size (downscaleToWidth returns them as
    they are): the device's byte-to-float pass (16 bytes per thread where the
    sizes allow, one otherwise) gives the host's frame / 255 exactly."""
    params, rest = O.random_cloud(73, 800, 0)
    cloud = px.GaussianCloud(params, 0, rest)
    views = O.orbit_views(2, width, height, seed=6)
    rs = np.random.default_rng(width)
    frames = [rs.integers(0, 256, width * height * 3, dtype=np.uint8) for _ in range(2)]
    t = px.SplatTrainer(cloud, [(v.camera(), np.zeros(width * height * 3, np.float32))
                                for v in views], px.TrainConfig(iterations=2))
    t.ingest_images([0, 1], frames, [(width, height)] * 2)
    a = px.SplatTrainer(cloud, [(v.camera(), f.astype(np.float32) / np.float32(255.0))
                                for v, f in zip(views, frames)], px.TrainConfig(iterations=2))
    assert t.step_batch(2, [0, 1]) == a.step_batch(2, [0, 1])
    for x in (t, a):
        x.close()

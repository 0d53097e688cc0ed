"""Parity of the sm_100a kernels (through the C ABI) with the CPU oracle and
the reference.

Tolerances, stated per quantity:
  * projection: the visible set, its order, depth, mean and clamp flags
    bit-exact; every other field bit-exact for gaussians whose exp() inputs
    glibc's expf rounds correctly (the device computes a correctly rounded
    exp; glibc differs in the last bit for ~0.06% of inputs), and within 1e-5
    relative (to the matrix scale for cov2d/conic) for the rest;
  * per-tile key lists: identical to the oracle's (equal depths ordered by
    gaussian index); against the reference's own lists, identical except that
    each run of equal depths holds the same set in ascending index, where the
    reference's std::sort leaves an unspecified order;
  * rendered images: within 1e-5 relative (floor 1e-3), except values that
    the oracle's decision margins (oracle/pxo.c pxo_pixel_decisions_f32)
    explain: a pixel with a decision (power sign, alpha floor, 0.99 cap,
    transmittance cutoff) within 2e-5 of its threshold may flip and move by at
    most 2e-2; against the reference's own order, a pixel where two entries of
    one depth both contribute follows the reference's unspecified tie order;
  * loss: 1e-5 relative; dL/drgb: 1e-5 of its largest magnitude;
  * gradients: 1e-4 relative, normwise per parameter group (the device sums in
    a different order, with atomics);
  * Adam: bit-exact; densify: counts, sources, the RNG state and all
    non-position values exact, split-child positions within 1e-6 (glibc's
    logf/cosf in the normal draw are not always correctly rounded).
"""
from __future__ import annotations

import ctypes as ct
import math
import os

import numpy as np
import pytest

import oracle_lib as O
import parallax_b200 as px
from parallax_b200._abi import PROJECTED_DTYPE, RasterOptions, TrainConfig

# Loss drift allowed over the 60-step trainer run (relative, worst step).
LOSS_DRIFT = 2e-5

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def ctx():
    available, name, reason = px.splat_gpu_availability()
    assert available, f"no usable device: {reason}"
    c = px.Context(0)
    yield c
    c.close()


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def golden_case(name):
    d = load(name)
    view = O.View(tuple(d["K"]), int(d["size"][0]), int(d["size"][1]), d["R"], d["t"])
    opt = RasterOptions(background=tuple(d["background"]), sh_degree=int(d["sh_degree"]),
                        min_alpha=float(d["min_alpha"]),
                        transmittance_cutoff=float(d["transmittance_cutoff"]),
                        screen_dilation=float(d["screen_dilation"]))
    cloud = px.GaussianCloud(d["params"], int(d["cloud_sh_degree"]), int(d["rest"]))
    return d, view, opt, cloud


def random_case(seed, count, sh, width, height, log_scale_mean=-3.0):
    params, rest = O.random_cloud(seed, count, sh, log_scale_mean=log_scale_mean)
    view = O.orbit_views(3, width, height, seed=seed)[seed % 3]
    opt = RasterOptions(sh_degree=sh, background=(0.1, 0.2, 0.3))
    return view, opt, px.GaussianCloud(params, sh, rest)


def ulps(a, b):
    a = np.ascontiguousarray(a, dtype=np.float32).view(np.int32).astype(np.int64)
    b = np.ascontiguousarray(b, dtype=np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)


CASES = ["golden:raster_sh0.npz", "golden:raster_sh3.npz", "random:0", "random:1", "random:2",
         "random:3"]


def make_case(case):
    kind, arg = case.split(":")
    if kind == "golden":
        _, view, opt, cloud = golden_case(arg)
        return view, opt, cloud
    sh = int(arg)
    return random_case(40 + sh, 3000, sh, 200 + 8 * sh, 150 - 5 * sh)


glibc_exp_is_correctly_rounded = O.glibc_exp_is_correctly_rounded


@pytest.mark.parametrize("case", CASES)
def test_projection_matches_oracle(ctx, case):
    view, opt, cloud = make_case(case)
    cam = view.camera()
    gpu = px.project_splats(cloud, cam, opt, ctx)
    ora = O.oracle_project(cloud.params, cloud.rest_per_channel, cloud.sh_degree, cam, opt)
    assert len(gpu) == len(ora)
    # both order near to far with equal depths by index: same sequence
    assert np.array_equal(gpu["index"], ora["index"])
    assert np.array_equal(gpu["depth"].view(np.uint32), ora["depth"].view(np.uint32))
    assert np.array_equal(gpu["mean"].view(np.uint32), ora["mean"].view(np.uint32))
    assert np.array_equal(gpu["clamped"], ora["clamped"])
    # Every field is bit-exact for gaussians whose four exp() inputs (three
    # log-scales, the opacity logit) glibc rounds correctly; the others differ
    # only through that last-bit difference in a scale or the opacity.
    p = cloud.params[:, gpu["index"]]
    exact = glibc_exp_is_correctly_rounded(np.stack([p[3], p[4], p[5], -p[10]])).all(axis=0)
    assert exact.mean() > 0.99
    for name in ["cov2d", "conic", "radius", "opacity", "color"]:
        a, b = gpu[name][exact], ora[name][exact]
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), name
    for name in ["cov2d", "conic"]:
        a, b = gpu[name][~exact], ora[name][~exact]
        if len(a):
            scale = np.abs(b).max(axis=1, keepdims=True)
            assert (np.abs(a - b) <= 1e-5 * scale).all(), name
    for name in ["radius", "opacity", "color"]:
        a, b = gpu[name][~exact], ora[name][~exact]
        if len(a):
            assert (np.abs(a - b) <= 1e-5 * np.maximum(np.abs(b), 1e-3)).all(), name


@pytest.mark.parametrize("case", CASES)
def test_tile_lists_match_oracle(ctx, case):
    view, opt, cloud = make_case(case)
    cam = view.camera()
    offsets, entries = px.tile_lists(cloud, cam, opt, ctx)
    ora = O.oracle_project(cloud.params, cloud.rest_per_channel, cloud.sh_degree, cam, opt)
    o_off, o_ent = O.oracle_tiles(ora, view.width, view.height)
    assert np.array_equal(offsets, o_off)
    assert np.array_equal(entries, ora["index"][o_ent])


def test_tile_lists_match_golden_reference_lists(ctx):
    for name in ["raster_sh0.npz", "raster_sh3.npz"]:
        d, view, opt, cloud = golden_case(name)
        offsets, entries = px.tile_lists(cloud, view.camera(), opt, ctx)
        assert np.array_equal(offsets, d["tile_offsets"])
        assert np.array_equal(entries, d["tile_entries"])


# An image value off by more than 1e-5 relative (floor 1e-3) must be explained:
# a branch flip (a decision of its pixel within FLIP_MARGIN of its threshold,
# where last-bit differences of the inputs can take it the other way), which may
# move the value by at most FLIP_BOUND; or, against the reference's own order
# only, a depth tie (two entries of one depth that both contribute there).
RTOL, FLOOR, FLIP_MARGIN, FLIP_BOUND = 1e-5, 1e-3, 2e-5, 2e-2


def check_image(got, want, channels, margin, tie=None, label=""):
    tie = np.zeros(margin.shape, bool) if tie is None else tie
    ex = O.explain_image_differences(got, want, channels, margin, tie, RTOL, FLOOR, FLIP_MARGIN)
    assert ex["unexplained"] == 0, (label, ex)
    diff = np.abs(np.asarray(got, np.float64) - want).reshape(-1, channels).max(axis=1)
    flip_only = (margin < FLIP_MARGIN) & ~tie
    if flip_only.any():
        assert diff[flip_only].max() <= FLIP_BOUND, (label, float(diff[flip_only].max()))
    print(label, ex)
    return ex


@pytest.mark.parametrize("case", CASES)
def test_render_matches_oracle(ctx, case):
    view, opt, cloud = make_case(case)
    cam = view.camera()
    rgb, T = px.render_splats(cloud, cam, opt, ctx)
    ora = O.oracle_project(cloud.params, cloud.rest_per_channel, cloud.sh_degree, cam, opt)
    o_rgb, o_T = O.oracle_rasterize(ora, cam, opt)
    margin, _, _ = O.oracle_pixel_decisions(ora, cam, opt)
    # both order equal depths by gaussian index: only branch flips may differ
    check_image(rgb, o_rgb, 3, margin, label=case)
    check_image(T, o_T, 1, margin, label=case + " T")


def test_render_matches_golden_reference_image(ctx):
    for name in ["raster_sh0.npz", "raster_sh3.npz"]:
        d, view, opt, cloud = golden_case(name)
        cam = view.camera()
        rgb, T = px.render_splats(cloud, cam, opt, ctx)
        proj = O.projected_from_fixture(d)
        margin, tie = O.tie_and_flip_pixels([proj], cam, opt)
        check_image(rgb, d["rgb"], 3, margin, tie, label=name)
        check_image(T, d["transmittance"], 1, margin, tie, label=name + " T")


def tie_fixture(ctx):
    d, view, opt, cloud = golden_case("ties.npz")
    proj = O.projected_from_fixture(d)
    depth_of = np.zeros(cloud.count, dtype=np.float32)
    depth_of[proj["index"]] = proj["depth"]
    return d, view, opt, cloud, proj, depth_of


def test_tile_lists_equal_the_references_own_lists_up_to_tie_order(ctx):
    """tests/golden/ties.npz: 900 gaussians on 30 depth planes; the reference's
    lists in its own (std::sort) order. The device's lists hold the same
    entries in the same order except within runs of equal depth, where they
    are the same set in ascending gaussian index (the specified tie-break)."""
    d, view, opt, cloud, proj, depth_of = tie_fixture(ctx)
    offsets, entries = px.tile_lists(cloud, view.camera(), opt, ctx)
    assert np.array_equal(offsets, d["tile_offsets"])
    ok, runs, reordered = O.lists_equal_up_to_ties(offsets, entries, d["tile_entries"], depth_of)
    assert ok, (runs, reordered)
    assert runs > 100 and reordered > 0, (runs, reordered)
    for tile in range(len(offsets) - 1):
        lo, hi = offsets[tile], offsets[tile + 1]
        for b, e in O.tie_runs(depth_of[entries[lo:hi]].view(np.uint32)):
            assert np.all(np.diff(entries[lo + b:lo + e]) > 0)


def test_render_with_depth_ties_differs_from_the_reference_only_where_ties_decide(ctx):
    d, view, opt, cloud, proj, _ = tie_fixture(ctx)
    cam = view.camera()
    rgb, _ = px.render_splats(cloud, cam, opt, ctx)
    ordered = O.tie_ordered(proj)
    margin, tie = O.tie_and_flip_pixels([proj, ordered], cam, opt)
    ex = check_image(rgb, d["rgb"], 3, margin, tie, label="ties vs reference order")
    assert ex["tie_pixels"] > 0, ex  # the reference's order does change the image there
    # against the reference's arithmetic in the specified order: flips only
    check_image(rgb, d["index_order_rgb"], 3, margin, label="ties vs index order")


def test_gradients_with_depth_ties_match_the_reference_in_index_order(ctx):
    d, view, opt, cloud, _, _ = tie_fixture(ctx)
    grads = px.SplatGradients.zeros(cloud)
    loss = px.render_and_accumulate(cloud, view.camera(), opt, d["target"], 0.2, grads, ctx)
    want = float(d["index_order_loss"])
    assert abs(loss - want) <= 1e-5 * abs(want)
    assert np.array_equal(grads.visible_count, d["index_order_visible_count"])
    errs = grad_errors(grads.params, d["index_order_grads"])
    assert max(errs.values()) <= 1e-4, errs


@pytest.mark.parametrize("size", [(16, 12), (37, 23), (64, 48), (128, 96)])
def test_loss_and_ssim_match_oracle(ctx, size):
    w, h = size
    rs = np.random.default_rng(w * h)
    rendered = rs.uniform(0, 1, w * h * 3).astype(np.float32)
    target = rs.uniform(0, 1, w * h * 3).astype(np.float32)
    for weight in [0.0, 0.2, 1.0]:
        loss, grad = px.photometric_loss(rendered, target, w, h, weight, ctx=ctx)
        o_loss, o_grad = O.oracle_loss(rendered, target, w, h, weight)
        assert abs(loss - o_loss) <= 1e-5 * abs(o_loss)
        assert np.abs(grad - o_grad).max() <= 1e-5 * np.abs(o_grad).max()
    s, g = px.mean_ssim(rendered, target, w, h, ctx=ctx)
    o_s, o_g = O.oracle_ssim(rendered, target, w, h)
    assert abs(s - o_s) <= 1e-5 * abs(o_s)
    assert np.abs(g - o_g).max() <= 1e-5 * np.abs(o_g).max()


def test_loss_matches_golden_reference(ctx):
    for name in ["raster_sh0.npz", "raster_sh3.npz"]:
        d, view, _, _ = golden_case(name)
        loss, grad = px.photometric_loss(d["rgb"], d["target"], view.width, view.height, 0.2,
                                         ctx=ctx)
        assert abs(loss - float(d["loss"])) <= 1e-5 * abs(float(d["loss"]))
        assert np.abs(grad - d["dL_drgb"]).max() <= 1e-5 * np.abs(d["dL_drgb"]).max()


GROUPS = {"position": slice(0, 3), "log_scale": slice(3, 6), "rotation": slice(6, 10),
          "opacity": slice(10, 11), "dc": slice(11, 14), "sh_rest": slice(14, None)}


def grad_errors(gpu, ref):
    out = {}
    for name, sl in GROUPS.items():
        a, b = gpu[sl], ref[sl]
        if b.size == 0:
            continue
        out[name] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))
    return out


@pytest.mark.parametrize("case", CASES)
def test_backward_matches_oracle(ctx, case):
    view, opt, cloud = make_case(case)
    cam = view.camera()
    ora = O.oracle_project(cloud.params, cloud.rest_per_channel, cloud.sh_degree, cam, opt)
    rgb, _ = O.oracle_rasterize(ora, cam, opt)
    target = np.random.default_rng(7).uniform(0, 1, rgb.shape).astype(np.float32)
    _, dL = O.oracle_loss(rgb, target, view.width, view.height, 0.2)
    grads = px.SplatGradients.zeros(cloud)
    px.rasterize_splats_backward(cloud, cam, opt, dL, grads, ctx)
    o_g, o_s, o_v = O.oracle_backward(cloud.params, cloud.rest_per_channel, cloud.sh_degree, cam,
                                      opt, ora, dL)
    assert np.array_equal(grads.visible_count, o_v)
    errs = grad_errors(grads.params, o_g)
    assert max(errs.values()) <= 1e-4, errs
    assert np.linalg.norm(grads.screen_gradient - o_s) <= 1e-4 * np.linalg.norm(o_s)


def test_backward_accumulates_rather_than_overwriting(ctx):
    view, opt, cloud = make_case("random:2")
    cam = view.camera()
    dL = np.random.default_rng(3).normal(0, 1e-5, view.width * view.height * 3).astype(np.float32)
    once = px.SplatGradients.zeros(cloud)
    px.rasterize_splats_backward(cloud, cam, opt, dL, once, ctx)
    twice = px.SplatGradients(once.params.copy(), once.screen_gradient.copy(),
                              once.visible_count.copy())
    px.rasterize_splats_backward(cloud, cam, opt, dL, twice, ctx)
    assert np.array_equal(twice.visible_count, 2 * once.visible_count)
    # the device sums with atomics in no fixed order: compare normwise per group
    errs = grad_errors(twice.params, 2 * once.params)
    assert max(errs.values()) <= 1e-5, errs


@pytest.mark.parametrize("fwd_px,bwd_px", [(1, 1), (2, 2), (4, 4), (1, 4), (4, 1)])
def test_pixels_per_thread_variants_agree(ctx, fwd_px, bwd_px):
    """The compositing kernels at 1, 2 and 4 pixels per thread: the same
    entries taken (transmittance bit-identical), colours within 1e-6 (the
    two-pixel form sums colour with fused multiply-adds), the gradients within
    1e-4 normwise of the reference (the adjoint sums in another order)."""
    lib = px.lib()
    old_f, old_b = ct.c_int32(), ct.c_int32()
    lib.pxs_get_raster_config(ct.byref(old_f), ct.byref(old_b))
    d, view, opt, cloud = golden_case("raster_sh3.npz")
    try:
        assert lib.pxs_set_raster_config(fwd_px, bwd_px) == 0
        rgb, T = px.render_splats(cloud, view.camera(), opt, ctx)
        grads = px.SplatGradients.zeros(cloud)
        loss = px.render_and_accumulate(cloud, view.camera(), opt, d["target"], 0.2, grads, ctx)
        assert lib.pxs_set_raster_config(1, 1) == 0
        rgb1, T1 = px.render_splats(cloud, view.camera(), opt, ctx)
        grads1 = px.SplatGradients.zeros(cloud)
        loss1 = px.render_and_accumulate(cloud, view.camera(), opt, d["target"], 0.2, grads1,
                                         ctx)
    finally:
        lib.pxs_set_raster_config(old_f.value, old_b.value)
    assert np.array_equal(T, T1)
    assert np.abs(rgb - rgb1).max() <= 1e-6 * max(1.0, np.abs(rgb1).max())
    assert abs(loss - loss1) <= 1e-5 * abs(loss1)
    assert np.array_equal(grads.visible_count, d["visible_count"])
    errs = grad_errors(grads.params, d["grads"])
    assert max(errs.values()) <= 1e-4, errs
    assert lib.pxs_set_raster_config(3, 0) == px._abi.PXS_ERR_INVALID


@pytest.mark.parametrize("seed,count,sh,size", [(5, 20000, 3, (640, 480)),
                                                (6, 60000, 3, (333, 251)),
                                                (7, 20000, 0, (480, 360))])
def test_two_pixel_compositing_takes_the_one_pixel_kernels_entries(ctx, seed, count, sh, size):
    """The two- and four-pixel compositing kernels round power, alpha and
    transmittance as the one-pixel kernel's scalar operations (the two-pixel
    form runs them as paired f32x2 instructions): on random clouds, dense
    enough that most pixels saturate, transmittance is bit-identical and
    colours agree to the paired colour FMA's rounding."""
    lib = px.lib()
    old_f, old_b = ct.c_int32(), ct.c_int32()
    lib.pxs_get_raster_config(ct.byref(old_f), ct.byref(old_b))
    view, opt, cloud = random_case(seed, count, sh, *size, log_scale_mean=-2.5)
    out = {}
    try:
        for f in (1, 2, 4):
            assert lib.pxs_set_raster_config(f, 2) == 0
            out[f] = px.render_splats(cloud, view.camera(), opt, ctx)
    finally:
        lib.pxs_set_raster_config(old_f.value, old_b.value)
    rgb1, T1 = out[1]
    assert (T1 < 0.5).mean() > 0.2  # the lists are long enough to matter
    for f in (2, 4):
        rgb, T = out[f]
        assert np.array_equal(T, T1), (f, int((T != T1).sum()))
        assert np.abs(rgb - rgb1).max() <= 1e-5 * max(1.0, np.abs(rgb1).max())


@pytest.mark.parametrize("shape", [(64, 256, 1, 1), (256, 64, 2, 2), (128, 128, 2, 1),
                                   (128, 256, 0, 2)])
def test_batch_and_tile_schedule_leave_results_unchanged(ctx, shape):
    """The per-block entry batch (64 / 128 / 256) and the tile schedule (tile
    order, heaviest first, persistent) of the two-pixel kernels change how the
    work is cut, not what is computed: transmittance and colours identical to
    the default launch shape, gradients within the adjoint's summation-order
    tolerance, visible counts identical."""
    lib = px.lib()
    fb, bb, fs, bs = shape
    old = [ct.c_int32() for _ in range(4)]
    lib.pxs_get_raster_schedule(*[ct.byref(x) for x in old])
    view, opt, cloud = make_case("random:3")
    target = np.random.default_rng(11).uniform(0, 1, view.width * view.height * 3).astype(
        np.float32)
    try:
        assert lib.pxs_set_raster_config(2, 2) == 0
        assert lib.pxs_set_raster_schedule(128, 256, 0, 0) == 0
        rgb0, T0 = px.render_splats(cloud, view.camera(), opt, ctx)
        g0 = px.SplatGradients.zeros(cloud)
        loss0 = px.render_and_accumulate(cloud, view.camera(), opt, target, 0.2, g0, ctx)
        assert lib.pxs_set_raster_schedule(fb, bb, fs, bs) == 0
        rgb1, T1 = px.render_splats(cloud, view.camera(), opt, ctx)
        g1 = px.SplatGradients.zeros(cloud)
        loss1 = px.render_and_accumulate(cloud, view.camera(), opt, target, 0.2, g1, ctx)
    finally:
        lib.pxs_set_raster_schedule(*[x.value for x in old])
    assert np.array_equal(T0, T1)
    assert np.array_equal(rgb0, rgb1)
    assert abs(loss0 - loss1) <= 1e-6 * abs(loss0)
    assert np.array_equal(g0.visible_count, g1.visible_count)
    errs = grad_errors(g1.params, g0.params)
    assert max(errs.values()) <= 1e-5, errs
    assert lib.pxs_set_raster_schedule(100, 0, -1, -1) == px._abi.PXS_ERR_INVALID
    assert lib.pxs_set_raster_schedule(0, 0, 3, -1) == px._abi.PXS_ERR_INVALID


@pytest.mark.parametrize("name", ["raster_sh0.npz", "raster_sh3.npz"])
def test_render_and_accumulate_matches_golden_reference(ctx, name):
    d, view, opt, cloud = golden_case(name)
    grads = px.SplatGradients.zeros(cloud)
    loss = px.render_and_accumulate(cloud, view.camera(), opt, d["target"], 0.2, grads, ctx)
    assert abs(loss - float(d["loss"])) <= 1e-5 * abs(float(d["loss"]))
    assert np.array_equal(grads.visible_count, d["visible_count"])
    errs = grad_errors(grads.params, d["grads"])
    assert max(errs.values()) <= 1e-4, errs


def test_gradients_match_fp64_finite_differences(ctx):
    """The reference's gradient check (SplatRasterTest.cpp:341-415): a 16x16
    tile, SH degree 2, min_alpha = cutoff = 0, a linear functional of the
    pixels. The device's FP32 gradient against double-precision central
    differences (step 1e-6) of the oracle's double instantiation."""
    params, rest = O.make_overlapping_cloud(2)
    view = O.make_view(16, 16)
    cam = view.camera()
    opt = RasterOptions(sh_degree=2, background=(0.2, 0.3, 0.4), min_alpha=0.0,
                        transmittance_cutoff=0.0)
    weights = O.make_target(16 * 16 * 3, 41) - np.float32(0.5)
    cloud = px.GaussianCloud(params, 2, rest)
    grads = px.SplatGradients.zeros(cloud)
    px.rasterize_splats_backward(cloud, cam, opt, weights, grads, ctx)
    p64 = params.astype(np.float64)
    w64 = weights.astype(np.float64)
    worst = {}
    for c in range(p64.shape[0]):
        for g in range(p64.shape[1]):
            h = 1e-6
            q = p64.copy()
            q[c, g] += h
            plus = O.oracle_objective_f64(q, rest, 2, cam, opt, w64, -1.0)
            q[c, g] -= 2 * h
            minus = O.oracle_objective_f64(q, rest, 2, cam, opt, w64, -1.0)
            numeric = (plus - minus) / (2 * h)
            err = abs(grads.params[c, g] - numeric) / max(abs(numeric), abs(grads.params[c, g]),
                                                          1e-3)
            group = next(n for n, sl in GROUPS.items()
                         if (sl.start or 0) <= c < (sl.stop if sl.stop is not None else 10 ** 9))
            worst[group] = max(worst.get(group, 0.0), err)
    assert max(worst.values()) <= 1e-4, worst


def device_buffers(arrays):
    torch = pytest.importorskip("torch")
    return [torch.from_numpy(a).cuda() for a in arrays]


@pytest.mark.parametrize("n,rest", [(4099, 15), (4096, 15), (1024, 3), (6, 0)])
def test_adam_is_bit_exact(ctx, n, rest):
    """Both forms of the Adam kernel: one gaussian per thread (any count) and
    four per thread with 16-byte accesses (counts that are multiples of 4)."""
    torch = pytest.importorskip("torch")
    rs = np.random.default_rng(5 + n)
    P = px.param_count(rest)
    params = rs.normal(0, 1, (P, n)).astype(np.float32)
    grads = rs.normal(0, 1e-3, (P, n)).astype(np.float32)
    m = rs.normal(0, 1e-4, (P, n)).astype(np.float32)
    v = np.abs(rs.normal(0, 1e-6, (P, n))).astype(np.float32)
    lr = np.array([1.6e-4 * 3.3, 5e-3, 1e-3, 0.05, 2.5e-3, 2.5e-3 / 20], dtype=np.float32)
    c1, c2 = np.float32(1) - np.float32(0.9) ** 3, np.float32(1) - np.float32(0.999) ** 3
    d = device_buffers([params, grads, m, v])
    status = px.lib().pxs_adam_device(ctx.handle, d[0].data_ptr(), d[1].data_ptr(),
                                      d[2].data_ptr(), d[3].data_ptr(), n, rest,
                                      lr.ctypes.data, 0.9, 0.999, 1e-15, float(c1), float(c2), 1)
    ctx.check(status)
    torch.cuda.synchronize()
    p_ref, m_ref, v_ref = params.copy(), m.copy(), v.copy()
    O.pxo().pxo_adam_f32(O.as_ptr(p_ref), O.as_ptr(grads), O.as_ptr(m_ref), O.as_ptr(v_ref), n,
                         rest, O.as_ptr(lr), ct.c_float(0.9), ct.c_float(0.999),
                         ct.c_float(1e-15), ct.c_float(c1), ct.c_float(c2))
    assert np.array_equal(d[0].cpu().numpy().view(np.uint32), p_ref.view(np.uint32))
    assert np.array_equal(d[2].cpu().numpy().view(np.uint32), m_ref.view(np.uint32))
    assert np.array_equal(d[3].cpu().numpy().view(np.uint32), v_ref.view(np.uint32))
    assert not d[1].any().item()  # gradients cleared


def densify_compare(gpu, ora):
    """Counts, sources, the RNG state and every non-position value are exact.
    Split children's positions add a normal sample drawn with logf/cosf, which
    glibc does not always round correctly (the device's are correctly rounded):
    those may differ by the last bit of the sample, far below 1e-6."""
    g_cloud, g_src, g_state, g_counts = gpu
    o_params, o_src, o_state, o_counts = ora
    assert tuple(g_counts) == tuple(o_counts)
    assert g_state == o_state
    assert np.array_equal(g_src, o_src)
    assert g_cloud.params.shape == o_params.shape
    assert np.array_equal(g_cloud.params[3:].view(np.uint32), o_params[3:].view(np.uint32))
    pos_a, pos_b = g_cloud.params[:3], o_params[:3]
    assert np.abs(pos_a - pos_b).max(initial=0.0) <= 1e-6
    kept = g_src >= 0
    assert np.array_equal(pos_a[:, kept].view(np.uint32), pos_b[:, kept].view(np.uint32))


def test_densify_matches_golden_reference(ctx):
    d = load("densify.npz")
    cloud = px.GaussianCloud(d["params"], 1, int(d["rest"]))
    for tag in ["a", "b", "c"]:
        cfg = TrainConfig(max_gaussians=int(d[f"{tag}_max"]))
        gpu = px.densify_and_prune(cloud, d["screen_gradient"], d["visible_count"], cfg,
                                   float(d["extent"]), int(d[f"{tag}_iteration"]), int(d["rng"]),
                                   ctx)
        densify_compare(gpu, (d[f"{tag}_params"], d[f"{tag}_source"], int(d[f"{tag}_rng"]),
                              tuple(d[f"{tag}_counts"])))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_densify_matches_oracle(ctx, seed):
    params, rest = O.random_cloud(seed, 5000, 3, log_scale_mean=-3.5)
    rs = np.random.default_rng(seed)
    screen = rs.uniform(0, 1e-3, 5000).astype(np.float32)
    visible = rs.integers(0, 4, 5000).astype(np.int32)
    cloud = px.GaussianCloud(params, 3, rest)
    for iteration, cap in [(700, 600000), (3500, 600000), (700, 6000), (700, 5000)]:
        cfg = TrainConfig(max_gaussians=cap)
        gpu = px.densify_and_prune(cloud, screen, visible, cfg, 2.7, iteration, 99 + seed, ctx)
        ora = O.oracle_densify(params, rest, screen, visible, cfg, 2.7, iteration, 99 + seed)
        densify_compare(gpu, ora)


def blob_scene(n_views=4, size=24):
    truth, _ = O.truth_cloud()
    views = O.ring_of_views(n_views, 1.6, size, size)
    images = [O.oracle_rasterize(O.oracle_project(truth, 0, 0, v.camera(), RasterOptions()),
                                 v.camera(), RasterOptions())[0] for v in views]
    return views, images


def test_trainer_follows_the_reference_schedule():
    """The golden trainer run (SplatTrainerTest.cpp blob scene, 60 iterations,
    densify every 20): same view order, same counts after each densify, losses
    within LOSS_DRIFT relative (the first step within 1e-5), same finished count."""
    d = load("trainer_blobs.npz")
    n_views = int(d["n_views"])
    views = []
    for i in range(n_views):
        view = O.View(tuple(d[f"view{i}_K"]), int(d[f"view{i}_size"][0]),
                      int(d[f"view{i}_size"][1]), d[f"view{i}_R"], d[f"view{i}_t"])
        views.append((view.camera(), d[f"image{i}"]))
    cfg = TrainConfig(**{name: d[f"cfg_{name}"].item() for name, _ in TrainConfig._fields_})
    trainer = px.SplatTrainer(px.GaussianCloud(d["start"], 0, 0), views, cfg)
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
    assert abs(trainer.state()["extent"] - float(d["extent"])) <= 1e-6
    finished = trainer.finish()
    assert finished.params.shape == d["finished"].shape
    logits = finished.params[10]
    assert (np.diff(logits) <= 0).all()


def test_trainer_drives_the_loss_down_and_cancels():
    views, images = blob_scene(6, 32)
    start, _ = O.rough_start()
    cfg = TrainConfig(iterations=400, sh_degree=0, sh_increase_interval=0,
                      densify_from_iteration=401, densify_until_iteration=401,
                      opacity_reset_interval=0)
    trainer = px.SplatTrainer(px.GaussianCloud(start, 0, 0),
                              [(v.camera(), im) for v, im in zip(views, images)], cfg)
    assert trainer.step()
    first = trainer.last_loss()
    assert trainer.train()
    assert trainer.smoothed_loss() < 0.5 * first
    # cancel at iteration 25 (SplatTrainerTest.cpp:195-209)
    cfg2 = TrainConfig(iterations=500, sh_degree=0, sh_increase_interval=0,
                       densify_from_iteration=501, densify_until_iteration=501,
                       opacity_reset_interval=0)
    t2 = px.SplatTrainer(px.GaussianCloud(start[:, :8].copy(), 0, 0),
                         [(v.camera(), im) for v, im in zip(views, images)], cfg2)
    seen = []
    done = t2.train(lambda p: (seen.append(p.iteration), p.iteration < 25)[1])
    assert not done and seen[-1] == 25 and t2.iteration == 25


def test_batched_and_graph_steps_match_the_plain_multi_view_step():
    params, rest = O.random_cloud(11, 20000, 3, log_scale_mean=-4.0)
    truth, _ = O.random_cloud(12, 20000, 3, log_scale_mean=-4.0)
    views = O.orbit_views(8, 160, 120, seed=4)
    images = [px.render_splats(px.GaussianCloud(truth, 3, rest), v.camera(),
                               RasterOptions(sh_degree=3))[0] for v in views]
    cfg = TrainConfig(iterations=100, sh_degree=3, sh_increase_interval=0,
                      densify_from_iteration=1000, densify_until_iteration=1000)
    pairs = [(v.camera(), im) for v, im in zip(views, images)]
    ids = [0, 3, 5, 6]
    results = []
    for mode in ["plain", "batched", "graph"]:
        t = px.SplatTrainer(px.GaussianCloud(params, 3, rest), pairs, cfg)
        losses = []
        for step in range(3):
            sel = [(i + step) % 8 for i in ids]
            if mode == "plain":
                losses.append(t.step_views(4, sel))
            else:
                losses.append(t.step_batch(4, sel, graph=(mode == "graph")))
        results.append((losses, t.cloud_params()))
        t.close()
    (l0, p0), (l1, p1), (l2, p2) = results
    assert np.allclose(l0, l1, rtol=1e-5) and np.allclose(l0, l2, rtol=1e-5)
    # positions move by ~lr (1e-3 here) per step; the three forms differ only in
    # the order the device sums gradients (atomics), far below a step
    assert np.abs(p0 - p1).max() <= 1e-4 and np.abs(p1 - p2).max() <= 1e-4


def test_one_view_steps_over_views_of_different_sizes():
    """pxs_trainer_step runs the batched step over its one view, sized with
    headroom from the first view it meets; with views of two sizes it runs
    without a captured graph, and a large view after small ones overflows
    the learned pair buffers, so that step is redone with larger ones. Step
    by step it matches the plain per-view step (pxs_trainer_step_views over
    the same view), up to the order in which the adjoint's atomics add."""
    params, rest = O.random_cloud(91, 20000, 3, log_scale_mean=-3.0)
    truth, _ = O.random_cloud(92, 20000, 3, log_scale_mean=-3.0)
    small = O.orbit_views(4, 96, 72, seed=10)
    large = O.orbit_views(2, 320, 240, radius=2.2, seed=11)
    views = small + large
    opt = RasterOptions(sh_degree=3)
    images = [px.render_splats(px.GaussianCloud(truth, 3, rest), v.camera(), opt)[0]
              for v in views]
    cfg = TrainConfig(iterations=12, sh_degree=3, sh_increase_interval=0,
                      densify_from_iteration=1000, densify_until_iteration=1000)
    pairs = [(v.camera(), im) for v, im in zip(views, images)]
    one = px.SplatTrainer(px.GaussianCloud(params, 3, rest), pairs, cfg)
    plain = px.SplatTrainer(px.GaussianCloud(params, 3, rest), pairs, cfg)
    lib = px.lib()
    la, lb, step_pairs = [], [], []
    while one.step():
        la.append(one.last_loss())
        lb.append(plain.step_views(1))  # the same shuffled view: the same schedule
        k, launches = ct.c_int64(), ct.c_int64()
        one._check(lib.pxs_trainer_step_info(one.handle, ct.byref(k), ct.byref(launches)))
        step_pairs.append(k.value)
    assert len(la) == 12
    assert one.state()["iteration"] == plain.state()["iteration"] == 12
    assert np.allclose(la, lb, rtol=1e-5)
    assert np.abs(one.cloud_params() - plain.cloud_params()).max() <= 1e-4
    # the large views list several times the small views' pairs
    assert max(step_pairs) > 3 * min(step_pairs)
    one.close()
    plain.close()


def test_a_batch_with_views_that_see_nothing():
    """A view whose camera faces away from the cloud projects no slot, builds
    empty tile lists and renders the background. Mixed into a batch with
    views that see the cloud, the batched and graph steps still match the
    plain per-view step; a batch of such views alone has a zero gradient, so
    Adam leaves every parameter exactly where it was (m = v = 0 give a zero
    update, SplatTrainer.cpp:56-65)."""
    params, rest = O.random_cloud(71, 20000, 3, log_scale_mean=-4.0)
    truth, _ = O.random_cloud(72, 20000, 3, log_scale_mean=-4.0)
    seeing = O.orbit_views(3, 160, 120, seed=8)
    away = []
    for eye in ([0.0, 0.0, -3.0], [3.0, 0.5, 0.0]):
        eye = np.array(eye)
        R = O.look_at(eye, eye * 3.0)  # looking outward: the cloud is behind
        away.append(O.View(seeing[0].K, 96, 64, R, -R @ eye))
    views = seeing + away
    opt = RasterOptions(sh_degree=3)
    images = [px.render_splats(px.GaussianCloud(truth, 3, rest), v.camera(), opt)[0]
              for v in views]
    for v, im in zip(away, images[3:]):
        assert len(px.project_splats(px.GaussianCloud(params, 3, rest), v.camera(), opt)) == 0
        assert np.allclose(im, 0.0)  # the default background is black
    cfg = TrainConfig(iterations=100, sh_degree=3, sh_increase_interval=0,
                      densify_from_iteration=1000, densify_until_iteration=1000)
    pairs = [(v.camera(), im) for v, im in zip(views, images)]
    results = []
    for mode in ("plain", "batched", "graph"):
        t = px.SplatTrainer(px.GaussianCloud(params, 3, rest), pairs, cfg)
        losses = []
        for sel in ([0, 3, 1, 4], [4, 2, 3]):
            if mode == "plain":
                losses.append(t.step_views(len(sel), sel))
            else:
                losses.append(t.step_batch(len(sel), sel, graph=(mode == "graph")))
        results.append((losses, t.cloud_params()))
        t.close()
    (l0, p0), (l1, p1), (l2, p2) = results
    assert np.allclose(l0, l1, rtol=1e-5) and np.allclose(l0, l2, rtol=1e-5)
    assert np.abs(p0 - p1).max() <= 1e-4 and np.abs(p1 - p2).max() <= 1e-4
    # only views that see nothing: black against black (L1 0, SSIM 1) and no
    # parameter moves; the quaternion rows are renormalised by every step
    # (SplatTrainer.cpp:247-248), which may move their last bit
    rot = slice(6, 10)
    for graph in (False, True):
        t = px.SplatTrainer(px.GaussianCloud(params, 3, rest), pairs, cfg)
        before = t.cloud_params()
        loss = t.step_batch(2, [3, 4], graph=graph)
        after = t.cloud_params()
        assert abs(loss) <= 1e-6
        keep = np.ones(after.shape[0], bool)
        keep[rot] = False
        assert np.array_equal(after[keep], before[keep])
        assert np.abs(after[rot] - before[rot]).max() <= 1e-6
        assert t.state()["iteration"] == 1
        t.close()


def test_a_graph_step_whose_tile_lists_overflow_is_redone():
    """The unsynchronised step runs with the pair and record capacities learned
    on its first batch (with headroom). A later batch with many more tile pairs
    -- cameras much closer -- overflows them: the step is discarded, the
    buffers grown and the step redone, matching the host-synchronised plain
    step as closely as the batched and plain forms match each other."""
    params, rest = O.random_cloud(61, 20000, 3, log_scale_mean=-2.5)
    truth, _ = O.random_cloud(62, 20000, 3, log_scale_mean=-2.5)
    far = O.orbit_views(2, 160, 120, radius=9.0, seed=5)
    near = O.orbit_views(2, 160, 120, radius=2.2, seed=6)
    views = far + near
    images = [px.render_splats(px.GaussianCloud(truth, 3, rest), v.camera(),
                               RasterOptions(sh_degree=3))[0] for v in views]
    cfg = TrainConfig(iterations=100, sh_degree=3, sh_increase_interval=0,
                      densify_from_iteration=1000, densify_until_iteration=1000)
    pairs = [(v.camera(), im) for v, im in zip(views, images)]
    lib = px.lib()
    results, step_pairs = [], []
    for mode in ("plain", "graph"):
        t = px.SplatTrainer(px.GaussianCloud(params, 3, rest), pairs, cfg)
        losses = []
        for sel in ([0, 1], [2, 3]):
            if mode == "plain":
                losses.append(t.step_views(2, sel))
            else:
                losses.append(t.step_batch(2, sel, graph=True))
                k, launches = ct.c_int64(), ct.c_int64()
                t._check(lib.pxs_trainer_step_info(t.handle, ct.byref(k), ct.byref(launches)))
                step_pairs.append(k.value)
        results.append((losses, t.cloud_params()))
        t.close()
    k_far, k_near = step_pairs
    print(f"tile pairs: far step {k_far}, near step {k_near}")
    # the capacity learned on the far step is 1.5 K + 65536 pairs
    assert k_near > 1.5 * k_far + 65536, "the near step did not overflow"
    (l0, p0), (l1, p1) = results
    assert np.allclose(l0, l1, rtol=1e-5)
    assert np.abs(p0 - p1).max() <= 1e-4


def test_train_splats_on_gpu_writes_back_a_finished_cloud():
    views, images = blob_scene(4, 16)
    start, _ = O.rough_start(10)
    start[10, 0] = -30.0  # transparent: pruned by finish()
    cfg = TrainConfig(iterations=30, sh_degree=0, sh_increase_interval=0,
                      densify_from_iteration=31, densify_until_iteration=31,
                      opacity_reset_interval=0)
    ok, err, out = px.train_splats_on_gpu(px.GaussianCloud(start, 0, 0),
                                          [(v.camera(), im) for v, im in zip(views, images)],
                                          cfg)
    assert ok, err
    assert out.count == 9
    assert (np.diff(out.params[10]) <= 0).all()
    cancelled_at = []
    ok, err, out2 = px.train_splats_on_gpu(
        px.GaussianCloud(start, 0, 0), [(v.camera(), im) for v, im in zip(views, images)], cfg,
        callback=lambda p: (cancelled_at.append(p.iteration), p.iteration < 5)[1])
    assert ok and cancelled_at[-1] == 5 and out2.count == 9


def test_edge_cases(ctx):
    empty = px.GaussianCloud(np.zeros((14, 0), np.float32), 0, 0)
    view = O.make_view()
    opt = RasterOptions(background=(0.25, 0.5, 0.75))
    rgb, T = px.render_splats(empty, view.camera(), opt, ctx)
    assert np.all(T == 1.0)
    assert np.allclose(rgb.reshape(-1, 3), [0.25, 0.5, 0.75])
    assert len(px.project_splats(empty, view.camera(), opt, ctx)) == 0
    # a single gaussian on the optical axis lands on the principal point
    b = O.CloudBuilder(0)
    b.add([0, 0, 0], [-2, -2, -2], [1, 0, 0, 0], 2.0, [0, 0, 0])
    one = px.GaussianCloud(b.params(), 0, 0)
    proj = px.project_splats(one, view.camera(), RasterOptions(), ctx)
    assert len(proj) == 1 and abs(proj["mean"][0][0] - view.K[2]) < 1e-4
    # behind the camera is dropped
    b.add([0, 0, -10], [-2, -2, -2], [1, 0, 0, 0], 3.0, [0, 0, 0])
    two = px.GaussianCloud(b.params(), 0, 0)
    assert len(px.project_splats(two, view.camera(), RasterOptions(), ctx)) == 1
    # zero-sized image and a loss over nothing
    loss, _ = px.photometric_loss(np.zeros(0, np.float32), np.zeros(0, np.float32), 0, 0, 0.2,
                                  ctx=ctx)
    assert loss == 0.0
    # odd image sizes still match the oracle
    view2, opt2, cloud2 = random_case(77, 2000, 1, 53, 29)
    rgb2, _ = px.render_splats(cloud2, view2.camera(), opt2, ctx)
    ora = O.oracle_project(cloud2.params, cloud2.rest_per_channel, 1, view2.camera(), opt2)
    o_rgb2, _ = O.oracle_rasterize(ora, view2.camera(), opt2)
    margin2, _, _ = O.oracle_pixel_decisions(ora, view2.camera(), opt2)
    check_image(rgb2, o_rgb2, 3, margin2, label="53x29")
    # a too-small key-list buffer is reported, not overrun
    c = cloud2.c_struct()
    cam = view2.camera()
    offsets = np.zeros(((53 + 15) // 16) * ((29 + 15) // 16) + 1, np.int32)
    entries = np.zeros(4, np.int32)
    total = ct.c_int64()
    status = px.lib().pxs_tile_lists(ctx.handle, ct.byref(c), ct.byref(cam), ct.byref(opt2),
                                     offsets.ctypes.data, entries.ctypes.data, 4,
                                     ct.byref(total))
    assert status == px._abi.PXS_ERR_CAPACITY and total.value > 4


def test_multi_scene_batch_matches_per_scene_trainers():
    """Several independent scenes of uneven sizes and resolutions in one
    batched step (one pass of each kernel over all views) against one trainer
    per scene stepping its own views: same losses, same clouds within the
    order in which the device sums gradients."""
    specs = [(2000, 64, 48, 51), (5000, 96, 72, 52), (800, 128, 96, 53)]
    opt = RasterOptions(sh_degree=3)
    clouds, scene_views = [], []
    for count, w, h, seed in specs:
        params, rest = O.random_cloud(seed, count, 3, log_scale_mean=-3.5)
        truth, _ = O.random_cloud(seed + 100, count, 3, log_scale_mean=-3.5)
        views = O.orbit_views(3, w, h, seed=seed)
        images = [px.render_splats(px.GaussianCloud(truth, 3, rest), v.camera(), opt)[0]
                  for v in views]
        clouds.append(px.GaussianCloud(params, 3, rest))
        scene_views.append([(v.camera(), im) for v, im in zip(views, images)])
    cfg = TrainConfig(iterations=100, sh_degree=3, sh_increase_interval=0,
                      densify_from_iteration=1000, densify_until_iteration=1000)
    joint = px.SplatTrainer.from_scenes(clouds, scene_views, cfg)
    single = [px.SplatTrainer(c, sv, cfg) for c, sv in zip(clouds, scene_views)]
    for step in range(3):
        ids = [s * 3 + (step + k) % 3 for s in range(3) for k in range(2)]  # 2 views a scene
        loss = joint.step_batch(len(ids), ids)
        losses = [t.step_batch(2, [(step + k) % 3 for k in range(2)]) for t in single]
        assert abs(loss - float(np.mean(losses))) <= 1e-5 * abs(loss)
    joined = joint.cloud_params()
    at = 0
    for c, t in zip(clouds, single):
        mine = joined[:, at:at + c.count]
        at += c.count
        assert np.abs(mine - t.cloud_params()).max() <= 1e-4
    # one scene of the joint trainer trains apart from the others
    with pytest.raises(px.PxsError):
        joint.finish()
    bad = TrainConfig(iterations=100, densify_from_iteration=10, densify_until_iteration=50)
    with pytest.raises(px.PxsError):
        px.SplatTrainer.from_scenes(clouds, scene_views, bad)
    for t in single + [joint]:
        t.close()

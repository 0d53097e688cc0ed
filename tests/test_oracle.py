"""Pins the CPU oracle (oracle/pxo.c) to the reference.

1. Against the committed golden fixtures (tests/golden/*.npz, written by
   tests/golden/make_golden.py from the reference's own functions): bit for bit.
2. Against the reference compiled from its sources (oracle/_ref), on fresh
   random cases, when that build is present: bit for bit.
3. The double-precision instantiation against central finite differences, on
   the reference's own gradient-check setup (SplatRasterTest.cpp:341-415).
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np
import pytest

import oracle_lib as O
from parallax_b200._abi import RasterOptions, TrainConfig, as_ptr

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
needs_ref = pytest.mark.skipif(not O.ref_available("ieee"),
                               reason="reference build oracle/_ref not present")


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def golden_view(d):
    return O.View(tuple(d["K"]), int(d["size"][0]), int(d["size"][1]), d["R"], d["t"])


def golden_options(d):
    return RasterOptions(background=tuple(d["background"]), sh_degree=int(d["sh_degree"]),
                         min_alpha=float(d["min_alpha"]),
                         transmittance_cutoff=float(d["transmittance_cutoff"]),
                         screen_dilation=float(d["screen_dilation"]))


def golden_projected(d):
    from parallax_b200._abi import PROJECTED_DTYPE
    n = len(d["proj_index"])
    p = np.zeros(n, dtype=PROJECTED_DTYPE)
    for name in PROJECTED_DTYPE.names:
        p[name] = d[f"proj_{name}"]
    return p


def assert_projected_equal(a, b):
    a = np.sort(a, order=["depth", "index"])
    b = np.sort(b, order=["depth", "index"])
    assert len(a) == len(b)
    for name in a.dtype.names:
        if a[name].dtype.kind == "f":
            assert np.array_equal(bits(a[name]), bits(b[name])), name
        else:
            assert np.array_equal(a[name], b[name]), name


@pytest.mark.parametrize("name", ["raster_sh0.npz", "raster_sh3.npz"])
def test_oracle_reproduces_golden_raster(name):
    d = load(name)
    view, opt = golden_view(d), golden_options(d)
    cam = view.camera()
    rest, sh = int(d["rest"]), int(d["cloud_sh_degree"])
    proj = O.oracle_project(d["params"], rest, sh, cam, opt)
    assert_projected_equal(proj, golden_projected(d))
    offsets, entries = O.oracle_tiles(proj, view.width, view.height)
    assert np.array_equal(offsets, d["tile_offsets"])
    assert np.array_equal(proj["index"][entries], d["tile_entries"])
    rgb, T = O.oracle_rasterize(proj, cam, opt)
    assert np.array_equal(bits(rgb), bits(d["rgb"]))
    assert np.array_equal(bits(T), bits(d["transmittance"]))
    loss, dL = O.oracle_loss(d["rgb"], d["target"], view.width, view.height,
                             float(d["ssim_weight"]))
    assert np.float32(loss) == d["loss"]
    assert np.array_equal(bits(dL), bits(d["dL_drgb"]))
    ssim, dssim = O.oracle_ssim(d["rgb"], d["target"], view.width, view.height)
    assert np.float32(ssim) == d["ssim"]
    assert np.array_equal(bits(dssim), bits(d["d_ssim"]))
    grads, screen, visible = O.oracle_backward(d["params"], rest, sh, cam, opt, proj,
                                               d["dL_drgb"])
    assert np.array_equal(bits(grads), bits(d["grads"]))
    assert np.array_equal(bits(screen), bits(d["screen_gradient"]))
    assert np.array_equal(visible, d["visible_count"])


def test_oracle_reproduces_golden_densify():
    d = load("densify.npz")
    for tag in ["a", "b", "c"]:
        cfg = TrainConfig(max_gaussians=int(d[f"{tag}_max"]))
        out, source, state, counts = O.oracle_densify(
            d["params"], int(d["rest"]), d["screen_gradient"], d["visible_count"], cfg,
            float(d["extent"]), int(d[f"{tag}_iteration"]), int(d["rng"]))
        assert tuple(counts) == tuple(d[f"{tag}_counts"])
        assert state == int(d[f"{tag}_rng"])
        assert np.array_equal(source, d[f"{tag}_source"])
        assert np.array_equal(bits(out), bits(d[f"{tag}_params"]))


@needs_ref
def test_camera_conversion_matches_reference():
    for view in O.orbit_views(5, 320, 240) + [O.make_view()] + O.ring_of_views(3, 1.6, 24, 20):
        assert bytes(view.camera()) == bytes(O.ref_camera(view))


@needs_ref
@pytest.mark.parametrize("sh", [0, 1, 2, 3])
def test_oracle_matches_reference_bit_for_bit(sh):
    params, rest = O.random_cloud(100 + sh, 1500, sh, log_scale_mean=-3.0)
    for view in O.orbit_views(2, 96, 72, seed=sh):
        cam = view.camera()
        opt = RasterOptions(sh_degree=sh, background=(0.1, 0.2, 0.3))
        a = O.oracle_project(params, rest, sh, cam, opt)
        b = O.ref_project(params, rest, sh, view, opt)
        assert_projected_equal(a, b)
        rgb_a, T_a = O.oracle_rasterize(b, cam, opt)
        rgb_b, T_b = O.ref_rasterize(b, view, opt)
        assert np.array_equal(bits(rgb_a), bits(rgb_b))
        assert np.array_equal(bits(T_a), bits(T_b))
        target = np.random.default_rng(sh).uniform(0, 1, rgb_a.shape).astype(np.float32)
        la, ga = O.oracle_loss(rgb_b, target, view.width, view.height, 0.2)
        lb, gb = O.ref_loss(rgb_b, target, view.width, view.height, 0.2)
        assert la == lb and np.array_equal(bits(ga), bits(gb))
        g1, s1, v1 = O.oracle_backward(params, rest, sh, cam, opt, b, gb)
        g2, s2, v2 = O.ref_backward(params, rest, sh, view, opt, gb)
        assert np.array_equal(bits(g1), bits(g2))
        assert np.array_equal(bits(s1), bits(s2))
        assert np.array_equal(v1, v2)


@needs_ref
def test_oracle_adam_matches_one_reference_trainer_step():
    libm = ct.CDLL("libm.so.6")
    libm.powf.restype = ct.c_float
    libm.powf.argtypes = [ct.c_float, ct.c_float]
    params, rest = O.random_cloud(3, 400, 2, log_scale_mean=-3.0)
    truth, _ = O.random_cloud(4, 400, 2, log_scale_mean=-3.0)
    view = O.orbit_views(1, 64, 48)[0]
    image, _ = O.ref_render(truth, rest, 2, view, RasterOptions(sh_degree=2))
    cfg = TrainConfig(iterations=10, sh_degree=2, sh_increase_interval=0)
    trainer = O.RefTrainer(params, rest, 2, [view], [image], cfg)
    assert trainer.step()
    after = trainer.cloud()
    extent = np.float32(trainer.state()["extent"])
    _, g, _, _ = O.oracle_render_and_accumulate(params, rest, 2, view.camera(),
                                                RasterOptions(sh_degree=2), image, 0.2)
    f = np.float32
    ratio = f(cfg.position_lr_final) / f(cfg.position_lr_initial)
    lr = np.array([f(f(cfg.position_lr_initial) * f(libm.powf(ratio, 0.0))) * extent,
                   cfg.scale_lr, cfg.rotation_lr, cfg.opacity_lr, cfg.dc_lr,
                   f(cfg.dc_lr) / f(cfg.sh_rest_lr_divider)], dtype=np.float32)
    c1 = f(1) - f(libm.powf(cfg.adam_beta1, 1.0))
    c2 = f(1) - f(libm.powf(cfg.adam_beta2, 1.0))
    p, m, v = params.copy(), np.zeros_like(params), np.zeros_like(params)
    O.pxo().pxo_adam_f32(as_ptr(p), as_ptr(g), as_ptr(m), as_ptr(v), p.shape[1], rest,
                         as_ptr(lr), ct.c_float(cfg.adam_beta1), ct.c_float(cfg.adam_beta2),
                         ct.c_float(cfg.adam_epsilon), ct.c_float(c1), ct.c_float(c2))
    assert np.array_equal(bits(p), bits(after))


@needs_ref
def test_oracle_densify_matches_reference_on_fresh_cases():
    params, rest = O.random_cloud(9, 1200, 2, log_scale_mean=-3.0)
    rs = np.random.default_rng(10)
    screen = rs.uniform(0, 1e-3, params.shape[1]).astype(np.float32)
    visible = rs.integers(0, 4, params.shape[1]).astype(np.int32)
    for iteration, cap in [(700, 600000), (3500, 600000), (700, 1500), (700, 1200)]:
        cfg = TrainConfig(max_gaussians=cap)
        a = O.oracle_densify(params, rest, screen, visible, cfg, 2.5, iteration, 12345)
        b = O.ref_densify(params, rest, screen, visible, cfg, 2.5, iteration, 12345)
        assert a[3] == b[3] and a[2] == b[2]
        assert np.array_equal(a[1], b[1])
        assert np.array_equal(bits(a[0]), bits(b[0]))


@needs_ref
def test_fast_math_reference_build_stays_close_to_the_ieee_build():
    """The reference ships with -ffast-math; its results differ from the IEEE
    build only by rounding. Measured here so the parity bar is honest."""
    if not O.ref_available("fast"):
        pytest.skip("fast build missing")
    params, rest = O.random_cloud(5, 2000, 3, log_scale_mean=-3.0)
    view = O.orbit_views(1, 128, 96)[0]
    opt = RasterOptions(sh_degree=3)
    a, _ = O.ref_render(params, rest, 3, view, opt, kind="ieee")
    b, _ = O.ref_render(params, rest, 3, view, opt, kind="fast")
    err = np.abs(a - b) / np.maximum(np.abs(a), 1e-2)
    assert np.mean(err > 1e-5) < 1e-3
    target = np.random.default_rng(0).uniform(0, 1, a.shape).astype(np.float32)
    la, _ = O.ref_loss(a, target, view.width, view.height, 0.2, kind="ieee")
    lb, _ = O.ref_loss(a, target, view.width, view.height, 0.2, kind="fast")
    assert abs(la - lb) <= 1e-5 * abs(la)


def test_f64_oracle_gradient_matches_central_differences():
    """The reference's gradient check (SplatRasterTest.cpp:341-415): one 16x16
    tile, SH degree 2, background (0.2, 0.3, 0.4), min_alpha = cutoff = 0, a
    linear functional of the pixels; here in double precision with step 1e-6."""
    params, rest = O.make_overlapping_cloud(2)
    view = O.make_view(16, 16)
    cam = view.camera()
    opt = RasterOptions(sh_degree=2, background=(0.2, 0.3, 0.4), min_alpha=0.0,
                        transmittance_cutoff=0.0)
    weights = O.make_target(16 * 16 * 3, 41) - np.float32(0.5)
    p64 = params.astype(np.float64)
    w64 = weights.astype(np.float64)
    lib = O.pxo()
    n = p64.shape[1]
    proj = np.zeros(n, dtype=O.PROJECTED_F64_DTYPE)
    opt_ = opt
    count = lib.pxo_project_f64(as_ptr(p64), n, rest, 2, ct.byref(cam), ct.byref(opt_),
                                as_ptr(proj))
    grads = np.zeros_like(p64)
    screen = np.zeros(n)
    visible = np.zeros(n, dtype=np.int32)
    lib.pxo_backward_f64(as_ptr(p64), n, rest, 2, ct.byref(cam), ct.byref(opt_), as_ptr(proj),
                         count, None, as_ptr(w64), as_ptr(grads), as_ptr(screen),
                         as_ptr(visible))
    worst = 0.0
    for c in range(p64.shape[0]):
        for g in range(n):
            h = 1e-6
            q = p64.copy()
            q[c, g] += h
            plus = O.oracle_objective_f64(q, rest, 2, cam, opt, w64, -1.0)
            q[c, g] -= 2 * h
            minus = O.oracle_objective_f64(q, rest, 2, cam, opt, w64, -1.0)
            numeric = (plus - minus) / (2 * h)
            scale = max(abs(numeric), abs(grads[c, g]), 1e-3)
            worst = max(worst, abs(numeric - grads[c, g]) / scale)
    assert worst < 1e-5


def test_tie_fixture_holds_the_references_own_scrambled_order():
    """tests/golden/ties.npz: 900 gaussians on 30 depth planes. The reference's
    std::sort leaves each run of equal depths in an unspecified order; the
    fixture keeps that order as it came out of projectSplats."""
    d = load("ties.npz")
    proj = golden_projected(d)
    runs = [(b, e) for b, e in O.tie_runs(proj["depth"].view(np.uint32)) if e - b > 1]
    assert len(runs) == 30
    assert sum(not np.all(np.diff(proj["index"][b:e]) > 0) for b, e in runs) == 30
    # the oracle sorts equal depths by gaussian index: the same splats, bit for
    # bit, in the specified order
    view, opt = golden_view(d), golden_options(d)
    ora = O.oracle_project(d["params"], int(d["rest"]), int(d["cloud_sh_degree"]),
                           view.camera(), opt)
    ordered = O.tie_ordered(proj)
    for name in ora.dtype.names:
        assert np.array_equal(np.ascontiguousarray(ora[name]).view(np.uint8),
                              np.ascontiguousarray(ordered[name]).view(np.uint8)), name


def test_tie_fixture_lists_and_image_differ_from_the_index_order_only_at_ties():
    d = load("ties.npz")
    view, opt = golden_view(d), golden_options(d)
    cam = view.camera()
    proj = golden_projected(d)
    ordered = O.tie_ordered(proj)
    offsets, entries = O.oracle_tiles(ordered, view.width, view.height)
    assert np.array_equal(offsets, d["tile_offsets"])
    depth_of = np.zeros(d["params"].shape[1], dtype=np.float32)
    depth_of[proj["index"]] = proj["depth"]
    ok, runs, reordered = O.lists_equal_up_to_ties(offsets, ordered["index"][entries],
                                                    d["tile_entries"], depth_of)
    assert ok and runs > 0 and reordered > 0, (runs, reordered)
    # the index-order image (the oracle) against the reference's own image:
    # every value off by more than 1e-5 is at a pixel that a depth tie decides
    rgb, _ = O.oracle_rasterize(ordered, cam, opt)
    assert np.array_equal(bits(rgb), bits(d["index_order_rgb"]))
    margin, tie = O.tie_and_flip_pixels([proj, ordered], cam, opt)
    ex = O.explain_image_differences(rgb, d["rgb"], 3, np.full_like(margin, np.inf), tie)
    assert ex["unexplained"] == 0, ex
    assert ex["tie_pixels"] > 0, ex  # the tie order changes the image
    # the oracle's gradient in the index order is the reference's arithmetic
    loss, g, s, v = O.oracle_render_and_accumulate(
        d["params"], int(d["rest"]), int(d["cloud_sh_degree"]), cam, opt, d["target"], 0.2)
    assert np.float32(loss) == d["index_order_loss"]
    assert np.array_equal(bits(g), bits(d["index_order_grads"]))
    assert np.array_equal(v, d["index_order_visible_count"])

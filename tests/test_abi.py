"""The C ABI without a GPU: the library loads, exports every entry point
include/pxs.h declares, and its host helpers agree with the reference."""
from __future__ import annotations

import ctypes as ct
import os
import re

import numpy as np
import pytest

import oracle_lib as O
import parallax_b200 as px
from parallax_b200._abi import Camera, TrainConfig

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not O.ref_available("ieee"), reason="reference build missing")


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "pxs.h")).read()
    return sorted(set(re.findall(r"\b(pxs_[a-z0-9_]+)\(", text)))


def test_library_exports_every_declared_entry_point():
    lib = px.lib()
    names = declared_symbols()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name


def test_version_string():
    assert b"sm_100a" in px.lib().pxs_version()


def test_availability_reports_a_reason_without_a_device():
    available, name, reason = px.splat_gpu_availability()
    if not available:
        assert reason  # the reference's contract: a reason a person can read


@needs_ref
def test_camera_from_pose_matches_the_reference_conversion():
    for view in O.orbit_views(6, 320, 240, seed=5) + [O.make_view()] + O.ring_of_views(4, 1.6, 24, 20):
        cam = px.SplatView(view.K, view.width, view.height, view.R, view.t).camera()
        assert bytes(cam) == bytes(O.ref_camera(view))


@needs_ref
def test_config_defaults_and_validation_match_the_reference():
    ours = TrainConfig()
    px.lib().pxs_train_config_defaults(ct.byref(ours))
    ref = TrainConfig()
    O.ref().ref_config_defaults(ct.byref(ref))
    assert bytes(ours) == bytes(ref)
    cases = [dict(iterations=0), dict(sh_degree=7), dict(split_scale_divider=0.8),
             dict(ssim_weight=1.5), dict(max_gaussians=0), dict(densify_interval=0), dict()]
    for case in cases:
        cfg = TrainConfig(**case)
        a = ct.create_string_buffer(128)
        b = ct.create_string_buffer(128)
        sa = px.lib().pxs_train_config_validate(ct.byref(cfg), a, 128)
        sb = O.ref().ref_config_validate(ct.byref(cfg), b, 128)
        assert (sa == 0) == (sb == 0), case
        assert a.value == b.value, case


def test_synthetic_generators_are_deterministic():
    a = px.synthetic_cloud(1, 1000, 3)
    b = px.synthetic_cloud(1, 1000, 3)
    c = px.synthetic_cloud(2, 1000, 3)
    assert np.array_equal(a.params, b.params)
    assert not np.array_equal(a.params, c.params)
    q = a.params[6:10]
    assert np.allclose(np.linalg.norm(q, axis=0), 1.0, atol=1e-5)
    assert a.params[0:3].min() >= -1.0 and a.params[0:3].max() <= 1.0
    cams = px.synthetic_cameras(3, 16, 320, 240, layout=0)
    for cam in cams:
        center = np.array(cam.center)
        assert abs(np.linalg.norm(center) - 3.0) < 1e-4
        R = np.array(cam.R).reshape(3, 3)
        # the optical axis points at the origin
        assert np.dot(R[2], -center / np.linalg.norm(center)) > 0.999
    ring = px.synthetic_cameras(3, 64, 1280, 720, layout=1)
    heights = np.array([c.center[1] for c in ring])
    assert (heights[:32] > 0).all() and (np.abs(heights[32:]) <= 0.2 + 1e-6).all()


def test_compute_entry_points_fail_loudly_without_a_device():
    available, _, _ = px.splat_gpu_availability()
    if available:
        pytest.skip("a device is present")
    with pytest.raises(px.PxsError):
        px.Context(0)

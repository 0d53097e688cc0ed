"""ctypes access to the CPU oracle (oracle/libpxo.so) and to the reference's
own splat code compiled from its sources (oracle/_ref/libpxref_*.so).

Test infrastructure only: the product never imports this module.
"""
from __future__ import annotations

import ctypes as ct
import math
import os
import subprocess
from dataclasses import dataclass
from typing import Optional

import numpy as np

from parallax_b200._abi import (
    PROJECTED_DTYPE,
    Camera,
    RasterOptions,
    TrainConfig,
    as_ptr,
    camera_from_pose,
    param_count,
    rest_per_channel,
)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")

_f32p = ct.POINTER(ct.c_float)
_f64p = ct.POINTER(ct.c_double)
_i32p = ct.POINTER(ct.c_int32)
_u32p = ct.POINTER(ct.c_uint32)


def build_oracle() -> None:
    """Builds oracle/libpxo.so (and oracle/_ref when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", ORACLE_DIR, "all"], check=True)


_PXO = None
_REF = {}


def pxo() -> ct.CDLL:
    """The C restatement."""
    global _PXO
    if _PXO is None:
        path = os.path.join(ORACLE_DIR, "libpxo.so")
        if not os.path.exists(path):
            build_oracle()
        _PXO = ct.CDLL(path)
        _PXO.pxo_project_f32.restype = ct.c_int32
        _PXO.pxo_build_tiles_f32.restype = ct.c_int64
        _PXO.pxo_build_tiles_f32.argtypes = [ct.c_void_p, ct.c_int32, ct.c_int32, ct.c_int32,
                                             ct.c_void_p, ct.c_void_p, ct.c_int64]
        _PXO.pxo_mean_ssim_f32.restype = ct.c_float
        _PXO.pxo_photometric_loss_f32.restype = ct.c_float
        _PXO.pxo_render_and_accumulate_f32.restype = ct.c_float
        _PXO.pxo_project_f64.restype = ct.c_int32
        _PXO.pxo_mean_ssim_f64.restype = ct.c_double
        _PXO.pxo_photometric_loss_f64.restype = ct.c_double
        _PXO.pxo_objective_f64.restype = ct.c_double
        _PXO.pxo_densify_and_prune.restype = ct.c_int32
        _PXO.pxo_next_normal.restype = ct.c_float
    return _PXO


def ref_available(kind: str = "ieee") -> bool:
    return os.path.exists(ref_path(kind))


def ref_path(kind: str = "ieee") -> str:
    name = "libpxshim.so" if kind == "shim" else f"libpxref_{kind}.so"
    return os.path.join(ORACLE_DIR, "_ref", name)


def ref(kind: str = "ieee") -> ct.CDLL:
    """The reference's own code: kind 'ieee' (parity), 'fast' (its release
    flags) or 'shim' (the IEEE build with the drop-in shim over libpxs.so)."""
    if kind not in _REF:
        lib = ct.CDLL(ref_path(kind))
        lib.ref_project.restype = ct.c_int
        lib.ref_photometric_loss.restype = ct.c_float
        lib.ref_mean_ssim.restype = ct.c_float
        lib.ref_render_and_accumulate.restype = ct.c_float
        lib.ref_render_and_accumulate_projected.restype = ct.c_float
        lib.ref_densify.restype = ct.c_int
        lib.ref_trainer_create.restype = ct.c_void_p
        lib.ref_trainer_create.argtypes = [
            ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p,
            ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]
        lib.ref_trainer_step.argtypes = [ct.c_void_p]
        lib.ref_trainer_train.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p]
        lib.ref_trainer_state.argtypes = [ct.c_void_p] + [ct.c_void_p] * 6
        lib.ref_trainer_download.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int]
        lib.ref_trainer_finish.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_void_p]
        lib.ref_trainer_destroy.argtypes = [ct.c_void_p]
        if kind == "shim":
            lib.ref_shim_trainer_create.restype = ct.c_void_p
            lib.ref_shim_trainer_create.argtypes = lib.ref_trainer_create.argtypes
            lib.ref_shim_render_and_accumulate.restype = ct.c_float
            lib.ref_shim_availability.argtypes = [ct.c_void_p, ct.c_char_p, ct.c_int,
                                                  ct.c_char_p, ct.c_int]
            lib.ref_shim_train_splats_on_gpu.argtypes = (
                [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_int] + [ct.c_void_p] * 6
                + [ct.c_int] + [ct.c_void_p] * 3 + [ct.c_char_p, ct.c_int])
        _REF[kind] = lib
    return _REF[kind]


_LIBM = ct.CDLL("libm.so.6")
_LIBM.expf.restype = ct.c_float
_LIBM.expf.argtypes = [ct.c_float]


def glibc_exp_is_correctly_rounded(values):
    """Per value: does glibc's expf (the oracle's and the reference's) equal the
    correctly rounded exp the device computes?"""
    flat = np.asarray(values, dtype=np.float32).reshape(-1)
    cr = np.exp(flat.astype(np.float64)).astype(np.float32)
    glibc = np.array([_LIBM.expf(float(x)) for x in flat], dtype=np.float32)
    return (cr.view(np.uint32) == glibc.view(np.uint32)).reshape(np.shape(values))


# ---------------------------------------------------------------- scenes


class Rng:
    """xorshift64 with a Box-Muller normal (testing/SyntheticScene.h:80-107)."""

    MASK = (1 << 64) - 1

    def __init__(self, seed: int = 88172645463325252):
        self.state = seed if seed else 1

    def next(self) -> int:
        s = self.state
        s ^= (s << 13) & self.MASK
        s ^= s >> 7
        s ^= (s << 17) & self.MASK
        self.state = s
        return s

    def uniform(self, lo: float = 0.0, hi: Optional[float] = None) -> float:
        u = (self.next() >> 11) * (1.0 / 9007199254740992.0)
        if hi is None:
            return u
        return lo + (hi - lo) * u

    def normal(self) -> float:
        u1 = max(1e-12, self.uniform())
        u2 = self.uniform()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


@dataclass
class View:
    """A double-precision SplatView: intrinsics (fx, fy, cx, cy), size and a
    camera-from-world pose."""

    K: tuple
    width: int
    height: int
    R: np.ndarray
    t: np.ndarray

    def camera(self) -> Camera:
        return camera_from_pose(self.K, self.width, self.height, self.R, self.t)

    def ref_args(self):
        K = np.ascontiguousarray(np.array(self.K, dtype=np.float64))
        R = np.ascontiguousarray(np.asarray(self.R, dtype=np.float64).reshape(9))
        t = np.ascontiguousarray(np.asarray(self.t, dtype=np.float64).reshape(3))
        self._keep = (K, R, t)
        return as_ptr(K), self.width, self.height, as_ptr(R), as_ptr(t)


def make_view(width: int = 48, height: int = 36, distance: float = 2.0) -> View:
    """makeView (SplatRasterTest.cpp:15-25)."""
    return View((0.9 * width, 0.9 * width, 0.5 * width, 0.5 * height), width, height,
                np.eye(3), np.array([0.0, 0.0, distance]))


def ring_of_views(count: int, radius: float, width: int, height: int):
    """ringOfViews (SplatTrainerTest.cpp:15-38)."""
    views = []
    for i in range(count):
        angle = 2.0 * math.pi * i / count
        eye = np.array([radius * math.sin(angle), 0.0, -radius * math.cos(angle)])
        forward = -eye / np.linalg.norm(eye)
        right = np.cross(np.array([0.0, 1.0, 0.0]), forward)
        right /= np.linalg.norm(right)
        down = np.cross(forward, right)
        R = np.stack([right, down, forward])
        views.append(View((1.1 * width, 1.1 * width, 0.5 * width, 0.5 * height), width, height,
                          R, -R @ eye))
    return views


def look_at(eye, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """Camera-from-world rotation for a camera at `eye` looking at `target`, +X
    right, +Y down, +Z forward (SyntheticScene.cpp:235-256)."""
    eye = np.asarray(eye, dtype=np.float64)
    forward = np.asarray(target, dtype=np.float64) - eye
    if np.linalg.norm(forward) < 1e-9:
        forward = np.array([0.0, 0.0, 1.0])
    forward = forward / np.linalg.norm(forward)
    world_up = np.asarray(up, dtype=np.float64)
    if abs(np.dot(world_up / np.linalg.norm(world_up), forward)) > 0.999:
        world_up = np.array([1.0, 0.0, 0.0]) if abs(forward[0]) < 0.9 else np.array([0.0, 0.0, 1.0])
    right = np.cross(forward, world_up / np.linalg.norm(world_up))
    right /= np.linalg.norm(right)
    down = np.cross(forward, right)
    return np.stack([right, down, forward])


class CloudBuilder:
    """Accumulates gaussians into the component-major float layout."""

    def __init__(self, rest: int):
        self.rest = rest
        self.rows = []

    def add(self, position, log_scale, rotation_wxyz, opacity_logit, dc, sh_rest=None):
        row = np.zeros(param_count(self.rest), dtype=np.float32)
        row[0:3] = position
        row[3:6] = log_scale
        row[6:10] = rotation_wxyz
        row[10] = opacity_logit
        row[11:14] = dc
        if self.rest:
            row[14:] = sh_rest
        self.rows.append(row)

    def params(self) -> np.ndarray:
        if not self.rows:
            return np.zeros((param_count(self.rest), 0), dtype=np.float32)
        return np.ascontiguousarray(np.stack(self.rows, axis=1).astype(np.float32))


def _normalized_quat(q):
    q = np.array(q, dtype=np.float32)
    w, x, y, z = q
    sq = np.float32(x * x + z * z) + np.float32(y * y + w * w)
    n = np.float32(np.sqrt(sq))
    return q / n


def make_gaussian(builder: CloudBuilder, position, log_scale, opacity_logit, rng: Rng):
    """makeGaussian (SplatRasterTest.cpp:27-41)."""
    q = [np.float32(rng.normal()) for _ in range(4)]
    if float(np.sqrt(np.float32(q[1] * q[1] + q[3] * q[3]) + np.float32(q[2] * q[2] + q[0] * q[0]))) < 1e-3:
        q = [1.0, 0.0, 0.0, 0.0]
    q = _normalized_quat(q)
    dc = [np.float32(rng.uniform(0.2, 1.2)) for _ in range(3)]
    rest = [np.float32(rng.uniform(-0.3, 0.3)) for _ in range(3 * builder.rest)]
    ls = np.float32(log_scale)
    builder.add(position, [ls, ls - np.float32(0.2), ls + np.float32(0.3)], q, opacity_logit, dc,
                rest if builder.rest else None)


def make_overlapping_cloud(sh_degree: int, count: int = 6):
    """makeOverlappingCloud (SplatRasterTest.cpp:45-59)."""
    builder = CloudBuilder(rest_per_channel(sh_degree))
    rng = Rng(77)
    for _ in range(count):
        pos = [np.float32(rng.uniform(-0.4, 0.4)), np.float32(rng.uniform(-0.3, 0.3)),
               np.float32(rng.uniform(-0.3, 0.3))]
        ls = np.float32(rng.uniform(-2.6, -2.0))
        op = np.float32(rng.uniform(-0.5, 1.5))
        make_gaussian(builder, pos, ls, op, rng)
    return builder.params(), builder.rest


def make_target(values: int, seed: int) -> np.ndarray:
    """makeTarget (SplatRasterTest.cpp:61-66)."""
    rng = Rng(seed)
    return np.array([np.float32(rng.uniform(0.0, 1.0)) for _ in range(values)], dtype=np.float32)


def truth_cloud():
    """truthCloud (SplatTrainerTest.cpp:41-57)."""
    builder = CloudBuilder(0)
    C0 = np.float32(0.28209479177387814)
    positions = [(-0.25, 0.0, 0.0), (0.25, 0.0, 0.0), (0.0, 0.2, 0.2)]
    colors = [(0.9, 0.2, 0.2), (0.2, 0.8, 0.3), (0.3, 0.3, 0.9)]
    ls = np.log(np.float32(0.12)).astype(np.float32)
    for p, c in zip(positions, colors):
        dc = [(np.float32(v) - np.float32(0.5)) / C0 for v in c]
        builder.add(p, [ls, ls, ls], [1, 0, 0, 0], 4.0, dc)
    return builder.params(), 0


def rough_start(count: int = 24, seed: int = 3):
    """roughStart (SplatTrainerTest.cpp:72-87)."""
    builder = CloudBuilder(0)
    rng = Rng(seed)
    ls = np.log(np.float32(0.1)).astype(np.float32)
    for _ in range(count):
        pos = [np.float32(rng.uniform(-0.4, 0.4)), np.float32(rng.uniform(-0.3, 0.3)),
               np.float32(rng.uniform(-0.3, 0.3))]
        builder.add(pos, [ls, ls, ls], [1, 0, 0, 0], 0.0, [0, 0, 0])
    return builder.params(), 0


def random_cloud(seed: int, count: int, sh_degree: int, log_scale_mean: float = -4.0):
    """A cloud with the benchmark distributions (means U[-1,1]^3, log sigma
    N(mean, 0.5), random unit quaternions, opacity logits N(0,1), RGB from dc
    N(0.5, 0.1), sh_rest N(0, 0.1)), generated with numpy for test sizes."""
    rs = np.random.default_rng(seed)
    rest = rest_per_channel(sh_degree)
    P = param_count(rest)
    p = np.zeros((P, count), dtype=np.float32)
    p[0:3] = rs.uniform(-1, 1, (3, count))
    p[3:6] = rs.normal(log_scale_mean, 0.5, (3, count))
    q = rs.normal(0, 1, (4, count))
    q /= np.linalg.norm(q, axis=0, keepdims=True)
    p[6:10] = q
    p[10] = rs.normal(0, 1, count)
    C0 = 0.28209479177387814
    p[11:14] = (rs.normal(0.5, 0.1, (3, count)) - 0.5) / C0
    if rest:
        p[14:] = rs.normal(0, 0.1, (3 * rest, count))
    return np.ascontiguousarray(p), rest


def orbit_views(count: int, width: int, height: int, radius: float = 3.0, fov: float = 60.0,
                seed: int = 3):
    """`count` cameras on a Fibonacci sphere of `radius` looking at the origin
    with a horizontal field of view `fov` (phoneIntrinsics, SyntheticScene.cpp:129-138)."""
    fx = (width * 0.5) / math.tan(math.radians(fov) * 0.5)
    views = []
    golden = math.pi * (3.0 - math.sqrt(5.0))
    rs = np.random.default_rng(seed)
    offset = rs.uniform(0, 2 * math.pi)
    for i in range(count):
        y = 1.0 - 2.0 * (i + 0.5) / count
        r = math.sqrt(max(0.0, 1.0 - y * y))
        a = golden * i + offset
        eye = radius * np.array([r * math.cos(a), y, r * math.sin(a)])
        R = look_at(eye, np.zeros(3))
        views.append(View((fx, fx, width * 0.5 - 0.5, height * 0.5 - 0.5), width, height, R,
                          -R @ eye))
    return views


# ------------------------------------------------------------ oracle calls


# pxo_splat_f64 with its C alignment padding
PROJECTED_F64_DTYPE = np.dtype([
    ("index", np.int32), ("mean", np.float64, 2), ("cov2d", np.float64, 3),
    ("conic", np.float64, 3), ("depth", np.float64), ("radius", np.float64),
    ("color", np.float64, 3), ("opacity", np.float64), ("clamped", np.uint32)], align=True)
assert PROJECTED_F64_DTYPE.itemsize == 128


def options(**kw) -> RasterOptions:
    return RasterOptions(**kw)


def oracle_project(params, rest, sh_degree, cam: Camera, opt: RasterOptions):
    n = params.shape[1]
    out = np.zeros(max(n, 1), dtype=PROJECTED_DTYPE)
    count = pxo().pxo_project_f32(as_ptr(params), n, rest, sh_degree, ct.byref(cam),
                                  ct.byref(opt), as_ptr(out))
    return out[:count].copy()


def oracle_tiles(projected, width, height):
    """(offsets, entries as projected indices)."""
    cols, rows = (width + 15) // 16, (height + 15) // 16
    offsets = np.zeros(cols * rows + 1, dtype=np.int32)
    proj = np.ascontiguousarray(projected)
    total = pxo().pxo_build_tiles_f32(as_ptr(proj), len(proj), width, height, as_ptr(offsets),
                                      None, 0)
    entries = np.zeros(max(total, 1), dtype=np.int32)
    pxo().pxo_build_tiles_f32(as_ptr(proj), len(proj), width, height, as_ptr(offsets),
                              as_ptr(entries), total)
    return offsets, entries[:total]


def oracle_rasterize(projected, cam: Camera, opt: RasterOptions):
    proj = np.ascontiguousarray(projected)
    rgb = np.zeros(cam.width * cam.height * 3, dtype=np.float32)
    T = np.zeros(cam.width * cam.height, dtype=np.float32)
    pxo().pxo_rasterize_f32(as_ptr(proj), len(proj), ct.byref(cam), ct.byref(opt), as_ptr(rgb),
                            as_ptr(T))
    return rgb, T


def oracle_pixel_decisions(projected, cam: Camera, opt: RasterOptions):
    """Per pixel, walking the list in `projected`'s order as the compositing loop
    does: (margin, kind, tie). margin is the least relative distance of any
    decision quantity (power, alpha against the floor and the 0.99 cap, T
    against the cutoff) from its threshold; kind says which (1 power, 2 floor,
    3 cap, 4 cutoff); tie is set where two contributing entries share a depth."""
    proj = np.ascontiguousarray(projected)
    n = cam.width * cam.height
    margin = np.zeros(n, dtype=np.float32)
    kind = np.zeros(n, dtype=np.int32)
    tie = np.zeros(n, dtype=np.int32)
    pxo().pxo_pixel_decisions_f32(as_ptr(proj), len(proj), ct.byref(cam), ct.byref(opt),
                                  as_ptr(margin), as_ptr(kind), as_ptr(tie))
    return margin, kind, tie.astype(bool)


def relative_error(got, want, floor=1e-3):
    """|got - want| / max(|want|, floor), elementwise."""
    return np.abs(np.asarray(got, np.float64) - want) / np.maximum(np.abs(want), floor)


def explain_image_differences(got, want, channels, margin, tie, rtol=1e-5, floor=1e-3,
                              flip_margin=2e-5):
    """Classifies every image value off by more than `rtol` (relative, with the
    given floor). A value is explained when its pixel had a decision within
    `flip_margin` of its threshold (a branch flip: the two sides' inputs differ
    in the last bits) or two contributing entries at one depth (a depth tie,
    whose order is the sort's tie-break). Returns a dict of counts; `unexplained`
    must be 0."""
    err = relative_error(got, want, floor).reshape(-1, channels)
    bad_px = (err > rtol).any(axis=1)
    flip = margin < flip_margin
    return {"values": int(err.size), "beyond_tol": int((err > rtol).sum()),
            "pixels_beyond_tol": int(bad_px.sum()),
            "flip_pixels": int((bad_px & flip).sum()),
            "tie_pixels": int((bad_px & ~flip & tie).sum()),
            "unexplained": int((bad_px & ~flip & ~tie).sum()),
            "candidate_flip_pixels": int(flip.sum()), "candidate_tie_pixels": int(tie.sum()),
            "max_rel_err": float(err.max()) if err.size else 0.0,
            "max_rel_err_explained_excluded":
                float(err[~(flip | tie)].max()) if (~(flip | tie)).any() else 0.0}


def oracle_loss(rendered, target, width, height, ssim_weight, want_grad=True):
    grad = np.zeros_like(rendered) if want_grad else None
    loss = pxo().pxo_photometric_loss_f32(as_ptr(rendered), as_ptr(target), width, height,
                                          ct.c_float(ssim_weight),
                                          as_ptr(grad) if want_grad else None)
    return loss, grad


def oracle_loss_f64(rendered, target, width, height, ssim_weight):
    """photometricLoss evaluated in double precision (the oracle's double
    instantiation) on float images."""
    lib = pxo()
    lib.pxo_photometric_loss_f64.restype = ct.c_double
    r = np.ascontiguousarray(rendered, dtype=np.float64)
    t = np.ascontiguousarray(target, dtype=np.float64)
    return float(lib.pxo_photometric_loss_f64(as_ptr(r), as_ptr(t), width, height,
                                              ct.c_double(ssim_weight), None))


def oracle_ssim(rendered, target, width, height, want_grad=True):
    grad = np.zeros_like(rendered) if want_grad else None
    s = pxo().pxo_mean_ssim_f32(as_ptr(rendered), as_ptr(target), width, height,
                                as_ptr(grad) if want_grad else None)
    return s, grad


def oracle_backward(params, rest, sh_degree, cam, opt, projected, dL):
    n = params.shape[1]
    grads = np.zeros_like(params)
    screen = np.zeros(n, dtype=np.float32)
    visible = np.zeros(n, dtype=np.int32)
    proj = np.ascontiguousarray(projected)
    pxo().pxo_backward_f32(as_ptr(params), n, rest, sh_degree, ct.byref(cam), ct.byref(opt),
                           as_ptr(proj), len(proj), None, as_ptr(dL), as_ptr(grads),
                           as_ptr(screen), as_ptr(visible))
    return grads, screen, visible


def oracle_render_and_accumulate(params, rest, sh_degree, cam, opt, target, ssim_weight):
    n = params.shape[1]
    grads = np.zeros_like(params)
    screen = np.zeros(n, dtype=np.float32)
    visible = np.zeros(n, dtype=np.int32)
    loss = pxo().pxo_render_and_accumulate_f32(
        as_ptr(params), n, rest, sh_degree, ct.byref(cam), ct.byref(opt), as_ptr(target),
        ct.c_float(ssim_weight), as_ptr(grads), as_ptr(screen), as_ptr(visible))
    return loss, grads, screen, visible


def oracle_gradient_f64_in_order(params, rest, sh_degree, cam, opt, order, target,
                                 ssim_weight):
    """The loss gradient evaluated in double precision (the oracle's double
    instantiation of projection, compositing, loss and backward) over the
    splats of `order` (gaussian indices, near to far, as a float projection
    listed them) in that order: the same entries and tie order as the float
    computation, without its rounding. Returns (loss, grads64)."""
    lib = pxo()
    lib.pxo_project_f64.restype = ct.c_int32
    lib.pxo_photometric_loss_f64.restype = ct.c_double
    n = params.shape[1]
    p64 = np.ascontiguousarray(params, dtype=np.float64)
    out = np.zeros(max(n, 1), dtype=PROJECTED_F64_DTYPE)
    count = lib.pxo_project_f64(as_ptr(p64), n, rest, sh_degree, ct.byref(cam), ct.byref(opt),
                                as_ptr(out))
    proj = out[:count]
    where = np.full(n, -1, dtype=np.int64)
    where[proj["index"]] = np.arange(count)
    pick = where[np.asarray(order)]
    listed = np.ascontiguousarray(proj[pick[pick >= 0]])
    pixels = cam.width * cam.height
    rgb = np.zeros(pixels * 3, dtype=np.float64)
    lib.pxo_rasterize_f64(as_ptr(listed), len(listed), ct.byref(cam), ct.byref(opt),
                          as_ptr(rgb), None)
    t64 = np.ascontiguousarray(target, dtype=np.float64)
    dL = np.zeros(pixels * 3, dtype=np.float64)
    loss = lib.pxo_photometric_loss_f64(as_ptr(rgb), as_ptr(t64), cam.width, cam.height,
                                        ct.c_double(ssim_weight), as_ptr(dL))
    grads = np.zeros_like(p64)
    screen = np.zeros(n, dtype=np.float64)
    visible = np.zeros(n, dtype=np.int32)
    lib.pxo_backward_f64(as_ptr(p64), n, rest, sh_degree, ct.byref(cam), ct.byref(opt),
                         as_ptr(listed), len(listed), as_ptr(rgb), as_ptr(dL), as_ptr(grads),
                         as_ptr(screen), as_ptr(visible))
    return float(loss), grads


def oracle_objective_f64(params64, rest, sh_degree, cam, opt, target64, ssim_weight):
    return pxo().pxo_objective_f64(as_ptr(params64), params64.shape[1], rest, sh_degree,
                                   ct.byref(cam), ct.byref(opt), as_ptr(target64),
                                   ct.c_double(ssim_weight))


# --------------------------------------------------------- reference calls


def ref_camera(view: View, kind="ieee") -> Camera:
    cam = Camera()
    ref(kind).ref_camera(*view.ref_args(), ct.byref(cam))
    return cam


def ref_project(params, rest, sh_degree, view: View, opt: RasterOptions, kind="ieee"):
    n = params.shape[1]
    out = np.zeros(max(n, 1), dtype=PROJECTED_DTYPE)
    count = ref(kind).ref_project(as_ptr(params), n, rest, sh_degree, *view.ref_args(),
                                  ct.byref(opt), as_ptr(out))
    return out[:count].copy()


def ref_render(params, rest, sh_degree, view: View, opt: RasterOptions, kind="ieee"):
    rgb = np.zeros(view.width * view.height * 3, dtype=np.float32)
    T = np.zeros(view.width * view.height, dtype=np.float32)
    ref(kind).ref_render(as_ptr(params), params.shape[1], rest, sh_degree, *view.ref_args(),
                         ct.byref(opt), as_ptr(rgb), as_ptr(T))
    return rgb, T


def ref_rasterize(projected, view: View, opt: RasterOptions, kind="ieee"):
    proj = np.ascontiguousarray(projected)
    rgb = np.zeros(view.width * view.height * 3, dtype=np.float32)
    T = np.zeros(view.width * view.height, dtype=np.float32)
    ref(kind).ref_rasterize(as_ptr(proj), len(proj), *view.ref_args(), ct.byref(opt),
                            as_ptr(rgb), as_ptr(T))
    return rgb, T


def projected_from_fixture(d):
    """The projected list a golden fixture stores as proj_* columns, in its
    stored order."""
    n = len(d["proj_index"])
    p = np.zeros(n, dtype=PROJECTED_DTYPE)
    for name in PROJECTED_DTYPE.names:
        p[name] = d[f"proj_{name}"]
    return p


def tie_and_flip_pixels(orders, cam: Camera, opt: RasterOptions):
    """(margin, tie) per pixel over several orders of one projected set: the
    least decision margin and whether a depth tie decides the pixel in any of
    them."""
    margin, tie = None, None
    for proj in orders:
        m, _, t = oracle_pixel_decisions(proj, cam, opt)
        margin = m if margin is None else np.minimum(margin, m)
        tie = t if tie is None else (tie | t)
    return margin, tie


def tie_ordered(projected):
    """A projected list re-sorted near to far with equal depths by gaussian
    index: the order the device produces (the reference's std::sort leaves
    equal depths in an unspecified order)."""
    return np.sort(np.ascontiguousarray(projected), order=["depth", "index"], kind="stable")


def ref_render_and_accumulate_projected(params, rest, sh_degree, view: View, opt: RasterOptions,
                                        projected, target, ssim_weight, kind="ieee"):
    """The reference's rasterizeSplats, photometricLoss and
    rasterizeSplatsBackward on `projected` in its given order:
    (loss, rgb, grads, screen_gradient, visible_count)."""
    n = params.shape[1]
    proj = np.ascontiguousarray(projected)
    rgb = np.zeros(view.width * view.height * 3, dtype=np.float32)
    grads = np.zeros_like(params)
    screen = np.zeros(n, dtype=np.float32)
    visible = np.zeros(n, dtype=np.int32)
    loss = ref(kind).ref_render_and_accumulate_projected(
        as_ptr(params), n, rest, sh_degree, *view.ref_args(), ct.byref(opt), as_ptr(proj),
        len(proj), as_ptr(np.ascontiguousarray(target, dtype=np.float32)),
        ct.c_float(ssim_weight), as_ptr(rgb), as_ptr(grads), as_ptr(screen), as_ptr(visible))
    return loss, rgb, grads, screen, visible


def tie_runs(depth_bits):
    """[(begin, end)] of the runs of equal values in a sorted sequence."""
    d = np.asarray(depth_bits)
    if len(d) == 0:
        return []
    cuts = np.flatnonzero(d[1:] != d[:-1]) + 1
    starts = np.concatenate([[0], cuts])
    ends = np.concatenate([cuts, [len(d)]])
    return list(zip(starts.tolist(), ends.tolist()))


def lists_equal_up_to_ties(offsets, got, want, depth_of):
    """Per-tile lists (flat gaussian ids cut by `offsets`) that hold the same
    ids in the same order, except that within each run of equal depth inside a
    tile the ids may come in any order. Returns (ok, runs, runs_reordered)."""
    got = np.asarray(got)
    want = np.asarray(want)
    if got.shape != want.shape:
        return False, 0, 0
    if not np.array_equal(depth_of[got].view(np.uint32), depth_of[want].view(np.uint32)):
        return False, 0, 0
    runs = reordered = 0
    for tile in range(len(offsets) - 1):
        lo, hi = int(offsets[tile]), int(offsets[tile + 1])
        dw = depth_of[want[lo:hi]].view(np.uint32)
        for b, e in tie_runs(dw):
            g, w = got[lo + b:lo + e], want[lo + b:lo + e]
            if e - b > 1:
                runs += 1
                if not np.array_equal(g, w):
                    reordered += 1
                    if not np.array_equal(np.sort(g), np.sort(w)):
                        return False, runs, reordered
            elif g[0] != w[0]:
                return False, runs, reordered
    return True, runs, reordered


def ref_loss(rendered, target, width, height, ssim_weight, kind="ieee"):
    grad = np.zeros_like(rendered)
    loss = ref(kind).ref_photometric_loss(as_ptr(rendered), as_ptr(target), width, height,
                                          ct.c_float(ssim_weight), as_ptr(grad))
    return loss, grad


def ref_ssim(rendered, target, width, height, kind="ieee"):
    grad = np.zeros_like(rendered)
    s = ref(kind).ref_mean_ssim(as_ptr(rendered), as_ptr(target), width, height, as_ptr(grad))
    return s, grad


def ref_backward(params, rest, sh_degree, view, opt, dL, kind="ieee"):
    n = params.shape[1]
    grads = np.zeros_like(params)
    screen = np.zeros(n, dtype=np.float32)
    visible = np.zeros(n, dtype=np.int32)
    ref(kind).ref_backward(as_ptr(params), n, rest, sh_degree, *view.ref_args(), ct.byref(opt),
                           as_ptr(dL), as_ptr(grads), as_ptr(screen), as_ptr(visible))
    return grads, screen, visible


def ref_render_and_accumulate(params, rest, sh_degree, view, opt, target, ssim_weight,
                              kind="ieee"):
    n = params.shape[1]
    grads = np.zeros_like(params)
    screen = np.zeros(n, dtype=np.float32)
    visible = np.zeros(n, dtype=np.int32)
    loss = ref(kind).ref_render_and_accumulate(
        as_ptr(params), n, rest, sh_degree, *view.ref_args(), ct.byref(opt), as_ptr(target),
        ct.c_float(ssim_weight), as_ptr(grads), as_ptr(screen), as_ptr(visible))
    return loss, grads, screen, visible


def ref_densify(params, rest, screen, visible, config: TrainConfig, extent, iteration, rng_state,
                kind="ieee"):
    n = params.shape[1]
    P = params.shape[0]
    buf = np.zeros(P * max(config.max_gaussians, n), dtype=np.float32)
    buf[: P * n] = params.reshape(-1)
    source = np.zeros(max(config.max_gaussians, 1), dtype=np.int32)
    st = ct.c_uint32(rng_state)
    cl, sp, pr = ct.c_int32(), ct.c_int32(), ct.c_int32()
    count = ref(kind).ref_densify(as_ptr(buf), n, rest, as_ptr(screen), as_ptr(visible),
                                  ct.byref(config), ct.c_float(extent), iteration, ct.byref(st),
                                  as_ptr(source), ct.byref(cl), ct.byref(sp), ct.byref(pr))
    out = buf[: P * count].reshape(P, count).copy()
    return out, source[:count].copy(), st.value, (cl.value, sp.value, pr.value)


def oracle_densify(params, rest, screen, visible, config: TrainConfig, extent, iteration,
                   rng_state):
    n = params.shape[1]
    P = params.shape[0]
    buf = np.zeros(P * max(config.max_gaussians, n) + P, dtype=np.float32)
    buf[: P * n] = params.reshape(-1)
    source = np.zeros(max(config.max_gaussians, 1), dtype=np.int32)
    st = ct.c_uint32(rng_state)
    cl, sp, pr = ct.c_int32(), ct.c_int32(), ct.c_int32()
    count = pxo().pxo_densify_and_prune(as_ptr(buf), n, rest, as_ptr(screen), as_ptr(visible),
                                        ct.byref(config), ct.c_float(extent), iteration,
                                        ct.byref(st), as_ptr(source), ct.byref(cl),
                                        ct.byref(sp), ct.byref(pr))
    out = buf[: P * count].reshape(P, count).copy()
    return out, source[:count].copy(), st.value, (cl.value, sp.value, pr.value)


class RefTrainer:
    """The reference's SplatTrainer with its CPU backend."""

    def __init__(self, params, rest, sh_degree, views, images, config: TrainConfig, kind="ieee"):
        self.lib = ref(kind)
        self.rest = rest
        self.P = params.shape[0]
        nv = len(views)
        K = np.ascontiguousarray(np.array([v.K for v in views], dtype=np.float64).reshape(-1))
        sizes = np.ascontiguousarray(np.array([[v.width, v.height] for v in views],
                                              dtype=np.int32).reshape(-1))
        R = np.ascontiguousarray(np.array([np.asarray(v.R).reshape(9) for v in views],
                                          dtype=np.float64).reshape(-1))
        t = np.ascontiguousarray(np.array([np.asarray(v.t).reshape(3) for v in views],
                                          dtype=np.float64).reshape(-1))
        self._images = [np.ascontiguousarray(im, dtype=np.float32) for im in images]
        ptrs = (ct.c_void_p * max(nv, 1))(*[im.ctypes.data for im in self._images])
        self.config = config
        create = self.lib.ref_shim_trainer_create if kind == "shim" else self.lib.ref_trainer_create
        self.handle = create(
            as_ptr(params), params.shape[1], rest, sh_degree, nv,
            as_ptr(K) if nv else None, as_ptr(sizes) if nv else None,
            as_ptr(R) if nv else None, as_ptr(t) if nv else None, ptrs, ct.byref(config))

    def step(self) -> bool:
        return bool(self.lib.ref_trainer_step(self.handle))

    def train(self, cancel_at: int = 0):
        seen = ct.c_int()
        done = self.lib.ref_trainer_train(self.handle, cancel_at, ct.byref(seen))
        return bool(done), seen.value

    def state(self):
        it, cnt, sh = ct.c_int(), ct.c_int(), ct.c_int()
        ll, sm, ex = ct.c_float(), ct.c_float(), ct.c_float()
        self.lib.ref_trainer_state(self.handle, ct.byref(it), ct.byref(cnt), ct.byref(ll),
                                   ct.byref(sm), ct.byref(ex), ct.byref(sh))
        return dict(iteration=it.value, count=cnt.value, last_loss=ll.value,
                    smoothed_loss=sm.value, extent=ex.value, sh_degree=sh.value)

    def cloud(self):
        cap = max(self.config.max_gaussians, self.state()["count"])
        buf = np.zeros(self.P * cap, dtype=np.float32)
        n = self.lib.ref_trainer_download(self.handle, as_ptr(buf), cap)
        return buf[: self.P * n].reshape(self.P, n).copy()

    def finish(self):
        cap = max(self.config.max_gaussians, self.state()["count"])
        buf = np.zeros(self.P * cap, dtype=np.float32)
        sh = ct.c_int()
        n = self.lib.ref_trainer_finish(self.handle, as_ptr(buf), cap, ct.byref(sh))
        return buf[: self.P * n].reshape(self.P, n).copy(), sh.value

    def __del__(self):
        if getattr(self, "handle", None):
            self.lib.ref_trainer_destroy(self.handle)
            self.handle = None

"""The reference arm of the training-step benchmark (baseline infrastructure).

Runs the reference's own CPU splat trainer, compiled from its sources into
oracle/_ref/libpxref_fast.so with its release flags (-O3 -ffast-math
-fno-finite-math-only), on the multi-view workload: every step renders,
scores (L1 + SSIM) and differentiates a batch of views, one view per host
thread, with the reference's CpuSplatBackend::renderAndAccumulate
(SplatTrainer.cpp:104-113), adds the per-view gradients and takes the
reference trainer's own Adam step (applyGradients, SplatTrainer.cpp:218-256).
See ref_batch_trainer_* in oracle/ref_api.cpp.

The scene is built without the product library: the clouds come from the
reference's own generator (parallax::testing::Rng, SyntheticScene.h:80-107,
through ref_synthetic_cloud), the cameras from `orbit_cameras` below, and the
targets are the truth cloud rendered by the reference's renderSplats,
quantised to 8-bit frames and divided by 255, as the product arm's are.
tests/test_ref_bench.py checks that this scene is the product's, bit for bit.
"""
from __future__ import annotations

import ctypes as ct
import math
import os
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_vp = ct.c_void_p


def library(kind: str = "fast") -> ct.CDLL:
    path = os.path.join(HERE, "_ref", f"libpxref_{kind}.so")
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing (make -C oracle ref, with the reference "
                                "sources present)")
    lib = ct.CDLL(path)
    lib.ref_synthetic_cloud.argtypes = [ct.c_uint64, ct.c_int, ct.c_int, ct.c_float, _vp]
    lib.ref_render.argtypes = [_vp, ct.c_int, ct.c_int, ct.c_int, _vp, ct.c_int, ct.c_int, _vp,
                               _vp, _vp, _vp, _vp]
    lib.ref_render.restype = None
    lib.ref_sizeof_train_config.restype = ct.c_int
    lib.ref_sizeof_raster_options.restype = ct.c_int
    lib.ref_bench_settings.argtypes = [_vp, _vp, ct.c_int, ct.c_int, ct.c_int]
    lib.ref_bench_settings.restype = None
    lib.ref_batch_trainer_create.restype = _vp
    lib.ref_batch_trainer_create.argtypes = [_vp, ct.c_int, ct.c_int, ct.c_int, ct.c_int, _vp,
                                             _vp, _vp, _vp, _vp, _vp, ct.c_int]
    lib.ref_batch_trainer_step.argtypes = [_vp, ct.c_int, _vp, _vp]
    lib.ref_batch_trainer_step.restype = ct.c_int
    lib.ref_batch_trainer_download.argtypes = [_vp, _vp, ct.c_int]
    lib.ref_batch_trainer_download.restype = ct.c_int
    lib.ref_batch_trainer_destroy.argtypes = [_vp]
    lib.ref_batch_trainer_destroy.restype = None
    return lib


def rest_per_channel(sh_degree: int) -> int:
    return (sh_degree + 1) ** 2 - 1


def synthetic_cloud(lib, seed: int, count: int, sh_degree: int, log_scale_mean: float = -4.0):
    rest = rest_per_channel(sh_degree)
    params = np.zeros((14 + 3 * rest, count), dtype=np.float32)
    if lib.ref_synthetic_cloud(seed, count, rest, ct.c_float(log_scale_mean),
                               params.ctypes.data) != 0:
        raise ValueError("ref_synthetic_cloud failed")
    return params


def _look_at(eye):
    """Camera-from-world rotation looking from `eye` at the origin (+X right,
    +Y down, +Z forward; SyntheticScene.cpp:235-258)."""
    forward = -np.asarray(eye, dtype=np.float64)
    if np.linalg.norm(forward) < 1e-9:
        forward = np.array([0.0, 0.0, 1.0])
    forward /= np.linalg.norm(forward)
    up = np.array([0.0, 1.0, 0.0])
    if abs(forward[1]) > 0.999:
        up = np.array([1.0, 0.0, 0.0]) if abs(forward[0]) < 0.9 else np.array([0.0, 0.0, 1.0])
    right = np.cross(forward, up)
    right /= np.linalg.norm(right)
    down = np.cross(forward, right)
    return np.stack([right, down, forward])


def orbit_cameras(seed: int, count: int, width: int, height: int, radius: float = 3.0,
                  fov_degrees: float = 60.0):
    """The benchmark's camera pool: `count` cameras on a Fibonacci sphere of
    `radius`, spun by a seeded angle, looking at the origin with phoneIntrinsics
    (SyntheticScene.cpp:129-138) at a horizontal field of view `fov_degrees`.
    Returns (K [count,4], R [count,9], t [count,3]) in double precision."""
    rs = np.random.default_rng(seed)
    fx = (width * 0.5) / math.tan(math.radians(fov_degrees) * 0.5)
    golden = math.pi * (3.0 - math.sqrt(5.0))
    spin = rs.uniform(0.0, 2.0 * math.pi)
    K = np.tile(np.array([fx, fx, width * 0.5 - 0.5, height * 0.5 - 0.5]), (count, 1))
    R = np.zeros((count, 9))
    t = np.zeros((count, 3))
    for i in range(count):
        y = 1.0 - 2.0 * (i + 0.5) / count
        r = math.sqrt(max(0.0, 1.0 - y * y))
        a = golden * i + spin
        eye = radius * np.array([r * math.cos(a), y, r * math.sin(a)])
        rot = _look_at(eye)
        R[i] = rot.reshape(9)
        t[i] = -rot @ eye
    return K, R, t


class ReferenceBatchStep:
    """The reference trainer on a multi-view workload: `gaussians` SH
    `sh_degree`, a pool of `pool` cameras at width x height, `views` views per
    step on `threads` host threads. Targets are rendered for `target_views`
    (default: the whole pool)."""

    def __init__(self, gaussians: int, sh_degree: int, pool: int, width: int, height: int,
                 threads: int, target_views=None, kind: str = "fast", log=None):
        self.lib = lib = library(kind)
        self.log = log or (lambda *_: None)
        t0 = time.perf_counter()
        self.rest = rest_per_channel(sh_degree)
        self.sh_degree = sh_degree
        self.count = gaussians
        truth = synthetic_cloud(lib, 1, gaussians, sh_degree)
        self.start = synthetic_cloud(lib, 2, gaussians, sh_degree)
        self.K, self.R, self.t = orbit_cameras(3, pool, width, height)
        self.width, self.height = width, height
        self.config = ct.create_string_buffer(lib.ref_sizeof_train_config())
        self.options = ct.create_string_buffer(lib.ref_sizeof_raster_options())
        lib.ref_bench_settings(self.config, self.options, sh_degree, 100000,
                               max(600000, gaussians))
        ids = list(range(pool)) if target_views is None else sorted(set(target_views))
        images = {}
        pending = list(ids)
        lock = threading.Lock()

        def render_worker():
            while True:
                with lock:
                    if not pending:
                        return
                    v = pending.pop()
                rgb = np.zeros(width * height * 3, dtype=np.float32)
                lib.ref_render(truth.ctypes.data, gaussians, self.rest, sh_degree,
                               self.K[v].ctypes.data, width, height, self.R[v].ctypes.data,
                               self.t[v].ctypes.data, self.options, rgb.ctypes.data, None)
                frame = np.rint(np.clip(rgb, 0.0, 1.0) * 255.0).astype(np.uint8)
                images[v] = frame.astype(np.float32) / np.float32(255.0)

        workers = [threading.Thread(target=render_worker)
                   for _ in range(max(1, min(os.cpu_count() or 1, len(ids))))]
        for w in workers:
            w.start()
        for w in workers:
            w.join()
        del truth
        self.target_seconds = time.perf_counter() - t0
        self.log(f"reference targets: {len(ids)} views in {self.target_seconds:.1f} s")
        blank = np.zeros(0, dtype=np.float32)
        self._images = [images.get(v, blank) for v in range(pool)]
        ptrs = (ct.c_void_p * pool)(*[im.ctypes.data for im in self._images])
        sizes = np.tile(np.array([width, height], dtype=np.int32), (pool, 1))
        self.threads = threads
        self.handle = lib.ref_batch_trainer_create(
            self.start.ctypes.data, gaussians, self.rest, sh_degree, pool, self.K.ctypes.data,
            sizes.ctypes.data, self.R.ctypes.data, self.t.ctypes.data, ptrs, self.config,
            threads)
        self._images = None  # the trainer holds its own copies
        self.loss = float("nan")

    def step(self, view_ids) -> float:
        ids = (ct.c_int32 * len(view_ids))(*view_ids)
        loss = ct.c_float()
        if not self.lib.ref_batch_trainer_step(self.handle, len(view_ids), ids, ct.byref(loss)):
            raise RuntimeError("the reference trainer refused the step")
        self.loss = loss.value
        return self.loss

    def cloud(self) -> np.ndarray:
        out = np.zeros((14 + 3 * self.rest, self.count), dtype=np.float32)
        n = self.lib.ref_batch_trainer_download(self.handle, out.ctypes.data, self.count)
        if n != self.count:
            raise RuntimeError("the reference cloud changed size")
        return out

    def close(self):
        if self.handle:
            self.lib.ref_batch_trainer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

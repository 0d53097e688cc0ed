"""Seeded benchmark scenes in double precision (views) and float32 (clouds).

Camera rigs look at the origin with the reference's lookAt convention (+X
right, +Y down, +Z forward; SyntheticScene.cpp:235-258) and phoneIntrinsics
(SyntheticScene.cpp:129-138). Clouds come from pxs_synthetic_cloud.
"""
from __future__ import annotations

import math
from typing import List

import numpy as np

from .splat import GaussianCloud, SplatView, synthetic_cloud


def look_at(eye, target=(0.0, 0.0, 0.0)) -> np.ndarray:
    eye = np.asarray(eye, dtype=np.float64)
    forward = np.asarray(target, dtype=np.float64) - eye
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


def phone_intrinsics(width: int, height: int, fov_degrees: float = 60.0):
    fx = (width * 0.5) / math.tan(math.radians(fov_degrees) * 0.5)
    return (fx, fx, width * 0.5 - 0.5, height * 0.5 - 0.5)


def orbit_views(seed: int, count: int, width: int, height: int, radius: float = 3.0,
                fov_degrees: float = 60.0, layout: int = 0) -> List[SplatView]:
    """layout 0: Fibonacci sphere; layout 1: half on the upper hemisphere, half
    on a walk-around ring at jittered height +-0.2 and radius +-0.1."""
    rs = np.random.default_rng(seed)
    K = phone_intrinsics(width, height, fov_degrees)
    golden = math.pi * (3.0 - math.sqrt(5.0))
    spin = rs.uniform(0.0, 2.0 * math.pi)
    hemisphere = count // 2 if layout == 1 else count
    views = []
    for i in range(count):
        if i < hemisphere:
            u = (i + 0.5) / hemisphere
            y = u if layout == 1 else 1.0 - 2.0 * u
            r = math.sqrt(max(0.0, 1.0 - y * y))
            a = golden * i + spin
            eye = radius * np.array([r * math.cos(a), y, r * math.sin(a)])
        else:
            j, ring = i - hemisphere, count - hemisphere
            a = 2.0 * math.pi * j / ring + rs.uniform(-0.05, 0.05)
            rr = radius + rs.uniform(-0.1, 0.1)
            eye = np.array([rr * math.cos(a), rs.uniform(-0.2, 0.2), rr * math.sin(a)])
        R = look_at(eye)
        views.append(SplatView(K, width, height, R, -R @ eye))
    return views


def crop_view(view: SplatView, x0: int, y0: int, width: int, height: int) -> SplatView:
    """The same camera seeing only the window [x0, x0+width) x [y0, y0+height)."""
    fx, fy, cx, cy = view.K
    return SplatView((fx, fy, cx - x0, cy - y0), width, height, view.R, view.t)


WORKLOADS = {
    # name: gaussians, SH degree, views per step, camera pool, width, height, layout
    "c1": dict(gaussians=20_000, sh_degree=0, views_per_step=1, pool=16, width=320, height=240,
               layout=0),
    "c3": dict(gaussians=200_000, sh_degree=3, views_per_step=1, pool=64, width=1280, height=720,
               layout=1),
    "c4": dict(gaussians=1_000_000, sh_degree=3, views_per_step=8, pool=64, width=1920,
               height=1440, layout=0),
}


def workload_scene(name: str):
    """(truth cloud, start cloud, views): seed 1 truth, seed 2 start, seed 3 cameras."""
    w = WORKLOADS[name]
    truth = synthetic_cloud(1, w["gaussians"], w["sh_degree"])
    start = synthetic_cloud(2, w["gaussians"], w["sh_degree"])
    views = orbit_views(3, w["pool"], w["width"], w["height"], layout=w["layout"])
    return truth, start, views


# Uneven batch of independent scans: 32 scenes, gaussian counts log-uniform in
# [5k, 150k], each at a resolution drawn from three phone sizes, 4 views each.
MULTI_SCENE = dict(scenes=32, min_count=5_000, max_count=150_000, sh_degree=3,
                   views_per_scene=4, resolutions=((320, 240), (640, 480), (1280, 720)))


def multi_scene_workload(seed: int = 5, **overrides):
    """[(truth cloud, start cloud, views)] per scene, all seeded from `seed`."""
    w = dict(MULTI_SCENE, **overrides)
    rs = np.random.default_rng(seed)
    lo, hi = math.log(w["min_count"]), math.log(w["max_count"])
    scenes = []
    for s in range(w["scenes"]):
        count = int(round(math.exp(rs.uniform(lo, hi))))
        width, height = w["resolutions"][int(rs.integers(len(w["resolutions"])))]
        truth = synthetic_cloud(1000 + 2 * s, count, w["sh_degree"])
        start = synthetic_cloud(1001 + 2 * s, count, w["sh_degree"])
        views = orbit_views(3000 + s, w["views_per_scene"], width, height)
        scenes.append((truth, start, views))
    return scenes

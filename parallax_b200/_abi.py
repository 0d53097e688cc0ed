"""ctypes mirrors of the plain structs in include/pxs.h.

Pure declarations: importing this module loads no library, so host-side code
and the tests can build inputs without a GPU.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

PXS_OK = 0
PXS_ERR_INVALID = 1
PXS_ERR_CUDA = 2
PXS_ERR_NO_MEMORY = 3
PXS_ERR_CAPACITY = 4
PXS_ERR_UNAVAILABLE = 5
PXS_ERR_TIMEOUT = 6

PXS_FORMAT_PLY = 0
PXS_FORMAT_SPLAT = 1
PXS_FORMAT_SPZ = 2

TILE = 16
C_POSITION, C_LOG_SCALE, C_ROTATION, C_OPACITY, C_DC, C_SH_REST = 0, 3, 6, 10, 11, 14


def param_count(rest_per_channel: int) -> int:
    """Floats per gaussian: 14 + 3 * higher-order SH coefficients per channel."""
    return 14 + 3 * rest_per_channel


def rest_per_channel(sh_degree: int) -> int:
    """shRestPerChannel (GaussianCloud.h:16-27)."""
    return {0: 0, 1: 3, 2: 8, 3: 15}.get(int(sh_degree), 0)


class Camera(ct.Structure):
    """pxs_camera: the float camera the rasteriser consumes."""

    _fields_ = [
        ("R", ct.c_float * 9),
        ("t", ct.c_float * 3),
        ("center", ct.c_float * 3),
        ("fx", ct.c_float),
        ("fy", ct.c_float),
        ("cx", ct.c_float),
        ("cy", ct.c_float),
        ("tan_half_x", ct.c_float),
        ("tan_half_y", ct.c_float),
        ("width", ct.c_int32),
        ("height", ct.c_int32),
    ]


class RasterOptions(ct.Structure):
    """pxs_raster_options, RasterOptions (SplatRaster.h:31-52) with its defaults."""

    _fields_ = [
        ("background", ct.c_float * 3),
        ("sh_degree", ct.c_int32),
        ("min_alpha", ct.c_float),
        ("transmittance_cutoff", ct.c_float),
        ("screen_dilation", ct.c_float),
    ]

    def __init__(self, background=(0.0, 0.0, 0.0), sh_degree=0, min_alpha=None,
                 transmittance_cutoff=1e-4, screen_dilation=0.3):
        super().__init__()
        for c in range(3):
            self.background[c] = background[c]
        self.sh_degree = sh_degree
        # 1.f / 255.f evaluated in single precision, as the reference's default
        self.min_alpha = float(np.float32(1.0) / np.float32(255.0)) if min_alpha is None else min_alpha
        self.transmittance_cutoff = transmittance_cutoff
        self.screen_dilation = screen_dilation


class ProjectedSplat(ct.Structure):
    """pxs_projected_splat, ProjectedSplat (SplatRaster.h:56-72)."""

    _fields_ = [
        ("index", ct.c_int32),
        ("mean", ct.c_float * 2),
        ("cov2d", ct.c_float * 3),
        ("conic", ct.c_float * 3),
        ("depth", ct.c_float),
        ("radius", ct.c_float),
        ("color", ct.c_float * 3),
        ("opacity", ct.c_float),
        ("clamped", ct.c_uint32),
    ]


PROJECTED_DTYPE = np.dtype([
    ("index", np.int32), ("mean", np.float32, 2), ("cov2d", np.float32, 3),
    ("conic", np.float32, 3), ("depth", np.float32), ("radius", np.float32),
    ("color", np.float32, 3), ("opacity", np.float32), ("clamped", np.uint32),
])
assert PROJECTED_DTYPE.itemsize == ct.sizeof(ProjectedSplat) == 64


class Cloud(ct.Structure):
    """pxs_cloud: component-major parameters (host or device pointer)."""

    _fields_ = [
        ("params", ct.c_void_p),
        ("count", ct.c_int32),
        ("rest_per_channel", ct.c_int32),
        ("sh_degree", ct.c_int32),
    ]


class Gradients(ct.Structure):
    """pxs_gradients: every entry point adds into these arrays."""

    _fields_ = [
        ("params", ct.c_void_p),
        ("screen_gradient", ct.c_void_p),
        ("visible_count", ct.c_void_p),
    ]


class TrainConfig(ct.Structure):
    """pxs_train_config, SplatTrainingConfig (SplatTrainer.h:25-94)."""

    _fields_ = [
        ("iterations", ct.c_int32),
        ("position_lr_initial", ct.c_float),
        ("position_lr_final", ct.c_float),
        ("dc_lr", ct.c_float),
        ("sh_rest_lr_divider", ct.c_float),
        ("opacity_lr", ct.c_float),
        ("scale_lr", ct.c_float),
        ("rotation_lr", ct.c_float),
        ("adam_beta1", ct.c_float),
        ("adam_beta2", ct.c_float),
        ("adam_epsilon", ct.c_float),
        ("ssim_weight", ct.c_float),
        ("sh_degree", ct.c_int32),
        ("sh_increase_interval", ct.c_int32),
        ("densify_from_iteration", ct.c_int32),
        ("densify_until_iteration", ct.c_int32),
        ("densify_interval", ct.c_int32),
        ("densify_grad_threshold", ct.c_float),
        ("percent_dense", ct.c_float),
        ("split_scale_divider", ct.c_float),
        ("opacity_reset_interval", ct.c_int32),
        ("opacity_reset_value", ct.c_float),
        ("prune_opacity", ct.c_float),
        ("prune_scale_fraction", ct.c_float),
        ("max_gaussians", ct.c_int32),
        ("seed", ct.c_uint32),
    ]

    def __init__(self, **overrides):
        super().__init__()
        defaults = dict(
            iterations=7000, position_lr_initial=1.6e-4, position_lr_final=1.6e-6,
            dc_lr=2.5e-3, sh_rest_lr_divider=20.0, opacity_lr=0.05, scale_lr=5e-3,
            rotation_lr=1e-3, adam_beta1=0.9, adam_beta2=0.999, adam_epsilon=1e-15,
            ssim_weight=0.2, sh_degree=3, sh_increase_interval=1000,
            densify_from_iteration=500, densify_until_iteration=5000, densify_interval=100,
            densify_grad_threshold=2e-4, percent_dense=0.01, split_scale_divider=1.6,
            opacity_reset_interval=3000, opacity_reset_value=0.01, prune_opacity=0.005,
            prune_scale_fraction=0.1, max_gaussians=600000, seed=7,
        )
        defaults.update(overrides)
        for key, value in defaults.items():
            setattr(self, key, value)


class Progress(ct.Structure):
    """pxs_progress, SplatTrainingProgress (SplatTrainer.h:96-104)."""

    _fields_ = [
        ("iteration", ct.c_int32),
        ("total_iterations", ct.c_int32),
        ("gaussian_count", ct.c_int32),
        ("loss", ct.c_float),
        ("smoothed_loss", ct.c_float),
    ]


PROGRESS_FN = ct.CFUNCTYPE(ct.c_int, ct.POINTER(Progress), ct.c_void_p)


def camera_from_pose(K, width, height, R, t) -> Camera:
    """The float camera projectSplats derives from a double SplatView
    (SplatRaster.cpp:206-212): casts of R, t, fx, fy, cx, cy; the centre
    -R^T t (SE3.h:46) and 0.5 * size / f evaluated in double first.

    Eigen evaluates each coefficient of the 3x3 double product as
    a0*b0 + (a1*b1 + a2*b2), which is reproduced here.
    """
    K = [float(v) for v in K]
    R = np.asarray(R, dtype=np.float64).reshape(3, 3)
    t = np.asarray(t, dtype=np.float64).reshape(3)
    cam = Camera()
    for i in range(9):
        cam.R[i] = float(np.float32(R.flat[i]))
    center = []
    for i in range(3):
        a0, a1, a2 = -R[0, i], -R[1, i], -R[2, i]
        center.append(float(a0 * t[0] + (a1 * t[1] + a2 * t[2])))
    for i in range(3):
        cam.t[i] = float(np.float32(t[i]))
        cam.center[i] = float(np.float32(center[i]))
    cam.fx, cam.fy, cam.cx, cam.cy = (float(np.float32(v)) for v in K)
    cam.tan_half_x = float(np.float32(0.5 * width / K[0]))
    cam.tan_half_y = float(np.float32(0.5 * height / K[1]))
    cam.width = int(width)
    cam.height = int(height)
    return cam


def as_ptr(array: np.ndarray) -> ct.c_void_p:
    """Address of a C-contiguous numpy array."""
    assert array.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return ct.c_void_p(array.ctypes.data)

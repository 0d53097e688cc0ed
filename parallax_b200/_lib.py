"""Loads parallax_b200/libpxs.so and declares the C ABI of include/pxs.h.

There is no fallback: if the library is missing the import of the compute
entry points fails with an error that says how to build it.
"""
from __future__ import annotations

import ctypes as ct
import os

from . import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
# PXS_LIBRARY names another build of the same library (for example one compiled
# with different kernel parameters); the default is the in-tree build.
LIBRARY = os.environ.get("PXS_LIBRARY") or os.path.join(HERE, "libpxs.so")

_LIB = None

_vp = ct.c_void_p
_i32 = ct.c_int32
_i64 = ct.c_int64
_f32 = ct.c_float


def _declare(lib: ct.CDLL) -> None:
    sig = {
        "pxs_version": (ct.c_char_p, []),
        "pxs_train_config_defaults": (None, [_vp]),
        "pxs_train_config_validate": (ct.c_int, [_vp, ct.c_char_p, ct.c_size_t]),
        "pxs_camera_from_pose": (None, [_vp, _i32, _i32, _vp, _vp, _vp]),
        "pxs_gpu_availability": (ct.c_int, [_vp, ct.c_char_p, ct.c_size_t, ct.c_char_p,
                                            ct.c_size_t]),
        "pxs_context_create": (ct.c_int, [_i32, _vp]),
        "pxs_context_destroy": (None, [_vp]),
        "pxs_context_last_error": (ct.c_char_p, [_vp]),
        "pxs_context_set_stream": (ct.c_int, [_vp, _vp]),
        "pxs_context_synchronize": (ct.c_int, [_vp]),
        "pxs_project": (ct.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
        "pxs_tile_lists": (ct.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp]),
        "pxs_render": (ct.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
        "pxs_photometric_loss": (ct.c_int, [_vp, _vp, _vp, _i32, _i32, _f32, _vp, _vp]),
        "pxs_mean_ssim": (ct.c_int, [_vp, _vp, _vp, _i32, _i32, _vp, _vp]),
        "pxs_backward": (ct.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
        "pxs_render_and_accumulate": (ct.c_int, [_vp, _vp, _vp, _vp, _vp, _f32, _vp, _vp]),
        "pxs_render_and_accumulate_device": (ct.c_int, [_vp, _vp, _vp, _vp, _vp, _f32, _vp,
                                                        _vp]),
        "pxs_adam_device": (ct.c_int, [_vp, _vp, _vp, _vp, _vp, _i32, _i32, _vp, _f32, _f32,
                                       _f32, _f32, _f32, _i32]),
        "pxs_trainer_create": (ct.c_int, [_vp, _vp, _vp, _vp, _i32, _i32, _vp]),
        "pxs_trainer_destroy": (None, [_vp]),
        "pxs_trainer_last_error": (ct.c_char_p, [_vp]),
        "pxs_trainer_step": (ct.c_int, [_vp, _vp]),
        "pxs_trainer_train": (ct.c_int, [_vp, A.PROGRESS_FN, _vp, _vp]),
        "pxs_trainer_step_batch": (ct.c_int, [_vp, _i32, _vp, _i32, _vp]),
        "pxs_trainer_step_views": (ct.c_int, [_vp, _i32, _vp, _vp]),
        "pxs_trainer_state": (ct.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
        "pxs_trainer_stream": (ct.c_int, [_vp, _vp]),
        "pxs_trainer_render": (ct.c_int, [_vp, _vp, _vp, _vp, _vp]),
        "pxs_measure_fp32_peak": (ct.c_int, [_i32, _vp]),
        "pxs_trainer_set_timing": (ct.c_int, [_vp, _i32]),
        "pxs_trainer_stage_times": (ct.c_int, [_vp, _vp, _i32, _vp, _vp]),
        "pxs_trainer_step_info": (ct.c_int, [_vp, _vp, _vp]),
        "pxs_trainer_pair_stats": (ct.c_int, [_vp, _vp, _vp]),
        "pxs_trainer_set_images": (ct.c_int, [_vp, _i32, _vp, _vp]),
        "pxs_trainer_download": (ct.c_int, [_vp, _vp, _i32, _vp]),
        "pxs_trainer_finish": (ct.c_int, [_vp, _vp, _i32, _vp]),
        "pxs_train_splats": (ct.c_int, [_vp, _vp, _vp, _i32, _vp, A.PROGRESS_FN, _vp,
                                        ct.c_char_p, ct.c_size_t]),
        "pxs_densify_and_prune": (ct.c_int, [_vp, _vp, _vp, _i32, _vp, _vp, _vp, _f32, _i32,
                                             _vp, _vp, _vp, _vp, _vp]),
        "pxs_photometric_loss_static": (ct.c_int, [_vp, _vp, _i32, _i32, _i32, _f32, _vp, _vp,
                                                   _vp, _vp, ct.c_char_p, ct.c_size_t]),
        "pxs_set_raster_config": (ct.c_int, [_i32, _i32]),
        "pxs_get_raster_config": (ct.c_int, [_vp, _vp]),
        "pxs_set_raster_schedule": (ct.c_int, [_i32, _i32, _i32, _i32]),
        "pxs_trainer_autotune_report": (ct.c_int, [_vp, ct.c_char_p, ct.c_size_t]),
        "pxs_get_raster_schedule": (ct.c_int, [_vp, _vp, _vp, _vp]),
        "pxs_trainer_autotune": (ct.c_int, [_vp, _i32, _vp, _vp, _vp]),
        "pxs_trainer_accumulate": (ct.c_int, [_vp, _i32, _vp, _i32, _vp]),
        "pxs_trainer_create_scenes": (ct.c_int, [_vp, _vp, _i32, _vp, _vp, _vp, _i32, _vp]),
        "pxs_export_cloud": (ct.c_int, [_vp, _vp, _i32, _i32, _vp, ct.c_size_t, _vp]),
        "pxs_downscale_to_width": (ct.c_int, [_vp, _vp, _i32, _i32, _i32, _vp, _vp, _vp, _vp]),
        "pxs_initialize_from_points": (ct.c_int, [_vp, _vp, _vp, _i32, _i32, _f32, _vp, _vp]),
        "pxs_trainer_ingest_images": (ct.c_int, [_vp, _i32, _vp, _vp, _vp, _vp]),
        "pxs_trainer_stage_images": (ct.c_int, [_vp, _i32, _vp, _vp, _vp, _vp]),
        "pxs_trainer_export": (ct.c_int, [_vp, _i32, _i32, _vp, ct.c_size_t, _vp]),
        "pxs_trainer_apply": (ct.c_int, [_vp, _f32]),
        "pxs_trainer_gradients": (ct.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
        "pxs_trainer_reduction_block": (ct.c_int, [_vp, _vp, _vp]),
        "pxs_synthetic_cloud": (ct.c_int, [ct.c_uint64, _i32, _i32, _f32, _vp]),
        "pxs_synthetic_cameras": (ct.c_int, [ct.c_uint64, _i32, _i32, ct.c_double, _i32, _i32,
                                             ct.c_double, _vp]),
    }
    for name, (restype, argtypes) in sig.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes


def lib() -> ct.CDLL:
    """The loaded library (raises when it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBRARY):
            raise RuntimeError(
                f"{LIBRARY} is missing: build it with `make -C parallax_b200/csrc` "
                "(or __graft_entry__.build())")
        loaded = ct.CDLL(LIBRARY)
        _declare(loaded)
        _LIB = loaded
    return _LIB


class PxsError(RuntimeError):
    """A pxs entry point returned a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"pxs status {status}: {message}")
        self.status = status


def check(status: int, message_fn) -> None:
    if status != A.PXS_OK:
        msg = message_fn()
        if isinstance(msg, bytes):
            msg = msg.decode(errors="replace")
        raise PxsError(status, msg)

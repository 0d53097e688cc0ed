"""parallax_b200 -- a B200-native (sm_100a) Gaussian-splat training core.

The compute lives in parallax_b200/libpxs.so (hand-written CUDA kernels and a
C++ host runtime behind the C ABI of include/pxs.h); this package is its
Python binding. There is no CPU path: the compute entry points raise when the
library is missing.
"""
from ._abi import (  # noqa: F401
    PROJECTED_DTYPE,
    Camera,
    RasterOptions,
    TrainConfig,
    camera_from_pose,
    param_count,
    rest_per_channel,
)
from ._lib import LIBRARY, PxsError, lib  # noqa: F401
from .splat import (  # noqa: F401
    Context,
    GaussianCloud,
    SplatGradients,
    SplatTrainer,
    SplatTrainingProgress,
    SplatView,
    default_context,
    densify_and_prune,
    downscale_to_width,
    export_cloud,
    initialize_from_points,
    mean_ssim,
    photometric_loss,
    project_splats,
    rasterize_splats_backward,
    render_and_accumulate,
    render_splats,
    splat_gpu_availability,
    synthetic_cameras,
    synthetic_cloud,
    tile_lists,
    train_splats_on_gpu,
)

__version__ = "0.1.0"

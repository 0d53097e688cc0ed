"""Python mirror of the reference's splat interface over the C ABI.

Names follow engine/native/cpp/include/parallax/splat/{SplatRaster,SplatTrainer,
SplatDensify,VulkanSplatTrainer}.h in snake_case; clouds are numpy arrays in
the component-major layout of include/pxs.h (P x N float32).
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from . import _abi as A
from ._lib import PxsError, check, lib


@dataclass
class GaussianCloud:
    """GaussianCloud (GaussianCloud.h:56-72) as a P x N float32 array."""

    params: np.ndarray
    sh_degree: int = 0
    rest_per_channel: int = 0

    def __post_init__(self):
        self.params = np.ascontiguousarray(self.params, dtype=np.float32)
        assert self.params.shape[0] == A.param_count(self.rest_per_channel)

    @property
    def count(self) -> int:
        return int(self.params.shape[1])

    def c_struct(self) -> A.Cloud:
        c = A.Cloud()
        c.params = self.params.ctypes.data if self.count else None
        c.count = self.count
        c.rest_per_channel = self.rest_per_channel
        c.sh_degree = self.sh_degree
        return c


@dataclass
class SplatView:
    """SplatView (SplatRaster.h:25-29): intrinsics (fx, fy, cx, cy), image size
    and a camera-from-world pose, in double precision."""

    K: Tuple[float, float, float, float]
    width: int
    height: int
    R: np.ndarray = field(default_factory=lambda: np.eye(3))
    t: np.ndarray = field(default_factory=lambda: np.zeros(3))

    def camera(self) -> A.Camera:
        cam = A.Camera()
        K = (ct.c_double * 4)(*self.K)
        R = (ct.c_double * 9)(*np.asarray(self.R, dtype=np.float64).reshape(9))
        t = (ct.c_double * 3)(*np.asarray(self.t, dtype=np.float64).reshape(3))
        lib().pxs_camera_from_pose(K, self.width, self.height, R, t, ct.byref(cam))
        return cam


def _camera(view) -> A.Camera:
    return view if isinstance(view, A.Camera) else view.camera()


class Context:
    """A device context: a CUDA stream and a grow-only workspace."""

    def __init__(self, device: int = 0):
        self._lib = lib()
        handle = ct.c_void_p()
        status = self._lib.pxs_context_create(device, ct.byref(handle))
        if status != A.PXS_OK:
            raise PxsError(status, "could not create a context on device %d" % device)
        self.handle = handle

    def check(self, status: int) -> None:
        check(status, lambda: self._lib.pxs_context_last_error(self.handle))

    def set_stream(self, stream_handle: Optional[int]) -> None:
        self.check(self._lib.pxs_context_set_stream(self.handle, stream_handle))

    def synchronize(self) -> None:
        self.check(self._lib.pxs_context_synchronize(self.handle))

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.pxs_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_DEFAULT: Optional[Context] = None


def default_context() -> Context:
    global _DEFAULT
    if _DEFAULT is None:
        _DEFAULT = Context(0)
    return _DEFAULT


def splat_gpu_availability() -> Tuple[bool, str, str]:
    """splatGpuAvailability (VulkanSplatTrainer.h:25): (available, device name, reason)."""
    available = ct.c_int32()
    name = ct.create_string_buffer(256)
    reason = ct.create_string_buffer(512)
    lib().pxs_gpu_availability(ct.byref(available), name, 256, reason, 512)
    return bool(available.value), name.value.decode(), reason.value.decode()


def project_splats(cloud: GaussianCloud, view, options: Optional[A.RasterOptions] = None,
                   ctx: Optional[Context] = None) -> np.ndarray:
    """projectSplats (SplatRaster.h:122-125): visible splats, near to far."""
    ctx = ctx or default_context()
    options = options or A.RasterOptions()
    out = np.zeros(max(cloud.count, 1), dtype=A.PROJECTED_DTYPE)
    count = ct.c_int32()
    c = cloud.c_struct()
    cam = _camera(view)
    ctx.check(lib().pxs_project(ctx.handle, ct.byref(c), ct.byref(cam), ct.byref(options),
                                out.ctypes.data, ct.byref(count)))
    return out[: count.value].copy()


def tile_lists(cloud: GaussianCloud, view, options: Optional[A.RasterOptions] = None,
               ctx: Optional[Context] = None) -> Tuple[np.ndarray, np.ndarray]:
    """The per-tile key lists (gaussian indices near to far) and their offsets."""
    ctx = ctx or default_context()
    options = options or A.RasterOptions()
    cam = _camera(view)
    tiles = ((cam.width + 15) // 16) * ((cam.height + 15) // 16)
    offsets = np.zeros(tiles + 1, dtype=np.int32)
    total = ct.c_int64()
    c = cloud.c_struct()
    status = lib().pxs_tile_lists(ctx.handle, ct.byref(c), ct.byref(cam), ct.byref(options),
                                  offsets.ctypes.data, None, 0, ct.byref(total))
    if status not in (A.PXS_OK, A.PXS_ERR_CAPACITY):
        ctx.check(status)
    entries = np.zeros(max(total.value, 1), dtype=np.int32)
    ctx.check(lib().pxs_tile_lists(ctx.handle, ct.byref(c), ct.byref(cam), ct.byref(options),
                                   offsets.ctypes.data, entries.ctypes.data, total.value,
                                   ct.byref(total)))
    return offsets, entries[: total.value].copy()


def render_splats(cloud: GaussianCloud, view, options: Optional[A.RasterOptions] = None,
                  ctx: Optional[Context] = None) -> Tuple[np.ndarray, np.ndarray]:
    """renderSplats (SplatRaster.h:131-132): (rgb H*W*3, transmittance H*W)."""
    ctx = ctx or default_context()
    options = options or A.RasterOptions()
    cam = _camera(view)
    rgb = np.zeros(cam.width * cam.height * 3, dtype=np.float32)
    T = np.zeros(cam.width * cam.height, dtype=np.float32)
    c = cloud.c_struct()
    ctx.check(lib().pxs_render(ctx.handle, ct.byref(c), ct.byref(cam), ct.byref(options),
                               rgb.ctypes.data, T.ctypes.data))
    return rgb, T


def photometric_loss(rendered: np.ndarray, target: np.ndarray, width: int, height: int,
                     ssim_weight: float, want_gradient: bool = True,
                     ctx: Optional[Context] = None):
    """photometricLoss (SplatRaster.h:153-154): (loss, dL/drgb or None)."""
    ctx = ctx or default_context()
    rendered = np.ascontiguousarray(rendered, dtype=np.float32)
    target = np.ascontiguousarray(target, dtype=np.float32)
    grad = np.zeros_like(rendered) if want_gradient else None
    loss = ct.c_float()
    ctx.check(lib().pxs_photometric_loss(ctx.handle, rendered.ctypes.data, target.ctypes.data,
                                         width, height, ssim_weight,
                                         grad.ctypes.data if want_gradient else None,
                                         ct.byref(loss)))
    return loss.value, grad


def mean_ssim(rendered: np.ndarray, target: np.ndarray, width: int, height: int,
              want_gradient: bool = True, ctx: Optional[Context] = None):
    """meanSsim (SplatRaster.h:158-159): (ssim, d ssim / d rendered or None)."""
    ctx = ctx or default_context()
    rendered = np.ascontiguousarray(rendered, dtype=np.float32)
    target = np.ascontiguousarray(target, dtype=np.float32)
    grad = np.zeros_like(rendered) if want_gradient else None
    value = ct.c_float()
    ctx.check(lib().pxs_mean_ssim(ctx.handle, rendered.ctypes.data, target.ctypes.data, width,
                                  height, grad.ctypes.data if want_gradient else None,
                                  ct.byref(value)))
    return value.value, grad


@dataclass
class SplatGradients:
    """SplatGradients (SplatRaster.h:87-115) in the parameter layout."""

    params: np.ndarray
    screen_gradient: np.ndarray
    visible_count: np.ndarray

    @classmethod
    def zeros(cls, cloud: GaussianCloud) -> "SplatGradients":
        return cls(np.zeros_like(cloud.params), np.zeros(cloud.count, np.float32),
                   np.zeros(cloud.count, np.int32))

    def c_struct(self) -> A.Gradients:
        g = A.Gradients()
        g.params = self.params.ctypes.data
        g.screen_gradient = self.screen_gradient.ctypes.data
        g.visible_count = self.visible_count.ctypes.data
        return g


def rasterize_splats_backward(cloud: GaussianCloud, view, options: Optional[A.RasterOptions],
                              dL_drgb: np.ndarray, gradients: SplatGradients,
                              ctx: Optional[Context] = None) -> SplatGradients:
    """rasterizeSplatsBackward (SplatRaster.h:139-143); adds into `gradients`."""
    ctx = ctx or default_context()
    options = options or A.RasterOptions()
    dL = np.ascontiguousarray(dL_drgb, dtype=np.float32)
    c = cloud.c_struct()
    g = gradients.c_struct()
    cam = _camera(view)
    ctx.check(lib().pxs_backward(ctx.handle, ct.byref(c), ct.byref(cam), ct.byref(options),
                                 dL.ctypes.data, ct.byref(g)))
    return gradients


def render_and_accumulate(cloud: GaussianCloud, view, options: Optional[A.RasterOptions],
                          target: np.ndarray, ssim_weight: float, gradients: SplatGradients,
                          ctx: Optional[Context] = None) -> float:
    """SplatBackend::renderAndAccumulate (SplatTrainer.h:118-122)."""
    ctx = ctx or default_context()
    options = options or A.RasterOptions()
    target = np.ascontiguousarray(target, dtype=np.float32)
    c = cloud.c_struct()
    g = gradients.c_struct()
    cam = _camera(view)
    loss = ct.c_float()
    ctx.check(lib().pxs_render_and_accumulate(ctx.handle, ct.byref(c), ct.byref(cam),
                                              ct.byref(options), target.ctypes.data,
                                              ssim_weight, ct.byref(g), ct.byref(loss)))
    return loss.value


def densify_and_prune(cloud: GaussianCloud, screen_gradient: np.ndarray,
                      visible_count: np.ndarray, config: A.TrainConfig, extent: float,
                      iteration: int, rng_state: int, ctx: Optional[Context] = None):
    """densifyAndPrune (SplatDensify.h:55-57). Returns (new cloud, source_index,
    new rng state, (cloned, split, pruned))."""
    ctx = ctx or default_context()
    P, n = cloud.params.shape
    cap = max(config.max_gaussians, n)
    buf = np.zeros(P * cap + 1, dtype=np.float32)
    buf[: P * n] = cloud.params.reshape(-1)
    source = np.zeros(cap + 1, dtype=np.int32)
    count = ct.c_int32(n)
    state = ct.c_uint32(rng_state)
    cl, sp, pr = ct.c_int32(), ct.c_int32(), ct.c_int32()
    screen = np.ascontiguousarray(screen_gradient, dtype=np.float32)
    visible = np.ascontiguousarray(visible_count, dtype=np.int32)
    ctx.check(lib().pxs_densify_and_prune(ctx.handle, buf.ctypes.data, ct.byref(count),
                                          cloud.rest_per_channel, screen.ctypes.data,
                                          visible.ctypes.data, ct.byref(config), extent,
                                          iteration, ct.byref(state), source.ctypes.data,
                                          ct.byref(cl), ct.byref(sp), ct.byref(pr)))
    m = count.value
    out = GaussianCloud(buf[: P * m].reshape(P, m).copy(), cloud.sh_degree, cloud.rest_per_channel)
    return out, source[:m].copy(), state.value, (cl.value, sp.value, pr.value)


@dataclass
class SplatTrainingProgress:
    iteration: int
    total_iterations: int
    gaussian_count: int
    loss: float
    smoothed_loss: float


def _views_to_c(views: Sequence[Tuple[object, np.ndarray]]):
    cams = (A.Camera * max(len(views), 1))()
    images = []
    for i, (view, image) in enumerate(views):
        cams[i] = _camera(view)
        images.append(np.ascontiguousarray(image, dtype=np.float32))
    ptrs = (ct.c_void_p * max(len(views), 1))(*[im.ctypes.data for im in images])
    return cams, images, ptrs


class SplatTrainer:
    """SplatTrainer (SplatTrainer.h:132-161) with the cloud, its gradients, the
    Adam moments and the training images resident on the GPU.

    `views` is a sequence of (SplatView or Camera, image H*W*3 float32)."""

    def __init__(self, initial: GaussianCloud, views, config: Optional[A.TrainConfig] = None,
                 device: int = 0):
        self._lib = lib()
        self.config = config or A.TrainConfig()
        self.rest = initial.rest_per_channel
        self.P = A.param_count(self.rest)
        cams, self._images, ptrs = _views_to_c(views)
        c = initial.c_struct()
        handle = ct.c_void_p()
        status = self._lib.pxs_trainer_create(ct.byref(self.config), ct.byref(c), cams, ptrs,
                                              len(views), device, ct.byref(handle))
        if status != A.PXS_OK:
            raise PxsError(status, "could not create the trainer")
        self.handle = handle

    @classmethod
    def from_scenes(cls, clouds: Sequence[GaussianCloud], scene_views,
                    config: Optional[A.TrainConfig] = None, device: int = 0) -> "SplatTrainer":
        """A trainer over several independent scenes (pxs_trainer_create_scenes):
        `scene_views[s]` lists scene s's (view, image) pairs; view ids run
        scene after scene. The scenes share one joined cloud, each view renders
        its own scene, and with more than one scene the config must not
        densify."""
        self = cls.__new__(cls)
        self._lib = lib()
        self.config = config or A.TrainConfig()
        self.rest = clouds[0].rest_per_channel
        self.P = A.param_count(self.rest)
        flat = [pair for views in scene_views for pair in views]
        cams, self._images, ptrs = _views_to_c(flat)
        self._clouds = [c.c_struct() for c in clouds]
        arr = (A.Cloud * len(clouds))(*self._clouds)
        counts = (ct.c_int32 * len(clouds))(*[len(v) for v in scene_views])
        handle = ct.c_void_p()
        status = self._lib.pxs_trainer_create_scenes(ct.byref(self.config), arr, len(clouds),
                                                     counts, cams, ptrs, device,
                                                     ct.byref(handle))
        if status != A.PXS_OK:
            raise PxsError(status, "could not create the multi-scene trainer")
        self.handle = handle
        self.scene_counts = [c.count for c in clouds]
        return self

    def _check(self, status: int) -> None:
        check(status, lambda: self._lib.pxs_trainer_last_error(self.handle))

    def step(self) -> bool:
        """One iteration on the next view; False once the schedule is done."""
        stepped = ct.c_int32()
        self._check(self._lib.pxs_trainer_step(self.handle, ct.byref(stepped)))
        return bool(stepped.value)

    def train(self, callback: Optional[Callable[[SplatTrainingProgress], bool]] = None) -> bool:
        """Runs to completion; False when the callback cancelled."""
        completed = ct.c_int32()
        if callback is None:
            fn = A.PROGRESS_FN(0)
        else:
            def trampoline(p, user):
                q = p.contents
                return 1 if callback(SplatTrainingProgress(q.iteration, q.total_iterations,
                                                           q.gaussian_count, q.loss,
                                                           q.smoothed_loss)) else 0
            fn = A.PROGRESS_FN(trampoline)
        self._check(self._lib.pxs_trainer_train(self.handle, fn, None, ct.byref(completed)))
        return bool(completed.value)

    def step_batch(self, n_views: int, view_ids: Optional[Sequence[int]] = None,
                   graph: bool = True) -> float:
        """Batched multi-view step (one pass of each kernel over all views)."""
        ids = None if view_ids is None else (ct.c_int32 * n_views)(*view_ids)
        loss = ct.c_float()
        self._check(self._lib.pxs_trainer_step_batch(self.handle, n_views, ids, int(graph),
                                                     ct.byref(loss)))
        return loss.value

    def accumulate(self, view_ids: Sequence[int], graph: bool = True) -> float:
        """The first half of a data-parallel step: gradients of these views into
        the device buffers, no optimiser step. Returns their mean loss."""
        n = len(view_ids)
        ids = (ct.c_int32 * n)(*view_ids)
        loss = ct.c_float()
        self._check(self._lib.pxs_trainer_accumulate(self.handle, n, ids, int(graph),
                                                     ct.byref(loss)))
        return loss.value

    def apply(self, loss: float = float("nan")) -> None:
        """The second half: the Adam step with the (summed) reduction block. With
        `loss` NaN the mean loss over all ranks' views comes from the block."""
        self._check(self._lib.pxs_trainer_apply(self.handle, ct.c_float(loss)))

    def reduction_block(self):
        """(device pointer, float count) of the one buffer a data-parallel step
        sums over the ranks: gradients, screen gradient, visible counts and the
        loss tail (pxs_trainer_reduction_block)."""
        b, n = ct.c_void_p(), ct.c_int64()
        self._check(self._lib.pxs_trainer_reduction_block(self.handle, ct.byref(b), ct.byref(n)))
        return b.value, n.value

    def gradient_buffers(self):
        """Device pointers of the gradient parts of the reduction block:
        [(pointer, element count, 'float32'), ...] for the parameter gradients,
        the screen gradient and the visible counts (as floats)."""
        g, sg, vc = ct.c_void_p(), ct.c_void_p(), ct.c_void_p()
        n, P = ct.c_int32(), ct.c_int32()
        self._check(self._lib.pxs_trainer_gradients(self.handle, ct.byref(g), ct.byref(sg),
                                                    ct.byref(vc), ct.byref(n), ct.byref(P)))
        return [(g.value, P.value * n.value, "float32"), (sg.value, n.value, "float32"),
                (vc.value, n.value, "float32")]

    def ingest_images(self, view_ids: Sequence[int], frames: Sequence[np.ndarray],
                      sizes: Sequence[Tuple[int, int]]) -> None:
        """Replaces the resident images of `view_ids` from 8-bit RGB frames of
        the given (width, height), downscaled on the device to each view's size."""
        n = len(view_ids)
        keep = [np.ascontiguousarray(f, dtype=np.uint8) for f in frames]
        ids = (ct.c_int32 * max(n, 1))(*view_ids)
        ptrs = (ct.c_void_p * max(n, 1))(*[f.ctypes.data for f in keep])
        ws = (ct.c_int32 * max(n, 1))(*[s[0] for s in sizes])
        hs = (ct.c_int32 * max(n, 1))(*[s[1] for s in sizes])
        self._check(self._lib.pxs_trainer_ingest_images(self.handle, n, ids, ptrs, ws, hs))

    def stage_images(self, view_ids: Sequence[int], frames: Sequence[np.ndarray],
                     sizes: Sequence[Tuple[int, int]]) -> None:
        """ingest_images without waiting: the frames are copied to the device
        while the current step runs and take effect at the next step (or the
        next ingest / set_images / stage call). The frames are kept referenced
        here until then; they must not be modified before that call returns."""
        n = len(view_ids)
        keep = [f if isinstance(f, np.ndarray) and f.dtype == np.uint8 and f.flags.c_contiguous
                else np.ascontiguousarray(f, dtype=np.uint8) for f in frames]
        ids = (ct.c_int32 * max(n, 1))(*view_ids)
        ptrs = (ct.c_void_p * max(n, 1))(*[f.ctypes.data for f in keep])
        ws = (ct.c_int32 * max(n, 1))(*[s[0] for s in sizes])
        hs = (ct.c_int32 * max(n, 1))(*[s[1] for s in sizes])
        self._check(self._lib.pxs_trainer_stage_images(self.handle, n, ids, ptrs, ws, hs))
        # held until a later stage call: the copy may still be reading them
        self._staged = getattr(self, "_staged", [])[-1:] + [keep]

    def export(self, fmt: str = "ply", fractional_bits: int = 12) -> bytes:
        """The trained cloud as the bytes of a .ply, .splat or .spz file."""
        status, data = _export(lambda out, cap, size: self._lib.pxs_trainer_export(
            self.handle, FORMATS[fmt], fractional_bits, out, cap, size), fmt)
        self._check(status)
        return data

    def stream(self) -> int:
        """The trainer's CUDA stream (a cudaStream_t as an integer)."""
        sp = ct.c_void_p()
        self._check(self._lib.pxs_trainer_stream(self.handle, ct.byref(sp)))
        return sp.value or 0

    def step_views(self, n_views: int, view_ids: Optional[Sequence[int]] = None) -> float:
        """Plain multi-view step (per-view kernel sequences, host-synchronised)."""
        ids = None if view_ids is None else (ct.c_int32 * n_views)(*view_ids)
        loss = ct.c_float()
        self._check(self._lib.pxs_trainer_step_views(self.handle, n_views, ids, ct.byref(loss)))
        return loss.value

    def state(self) -> dict:
        it, cnt, sh = ct.c_int32(), ct.c_int32(), ct.c_int32()
        ll, sm, ex = ct.c_float(), ct.c_float(), ct.c_float()
        self._check(self._lib.pxs_trainer_state(self.handle, ct.byref(it), ct.byref(cnt),
                                                ct.byref(ll), ct.byref(sm), ct.byref(ex),
                                                ct.byref(sh)))
        return dict(iteration=it.value, count=cnt.value, last_loss=ll.value,
                    smoothed_loss=sm.value, extent=ex.value, sh_degree=sh.value)

    @property
    def iteration(self) -> int:
        return self.state()["iteration"]

    def sh_degree_in_use(self) -> int:
        return self.state()["sh_degree"]

    def last_loss(self) -> float:
        return self.state()["last_loss"]

    def smoothed_loss(self) -> float:
        return self.state()["smoothed_loss"]

    def scene_extent(self) -> float:
        return self.state()["extent"]

    def cloud_params(self) -> np.ndarray:
        n = self.state()["count"]
        buf = np.zeros(self.P * max(n, 1), dtype=np.float32)
        count = ct.c_int32()
        self._check(self._lib.pxs_trainer_download(self.handle, buf.ctypes.data, n,
                                                   ct.byref(count)))
        return buf[: self.P * count.value].reshape(self.P, count.value).copy()

    def finish(self) -> GaussianCloud:
        """Prune, sort by opacity and hand the cloud over (SplatTrainer.cpp:378-383)."""
        n = self.state()["count"]
        buf = np.zeros(self.P * max(n, 1), dtype=np.float32)
        count = ct.c_int32()
        self._check(self._lib.pxs_trainer_finish(self.handle, buf.ctypes.data, n,
                                                 ct.byref(count)))
        m = count.value
        return GaussianCloud(buf[: self.P * m].reshape(self.P, m).copy(), self.config.sh_degree,
                             self.rest)

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.pxs_trainer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


FORMATS = {"ply": A.PXS_FORMAT_PLY, "splat": A.PXS_FORMAT_SPLAT, "spz": A.PXS_FORMAT_SPZ}


def _export(call, fmt: str) -> bytes:
    size = ct.c_size_t()
    status = call(None, 0, ct.byref(size))
    if status not in (A.PXS_OK, A.PXS_ERR_CAPACITY):
        return status, b""
    buf = (ct.c_uint8 * max(size.value, 1))()
    status = call(buf, size.value, ct.byref(size))
    return status, bytes(buf[: size.value])


def export_cloud(cloud: GaussianCloud, fmt: str = "ply", fractional_bits: int = 12,
                 ctx: Optional[Context] = None) -> bytes:
    """The bytes writeGaussianPly / writeSplat / writeSpz (GaussianCloud.h:95-131)
    would write for `cloud`, packed on the device: fmt is "ply", "splat" or "spz"."""
    ctx = ctx or default_context()
    c = cloud.c_struct()
    status, data = _export(lambda out, cap, size: lib().pxs_export_cloud(
        ctx.handle, ct.byref(c), FORMATS[fmt], fractional_bits, out, cap, size), fmt)
    ctx.check(status)
    return data


def initialize_from_points(points: np.ndarray, colors: Optional[np.ndarray] = None,
                           sh_degree: int = 0, initial_opacity: float = 0.1,
                           ctx: Optional[Context] = None) -> GaussianCloud:
    """initializeFromPointCloud (GaussianCloud.cpp:199-257) with the spacing
    search on the device. points: (n, 3) float32; colors: (n, 3) uint8 or None."""
    ctx = ctx or default_context()
    pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
    n = pts.shape[0]
    cols = None if colors is None else np.ascontiguousarray(colors, dtype=np.uint8).reshape(-1, 3)
    rest = ct.c_int32()
    ctx.check(lib().pxs_initialize_from_points(ctx.handle, None, None, n, sh_degree,
                                               ct.c_float(initial_opacity), None, ct.byref(rest)))
    out = np.zeros((A.param_count(rest.value), n), dtype=np.float32)
    ctx.check(lib().pxs_initialize_from_points(
        ctx.handle, pts.ctypes.data if n else None, None if cols is None else cols.ctypes.data,
        n, sh_degree, ct.c_float(initial_opacity), out.ctypes.data if n else None,
        ct.byref(rest)))
    return GaussianCloud(out, max(0, min(3, sh_degree)), rest.value)


def downscale_to_width(rgb: np.ndarray, width: int, height: int, target_width: int,
                       ctx: Optional[Context] = None):
    """downscaleToWidth (ImageIo.cpp:300-337) on the device: (bytes H*W*3 uint8,
    floats H*W*3 = bytes / 255, out_width, out_height)."""
    ctx = ctx or default_context()
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    w, h = ct.c_int32(), ct.c_int32()
    ctx.check(lib().pxs_downscale_to_width(ctx.handle, None, width, height, target_width, None,
                                           None, ct.byref(w), ct.byref(h)))
    out = np.zeros(w.value * h.value * 3, dtype=np.uint8)
    lin = np.zeros(w.value * h.value * 3, dtype=np.float32)
    ctx.check(lib().pxs_downscale_to_width(ctx.handle, rgb.ctypes.data, width, height,
                                           target_width, out.ctypes.data, lin.ctypes.data,
                                           ct.byref(w), ct.byref(h)))
    return out, lin, w.value, h.value


def train_splats_on_gpu(cloud: GaussianCloud, views, config: A.TrainConfig,
                        callback: Optional[Callable[[SplatTrainingProgress], bool]] = None):
    """trainSplatsOnGpu (VulkanSplatTrainer.h:35-37): returns (ok, error, cloud)."""
    P, n = cloud.params.shape
    cap = max(config.max_gaussians, n)
    buf = np.zeros(P * cap + 1, dtype=np.float32)
    buf[: P * n] = cloud.params.reshape(-1)
    c = A.Cloud()
    c.params = buf.ctypes.data
    c.count = n
    c.rest_per_channel = cloud.rest_per_channel
    c.sh_degree = cloud.sh_degree
    cams, images, ptrs = _views_to_c(views)
    if callback is None:
        fn = A.PROGRESS_FN(0)
    else:
        def trampoline(p, user):
            q = p.contents
            return 1 if callback(SplatTrainingProgress(q.iteration, q.total_iterations,
                                                       q.gaussian_count, q.loss,
                                                       q.smoothed_loss)) else 0
        fn = A.PROGRESS_FN(trampoline)
    error = ct.create_string_buffer(512)
    status = lib().pxs_train_splats(ct.byref(c), cams, ptrs, len(views), ct.byref(config), fn,
                                    None, error, 512)
    if status != A.PXS_OK:
        return False, error.value.decode(), cloud
    m = c.count
    return True, "", GaussianCloud(buf[: P * m].reshape(P, m).copy(), c.sh_degree,
                                   cloud.rest_per_channel)


def synthetic_cloud(seed: int, count: int, sh_degree: int, log_scale_mean: float = -4.0):
    """A seeded cloud with the benchmark distributions (pxs_synthetic_cloud)."""
    rest = A.rest_per_channel(sh_degree)
    params = np.zeros((A.param_count(rest), count), dtype=np.float32)
    status = lib().pxs_synthetic_cloud(seed, count, rest, log_scale_mean, params.ctypes.data)
    if status != A.PXS_OK:
        raise PxsError(status, "pxs_synthetic_cloud failed")
    return GaussianCloud(params, sh_degree, rest)


def synthetic_cameras(seed: int, count: int, width: int, height: int, layout: int = 0,
                      radius: float = 3.0, fov_degrees: float = 60.0) -> List[A.Camera]:
    """Seeded camera rigs looking at the origin (pxs_synthetic_cameras)."""
    cams = (A.Camera * max(count, 1))()
    status = lib().pxs_synthetic_cameras(seed, count, layout, radius, width, height,
                                         fov_degrees, cams)
    if status != A.PXS_OK:
        raise PxsError(status, "pxs_synthetic_cameras failed")
    return [cams[i] for i in range(count)]

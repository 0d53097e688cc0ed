#!/usr/bin/env python
"""Gaussian-splat training step benchmark on B200.

Workload (default "c4"): 1M gaussians, SH degree 3, a 64-camera pool at
1920x1440 (Fibonacci sphere, radius 3, 60 degree FOV), 8 views per step
rendered, differentiated and accumulated, then one Adam step. Synthetic data:
truth cloud seed 1 (targets rendered from it), start cloud seed 2, cameras
seed 3; inputs are larger than L2 (1M gaussians x 236 B of parameters, 8 x 33 MB
of targets per step), so no L2 flush is needed between steps.

Arms:
  ours (default)  the batched, CUDA-graph-captured step; also the plain
                  per-view form, the end-to-end step through the C ABI with the
                  step's 8-bit target frames copied from pinned host memory and
                  converted on the device (and, beside it, FP32 images), per-stage
                  device timing, the roofline of the dominant kernel and, on
                  rank 0 at N=1, the reference CPU trainer's rate on a bounded
                  sample.
  reference       the reference's own CPU implementation (compiled from its
                  sources into oracle/_ref with its release flags) on a bounded
                  sample of the same workload, one view per host thread.

Multi-GPU (torchrun): data parallel over views; each rank renders and
differentiates its own 8 views per step (weak scaling), the gradients are summed
with an NCCL all-reduce, every rank applies the same Adam step.
"""
from __future__ import annotations

import argparse
import ctypes as ct
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STAGES = ["project", "bin", "forward", "loss", "backward", "param_grads", "adam"]
METRIC = "train steps/s (fwd+bwd+Adam, 8 views of 1920x1440, 1M gaussians SH3), batched graph-captured step"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", default="c4")
    p.add_argument("--views", type=int, default=0,
                   help="views per step (default: the workload's); a smaller case for profiling")
    p.add_argument("--pool", type=int, default=0,
                   help="use only the first N cameras of the pool (smaller device footprint, "
                        "for profiler captures); 0 = the workload's pool")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--px", default="",
                   help="pixels per thread 'F,B' for compositing and its adjoint "
                        "(default: the autotuner picks)")
    return p.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ------------------------------------------------------------- clocks


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.file,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


# ------------------------------------------------- reference CPU sample

CROPS = [(0, 0), (1, 1), (2, 2), (3, 3), (0, 2), (1, 3), (2, 0), (3, 1)]


def load_cpu_baseline():
    """The reference compiled from its sources with its own release flags, or
    the C restatement when that build is absent. Returns (kind, lib)."""
    ref = os.path.join(ROOT, "oracle", "_ref", "libpxref_fast.so")
    if os.path.exists(ref):
        lib = ct.CDLL(ref)
        view = [_vp, ct.c_int, ct.c_int, ct.c_int, _vp, ct.c_int, ct.c_int, _vp, _vp, _vp]
        _sig(lib.ref_project, ct.c_int, view + [_vp])
        _sig(lib.ref_render, None, view + [_vp, _vp])
        _sig(lib.ref_render_and_accumulate, ct.c_float,
             view + [_vp, ct.c_float, _vp, _vp, _vp])
        return "reference", lib
    port = os.path.join(ROOT, "oracle", "libpxo.so")
    if not os.path.exists(port):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    lib = ct.CDLL(port)
    i32 = ct.c_int32
    _sig(lib.pxo_project_f32, i32, [_vp, i32, i32, i32, _vp, _vp, _vp])
    _sig(lib.pxo_rasterize_f32, None, [_vp, i32, _vp, _vp, _vp, _vp])
    _sig(lib.pxo_render_and_accumulate_f32, ct.c_float,
         [_vp, i32, i32, i32, _vp, _vp, _vp, ct.c_float, _vp, _vp, _vp])
    return "port", lib


_vp = ct.c_void_p


def _sig(fn, restype, argtypes):
    fn.restype = restype
    fn.argtypes = argtypes


class CpuSample:
    """One view per host thread: the reference's projectSplats over the full
    view, then renderAndAccumulate (project, rasterise, L1+SSIM, backward) on a
    1/16 window of it. A full view's cost is estimated as
    t(project full) + 16 * (t(renderAndAccumulate window) - t(project window)):
    compositing, loss and backward scale with pixels, projection does not."""

    def __init__(self, truth, start, views, kind, lib, threads):
        from parallax_b200.scenes import crop_view

        self.kind, self.lib = kind, lib
        self.start = start
        self.views = views[:8]
        self.threads = threads
        self.jobs = []
        w, h = self.views[0].width // 4, self.views[0].height // 4
        for i, view in enumerate(self.views):
            cx, cy = CROPS[i % len(CROPS)]
            crop = crop_view(view, cx * w, cy * h, w, h)
            target = self.render(truth, crop)  # the reference renders its own targets
            self.jobs.append((view, crop, target))

    def _view_args(self, v):
        K = np.array(v.K, dtype=np.float64)
        R = np.ascontiguousarray(np.asarray(v.R, dtype=np.float64).reshape(9))
        t = np.ascontiguousarray(np.asarray(v.t, dtype=np.float64).reshape(3))
        return (K, R, t)

    def render(self, cloud, view):
        rgb = np.zeros(view.width * view.height * 3, dtype=np.float32)
        if self.kind == "reference":
            K, R, t = self._view_args(view)
            self.lib.ref_render(cloud.params.ctypes.data, cloud.count, cloud.rest_per_channel,
                                cloud.sh_degree, K.ctypes.data, view.width, view.height,
                                R.ctypes.data, t.ctypes.data, ct.byref(self.options()),
                                rgb.ctypes.data, None)
        else:
            cam = view.camera()
            proj = np.zeros(cloud.count * 64 + 64, dtype=np.uint8)
            n = self.lib.pxo_project_f32(cloud.params.ctypes.data, cloud.count,
                                         cloud.rest_per_channel, cloud.sh_degree, ct.byref(cam),
                                         ct.byref(self.options()), proj.ctypes.data)
            self.lib.pxo_rasterize_f32(proj.ctypes.data, n, ct.byref(cam),
                                       ct.byref(self.options()), rgb.ctypes.data, None)
        return rgb

    def options(self):
        from parallax_b200 import RasterOptions
        return RasterOptions(sh_degree=3)

    def project(self, view):
        c = self.start
        out = np.zeros(c.count * 64 + 64, dtype=np.uint8)
        if self.kind == "reference":
            K, R, t = self._view_args(view)
            self.lib.ref_project(c.params.ctypes.data, c.count, c.rest_per_channel, c.sh_degree,
                                 K.ctypes.data, view.width, view.height, R.ctypes.data,
                                 t.ctypes.data, ct.byref(self.options()), out.ctypes.data)
        else:
            cam = view.camera()
            self.lib.pxo_project_f32(c.params.ctypes.data, c.count, c.rest_per_channel,
                                     c.sh_degree, ct.byref(cam), ct.byref(self.options()),
                                     out.ctypes.data)

    def render_and_accumulate(self, view, target):
        c = self.start
        grads = np.zeros_like(c.params)
        screen = np.zeros(c.count, dtype=np.float32)
        visible = np.zeros(c.count, dtype=np.int32)
        if self.kind == "reference":
            K, R, t = self._view_args(view)
            self.lib.ref_render_and_accumulate(
                c.params.ctypes.data, c.count, c.rest_per_channel, c.sh_degree, K.ctypes.data,
                view.width, view.height, R.ctypes.data, t.ctypes.data, ct.byref(self.options()),
                target.ctypes.data, ct.c_float(0.2), grads.ctypes.data, screen.ctypes.data,
                visible.ctypes.data)
        else:
            cam = view.camera()
            self.lib.pxo_render_and_accumulate_f32(
                c.params.ctypes.data, c.count, c.rest_per_channel, c.sh_degree, ct.byref(cam),
                ct.byref(self.options()), target.ctypes.data, ct.c_float(0.2),
                grads.ctypes.data, screen.ctypes.data, visible.ctypes.data)

    def run(self):
        """Estimated seconds for one full step (8 views) on `threads` threads."""
        estimates = [0.0] * len(self.jobs)

        def work(i):
            view, crop, target = self.jobs[i]
            t0 = time.perf_counter()
            self.project(view)
            t1 = time.perf_counter()
            self.project(crop)
            t2 = time.perf_counter()
            self.render_and_accumulate(crop, target)
            t3 = time.perf_counter()
            estimates[i] = (t1 - t0) + 16.0 * max(0.0, (t3 - t2) - (t2 - t1))

        pending = list(range(len(self.jobs)))
        while pending:
            batch, pending = pending[: self.threads], pending[self.threads:]
            ts = [threading.Thread(target=work, args=(i,)) for i in batch]
            for t in ts:
                t.start()
            for t in ts:
                t.join()
        return sum(estimates) / min(self.threads, len(self.jobs))

    def describe(self):
        v = self.views[0]
        return (f"{len(self.jobs)} views, one per thread: the reference's projectSplats over the "
                f"full {v.width}x{v.height} view plus renderAndAccumulate on a "
                f"{v.width // 4}x{v.height // 4} window (1/16 of the pixels); a view costs "
                f"t(project) + 16 x t(window fwd+loss+bwd); step = sum over 8 views / threads; "
                f"1M gaussians SH3, {self.kind} build")


# ------------------------------------------------------------ our arm


def stage_work(w, P, N, V, K, E, Q, pixels):
    """Algorithmic work per stage: (bytes, flops)."""
    return {
        "project": (N * (4 * P + 52 * V), 0),
        "bin": (K * 24, 0),
        "forward": (0, 17 * E + 10 * Q),
        "loss": (0, 480 * 3 * pixels),
        "backward": (0, 17 * E + 58 * Q),
        "param_grads": (N * (4 * P * 2 + 92 * V), 0),
        "adam": (28 * N * P, 0),
    }


def run_ours(args):
    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import parallax_b200 as px
    from parallax_b200.scenes import WORKLOADS, workload_scene

    w = WORKLOADS[args.workload]
    V = args.views or w["views_per_step"]
    truth, start, views = workload_scene(args.workload)
    if args.pool > 0:
        views = views[:args.pool]
    P = px.param_count(start.rest_per_channel)
    N = start.count

    # targets: the truth cloud rendered on the device, kept in pinned host memory
    opts = px.RasterOptions(sh_degree=w["sh_degree"])
    lib = px.lib()
    renderer = px.SplatTrainer(truth, [], px.TrainConfig(iterations=1))
    pinned = []
    for view in views:
        buf = torch.empty(view.width * view.height * 3, dtype=torch.float32, pin_memory=True)
        arr = buf.numpy()
        cam = view.camera()
        renderer._check(lib.pxs_trainer_render(renderer.handle, ct.byref(cam), ct.byref(opts),
                                               arr.ctypes.data, None))
        pinned.append((buf, arr))
    renderer.close()
    del renderer
    # the same targets as 8-bit frames, the reference's image format before
    # downscaleToWidth; the trainer trains on frame / 255 (ingested on the device)
    frames = []
    for _, arr in pinned:
        fbuf = torch.empty(arr.size, dtype=torch.uint8, pin_memory=True)
        fbuf.numpy()[:] = np.rint(np.clip(arr, 0.0, 1.0) * 255.0).astype(np.uint8)
        frames.append(fbuf)

    cfg = px.TrainConfig(iterations=100000, sh_degree=w["sh_degree"], sh_increase_interval=0,
                         densify_from_iteration=10 ** 9, densify_until_iteration=10 ** 9,
                         opacity_reset_interval=0, max_gaussians=max(600000, N))
    trainer = px.SplatTrainer(start, [(v.camera(), arr) for v, (_, arr) in zip(views, pinned)],
                              cfg, device=local)
    def ingest(ids):
        id_arr = (ct.c_int32 * len(ids))(*ids)
        ptrs = (ct.c_void_p * len(ids))(*[frames[i].data_ptr() for i in ids])
        ws = (ct.c_int32 * len(ids))(*[views[i].width for i in ids])
        hs = (ct.c_int32 * len(ids))(*[views[i].height for i in ids])
        trainer._check(lib.pxs_trainer_ingest_images(trainer.handle, len(ids), id_arr, ptrs,
                                                     ws, hs))

    ingest(list(range(len(views))))
    sp = ct.c_void_p()
    trainer._check(lib.pxs_trainer_stream(trainer.handle, ct.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value)
    pool = len(views)

    def ids_for(step):
        base = (step * V + rank * 7) % pool
        return [(base + i) % pool for i in range(V)]

    if world > 1:
        # data parallel over views: each rank renders its own V views, the
        # gradient buffers are summed over the ranks, every rank takes the
        # same Adam step
        from parallax_b200.data_parallel import DataParallelStep
        dp_step = DataParallelStep(trainer, device="cuda")

        def batch_step(step, graph=True):
            return dp_step(ids_for(step))
    else:
        def batch_step(step, graph=True):
            return trainer.step_batch(V, ids_for(step), graph=graph)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def timed(fn, steps):
        barrier()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for s in range(steps):
            fn(s)
        b.record(stream)
        b.synchronize()
        torch.cuda.synchronize()
        barrier()
        ms = a.elapsed_time(b) / steps
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    step_counter = [0]

    def next_batch(_):
        step_counter[0] += 1
        batch_step(step_counter[0])

    # the autotuner picks pixels per thread for compositing and its adjoint
    fpx, bpx = ct.c_int32(), ct.c_int32()
    if args.px:
        f_, b_ = (int(x) for x in args.px.split(","))
        trainer._check(lib.pxs_set_raster_config(f_, b_))
        lib.pxs_get_raster_config(ct.byref(fpx), ct.byref(bpx))
    else:
        ids0 = (ct.c_int32 * V)(*ids_for(0))
        trainer._check(lib.pxs_trainer_autotune(trainer.handle, V, ids0, ct.byref(fpx),
                                                ct.byref(bpx)))

    # warm-up: capture the graph, then once more with stage timing on
    for _ in range(max(args.warmup, 3)):
        next_batch(0)
    trainer._check(lib.pxs_trainer_set_timing(trainer.handle, 1))
    next_batch(0)
    trainer._check(lib.pxs_trainer_set_timing(trainer.handle, 1))  # reset the totals

    clocks = ClockSampler(local)
    clocks.start()
    ms_batched = timed(next_batch, args.steps)
    clock_info = clocks.stop()

    stage_ms = (ct.c_float * len(STAGES))()
    n_stages, n_steps = ct.c_int32(), ct.c_int32()
    trainer._check(lib.pxs_trainer_stage_times(trainer.handle, stage_ms, len(STAGES),
                                               ct.byref(n_stages), ct.byref(n_steps)))
    per_stage = {s: stage_ms[i] / max(n_steps.value, 1) for i, s in enumerate(STAGES)}
    pairs, launches = ct.c_int64(), ct.c_int64()
    trainer._check(lib.pxs_trainer_step_info(trainer.handle, ct.byref(pairs), ct.byref(launches)))
    kernels_per_step = launches.value
    evaluated, contributing = ct.c_int64(), ct.c_int64()
    trainer._check(lib.pxs_trainer_pair_stats(trainer.handle, ct.byref(evaluated),
                                              ct.byref(contributing)))
    trainer._check(lib.pxs_trainer_set_timing(trainer.handle, 0))
    next_batch(0)  # re-capture without the timing events

    result = {}
    ms_plain = None
    if not args.no_plain and world == 1:
        def plain_step(_):
            step_counter[0] += 1
            trainer.step_views(V, ids_for(step_counter[0]))
        plain_step(0)
        ms_plain = timed(plain_step, max(3, args.steps // 2))

    e2e = None
    if not args.no_e2e:
        # each step's 8-bit frames cross from pinned host memory and are
        # converted on the device (pxs_trainer_ingest_images), then the step
        # runs and its loss is read back
        def e2e_step(_):
            step_counter[0] += 1
            ingest(ids_for(step_counter[0]))
            batch_step(step_counter[0])  # reads the loss back to the host

        # the same with the targets uploaded as FP32 images (pxs_trainer_set_images)
        def e2e_float_step(_):
            step_counter[0] += 1
            ids = ids_for(step_counter[0])
            id_arr = (ct.c_int32 * V)(*ids)
            ptrs = (ct.c_void_p * V)(*[pinned[i][1].ctypes.data for i in ids])
            trainer._check(lib.pxs_trainer_set_images(trainer.handle, V, id_arr, ptrs))
            batch_step(step_counter[0])

        e2e_step(0)
        ms_e2e = timed(e2e_step, args.steps)
        h2d = sum(views[i].width * views[i].height * 3 for i in ids_for(0))
        e2e_float_step(0)
        ms_e2e_float = timed(e2e_float_step, args.steps)
        # restore the 8-bit targets of the views the float leg replaced
        ingest(list(range(len(views))))
        e2e = {"value": world * 1000.0 / ms_e2e, "unit": "steps/s", "ms_per_step": ms_e2e,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 4 + 4,
               "inputs": "8-bit RGB frames at the view size, converted on the device",
               "fp32_targets": {"value": world * 1000.0 / ms_e2e_float,
                                "ms_per_step": ms_e2e_float, "h2d_bytes_per_step": 4 * h2d,
                                "inputs": "FP32 RGB images (pxs_trainer_set_images)"}}

    # roofline of the dominant kernel and of the whole step
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    hbm_source = "measured" if "hbm_gbs" in peaks else "fallback"
    fp32 = ct.c_float()
    if lib.pxs_measure_fp32_peak(local, ct.byref(fp32)) != 0:
        fp32.value = 74.0
    pixels = sum(views[i].width * views[i].height for i in ids_for(0))
    work = stage_work(w, P, N, V, pairs.value, evaluated.value, contributing.value, pixels)
    dominant = max(per_stage, key=per_stage.get)
    bytes_, flops = work[dominant]
    dom_ms = per_stage[dominant]
    if flops > 0:
        achieved = flops / (dom_ms * 1e-3) / 1e12
        roofline = {"kernel": dominant, "bound": "fp32", "achieved": achieved,
                    "peak": fp32.value, "unit": "TFLOP/s", "frac": achieved / fp32.value,
                    "peak_source": "measured FP32 FMA microkernel (pxs_measure_fp32_peak)"}
    else:
        achieved = bytes_ / (dom_ms * 1e-3) / 1e9
        roofline = {"kernel": dominant, "bound": "hbm", "achieved": achieved, "peak": hbm,
                    "unit": "GB/s", "frac": achieved / hbm,
                    "peak_source": f"{hbm_source} MEASURED_PEAKS.json hbm_gbs"}
    roofline["traffic"] = traffic_from_profiles(dominant)
    roofline["launch_ms"] = dom_ms
    t_roof = 0.0
    for s, (b_, f_) in work.items():
        t_roof += max(b_ / (hbm * 1e9), f_ / (fp32.value * 1e12))
    step_roofline = {"t_roofline_ms": t_roof * 1e3, "t_measured_ms": ms_batched,
                     "frac": t_roof * 1e3 / ms_batched}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            kind, clib = load_cpu_baseline()
            threads = min(8, os.cpu_count() or 1)
            sample = CpuSample(truth, start, views, kind, clib, threads)
            seconds = sample.run()
            cpu = {"value": 1.0 / seconds, "unit": "steps/s", "cores": threads, "kind": kind,
                   "sample": sample.describe(), "seconds_per_step_estimate": seconds,
                   "host_cores": os.cpu_count()}
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "steps/s", "cores": 0, "kind": "unavailable",
                   "sample": f"failed: {exc}"}

    line = {
        "metric": METRIC,
        "value": world * 1000.0 / ms_batched,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_batched,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": "synthetic (seeded: truth cloud 1, start cloud 2, cameras 3; targets rendered "
                "from the truth cloud, quantised to 8-bit frames)",
        "config": {"workload": f"{args.workload}: {N} gaussians SH{w['sh_degree']}, "
                               f"{V} views/step at {w['width']}x{w['height']} from a {pool}-camera "
                               "pool, fwd+L1/SSIM+bwd+Adam",
                   "gaussians": N, "views_per_step": V, "width": w["width"],
                   "height": w["height"], "parallelism": f"dp{world} over views",
                   "l2": "inputs larger than L2 (no flush)",
                   "pixels_per_thread": {"forward": fpx.value, "backward": bpx.value}},
        "plain": {"ms_per_step": ms_plain,
                  "value": world * 1000.0 / ms_plain if ms_plain else None,
                  "batched_over_plain": (ms_plain / ms_batched) if ms_plain else None,
                  "form": "per-view kernel sequences, host-synchronised pair counts, no graph"},
        "e2e": e2e,
        "gpu_launches": kernels_per_step * args.steps,
        "kernels_per_step": kernels_per_step,
        "stage_ms": per_stage,
        "pairs_per_step": pairs.value,
        "evaluated_pairs": evaluated.value,
        "contributing_pairs": contributing.value,
        "roofline": roofline,
        "step_roofline": step_roofline,
        "cpu_baseline": cpu,
        "clocks": clock_info,
    }
    trainer.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def run_multi_scene(args):
    """The uneven batch of independent scans: 32 scenes (5k-150k gaussians SH3,
    320x240 / 640x480 / 1280x720), 4 views each; one step renders and
    differentiates all 128 views in one pass of each kernel and takes every
    scene's Adam step (a multi-scene trainer, pxs_trainer_create_scenes)."""
    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    import parallax_b200 as px
    from parallax_b200.scenes import MULTI_SCENE, multi_scene_workload

    scenes = multi_scene_workload(5)
    lib = px.lib()
    opts = px.RasterOptions(sh_degree=MULTI_SCENE["sh_degree"])
    scene_views, starts = [], []
    for truth, start, views in scenes:
        renderer = px.SplatTrainer(truth, [], px.TrainConfig(iterations=1))
        pairs = []
        for view in views:
            arr = np.empty(view.width * view.height * 3, dtype=np.float32)
            cam = view.camera()
            renderer._check(lib.pxs_trainer_render(renderer.handle, ct.byref(cam),
                                                   ct.byref(opts), arr.ctypes.data, None))
            pairs.append((cam, arr))
        renderer.close()
        scene_views.append(pairs)
        starts.append(start)
    cfg = px.TrainConfig(iterations=100000, sh_degree=MULTI_SCENE["sh_degree"],
                         sh_increase_interval=0, densify_from_iteration=10 ** 9,
                         densify_until_iteration=10 ** 9, opacity_reset_interval=0)
    trainer = px.SplatTrainer.from_scenes(starts, scene_views, cfg, device=local)
    n_views = sum(len(v) for v in scene_views)
    ids = list(range(n_views))
    sp = ct.c_void_p()
    trainer._check(lib.pxs_trainer_stream(trainer.handle, ct.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value)
    fpx, bpx = ct.c_int32(), ct.c_int32()
    id_arr = (ct.c_int32 * n_views)(*ids)
    trainer._check(lib.pxs_trainer_autotune(trainer.handle, n_views, id_arr, ct.byref(fpx),
                                            ct.byref(bpx)))
    for _ in range(max(args.warmup, 3)):
        trainer.step_batch(n_views, ids)
    trainer._check(lib.pxs_trainer_set_timing(trainer.handle, 1))
    trainer.step_batch(n_views, ids)
    trainer._check(lib.pxs_trainer_set_timing(trainer.handle, 1))
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.steps):
        trainer.step_batch(n_views, ids)
    b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b) / args.steps
    stage_ms = (ct.c_float * len(STAGES))()
    n_stages, n_steps = ct.c_int32(), ct.c_int32()
    trainer._check(lib.pxs_trainer_stage_times(trainer.handle, stage_ms, len(STAGES),
                                               ct.byref(n_stages), ct.byref(n_steps)))
    pairs, launches = ct.c_int64(), ct.c_int64()
    trainer._check(lib.pxs_trainer_step_info(trainer.handle, ct.byref(pairs), ct.byref(launches)))
    counts = [c.count for c in starts]
    line = {
        "metric": "train steps/s (fwd+bwd+Adam), 32 independent scenes x 4 views in one "
                  "batched graph-captured step",
        "value": 1000.0 / ms, "unit": "steps/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic (seeded: scene s truth cloud 1000+2s, start 1001+2s, cameras 3000+s)",
        "config": {"workload": f"c5: {len(starts)} scenes, {sum(counts)} gaussians "
                               f"({min(counts)}..{max(counts)}) SH{MULTI_SCENE['sh_degree']}, "
                               f"{n_views} views of 320x240 / 640x480 / 1280x720",
                   "pixels_per_thread": {"forward": fpx.value, "backward": bpx.value}},
        "gpu_launches": launches.value * args.steps, "kernels_per_step": launches.value,
        "pairs_per_step": pairs.value,
        "stage_ms": {s: stage_ms[i] / max(n_steps.value, 1) for i, s in enumerate(STAGES)},
    }
    trainer.close()
    print(json.dumps(line))


def traffic_from_profiles(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    try:
        return json.load(open(path)).get(kernel)
    except (OSError, ValueError):
        return None


# ------------------------------------------------------- reference arm


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    import parallax_b200 as px  # host-side scene generation only
    from parallax_b200.scenes import WORKLOADS, orbit_views

    w = WORKLOADS[args.workload]
    try:
        kind, clib = load_cpu_baseline()
    except Exception as exc:
        print(json.dumps({"impl": "reference", "unavailable": f"no CPU build: {exc}"}))
        return
    truth = px.synthetic_cloud(1, w["gaussians"], w["sh_degree"])
    start = px.synthetic_cloud(2, w["gaussians"], w["sh_degree"])
    views = orbit_views(3, w["pool"], w["width"], w["height"], layout=w["layout"])
    threads = min(8, os.cpu_count() or 1)
    sample = CpuSample(truth, start, views, kind, clib, threads)
    for _ in range(args.warmup):
        sample.run()
    times = [sample.run() for _ in range(args.steps)]
    seconds = statistics.median(times)
    value = 1.0 / seconds
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": seconds * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": "synthetic (seeded, same scene as ours; targets rendered by the reference)",
        "config": {"workload": f"{args.workload}: {w['gaussians']} gaussians SH{w['sh_degree']}, "
                               f"{w['views_per_step']} views/step at {w['width']}x{w['height']}",
                   "parallelism": "host threads, one view each"},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads, "kind": kind,
                         "sample": sample.describe()},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "c5":
        run_multi_scene(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

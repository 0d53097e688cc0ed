"""Data parallelism over views: one trainer per GPU over the same cloud.

The reference trains one view per step on one device (SplatTrainer.cpp:326-362).
Its gradients are sums over views (SplatRaster.h:133-137), so a step over the
views of several GPUs is: every rank renders and differentiates its own views
(pxs_trainer_accumulate), the gradient buffers are summed over the ranks in
place (one all-reduce per buffer), and every rank takes the same Adam step with
the same sums (pxs_trainer_apply). The densify decisions depend only on those
sums and on the cloud, so the replicas stay identical.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence

_DTYPES = {"float32": "<f4", "int32": "<i4"}


class _DeviceArray:
    """A device buffer described by __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr: int, count: int, dtype: str):
        self.__cuda_array_interface__ = {
            "shape": (count,), "typestr": _DTYPES[dtype], "data": (ptr, False), "version": 3,
            "strides": None}


def device_tensors(buffers) -> List["object"]:
    """torch tensors aliasing (pointer, count, dtype) device buffers."""
    import torch

    return [torch.as_tensor(_DeviceArray(p, n, d), device="cuda") for p, n, d in buffers
            if n > 0]


def all_reduce_sum(tensors, group=None) -> None:
    """Sums each tensor over the ranks of `group`, in place."""
    import torch.distributed as dist

    for t in tensors:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def mean_loss(loss: float, n_views: int, group=None, device: str = "cpu") -> float:
    """The mean loss over every rank's views, from this rank's mean."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([loss * n_views, float(n_views)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t[0] / t[1]) if t[1] > 0 else 0.0


class DataParallelStep:
    """One data-parallel step of `trainer` (a SplatTrainer, or anything with
    accumulate / apply / gradient tensors):

        step = DataParallelStep(trainer)
        loss = step(view_ids_of_this_rank)

    `buffers` returns the tensors to sum (default: the trainer's device
    gradient buffers); `reduce` sums them over the ranks (default: an
    all-reduce over `group`); `device` is where the loss is reduced."""

    def __init__(self, trainer, group=None, buffers: Optional[Callable[[], list]] = None,
                 reduce: Optional[Callable[[list], None]] = None, device: str = "cuda",
                 graph: bool = True):
        self.trainer = trainer
        self.group = group
        self.buffers = buffers or (lambda: device_tensors(trainer.gradient_buffers()))
        self.reduce = reduce or (lambda ts: all_reduce_sum(ts, group))
        self.device = device
        self.graph = graph

    def __call__(self, view_ids: Sequence[int]) -> float:
        loss = self.trainer.accumulate(view_ids, self.graph)
        if self.device == "cuda":
            # the sums run ordered on the trainer's stream, so its Adam step
            # (queued by apply) waits for them
            import torch

            with torch.cuda.stream(torch.cuda.ExternalStream(self.trainer.stream())):
                self.reduce(self.buffers())
        else:
            self.reduce(self.buffers())
        total = mean_loss(loss, len(view_ids), self.group, self.device)
        self.trainer.apply(total)
        return total

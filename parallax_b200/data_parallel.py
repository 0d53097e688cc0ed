"""Data parallelism over views: one trainer per GPU over the same cloud.

The reference trains one view per step on one device (SplatTrainer.cpp:326-362).
Its gradients are sums over views (SplatRaster.h:133-137), so a step over the
views of several GPUs is: every rank renders and differentiates its own views
(pxs_trainer_accumulate), the trainer's reduction block -- parameter
gradients, screen gradient, visible counts and the loss -- is summed over the
ranks with one all-reduce in place, and every rank takes the same Adam step
with the same sums (pxs_trainer_apply), reading the mean loss over all ranks'
views from the block. The densify decisions depend only on those sums and on
the cloud, so the replicas stay identical.
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


def _block_tensor(block):
    """A trainer's reduction block as a tensor: a (device pointer, float count)
    pair is aliased in place; a tensor is taken as it is."""
    if isinstance(block, tuple):
        return device_tensors([(block[0], block[1], "float32")])[0]
    return block


class DataParallelStep:
    """One data-parallel step of `trainer` (a SplatTrainer, or anything with
    accumulate / apply / reduction_block):

        step = DataParallelStep(trainer)
        step(view_ids_of_this_rank)

    `block` returns the one tensor to sum (default: the trainer's device
    reduction block); `reduce` sums a list of tensors over the ranks (default:
    an all-reduce over `group`); `device` "cuda" runs the sum on the trainer's
    stream. Returns the trainer's last loss when it has one."""

    def __init__(self, trainer, group=None, block: Optional[Callable[[], object]] = None,
                 reduce: Optional[Callable[[list], None]] = None, device: str = "cuda",
                 graph: bool = True):
        self.trainer = trainer
        self.group = group
        self.block = block or (lambda: _block_tensor(trainer.reduction_block()))
        self.reduce = reduce or (lambda ts: all_reduce_sum(ts, group))
        self.device = device
        self.graph = graph

    def __call__(self, view_ids: Sequence[int]):
        self.trainer.accumulate(view_ids, self.graph)
        if self.device == "cuda":
            # the sum runs ordered on the trainer's stream, so the Adam step
            # that apply queues there waits for it
            import torch

            with torch.cuda.stream(torch.cuda.ExternalStream(self.trainer.stream())):
                self.reduce([self.block()])
        else:
            self.reduce([self.block()])
        self.trainer.apply(float("nan"))  # the mean loss comes from the summed block
        last = getattr(self.trainer, "last_loss", None)
        return last() if callable(last) else last

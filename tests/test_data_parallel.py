"""The data-parallel step over two ranks (gloo on CPU): every rank ends with
the summed gradients and the mean loss over all ranks' views, and the ranks
take identical optimiser steps. A stand-in trainer with host buffers takes the
place of the GPU trainer; the GPU test drives the real one on one device."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from parallax_b200.data_parallel import DataParallelStep


class HostTrainer:
    """accumulate / apply on host buffers: the gradients of view v are
    (v + 1) * base, the loss of view v is v."""

    def __init__(self, n):
        self.base = np.arange(n, dtype=np.float32)
        self.grads = torch.zeros(n, dtype=torch.float32)
        self.screen = torch.zeros(n, dtype=torch.float32)
        self.visible = torch.zeros(n, dtype=torch.int32)
        self.params = torch.zeros(n, dtype=torch.float32)
        self.losses = []

    def accumulate(self, view_ids, graph=True):
        for v in view_ids:
            self.grads += torch.from_numpy((v + 1) * self.base)
            self.screen += 0.5
            self.visible += 1
        return float(np.mean(view_ids))

    def apply(self, loss):
        self.params -= 0.01 * self.grads  # stands in for the optimiser
        self.grads.zero_()
        self.screen.zero_()
        self.visible.zero_()
        self.losses.append(loss)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = HostTrainer(6)
        step = DataParallelStep(t, buffers=lambda: [t.grads, t.screen, t.visible],
                                device="cpu")
        views = [[0, 2], [1, 3]][rank]
        seen = []
        for _ in range(2):
            before = t.grads.clone()
            orig = t.apply

            def capture(loss, t=t, orig=orig):
                seen.append((t.grads.clone().numpy(), t.screen.clone().numpy(),
                             t.visible.clone().numpy()))
                orig(loss)
            t.apply = capture
            step(views)
            t.apply = orig
            assert before.abs().sum() == 0
        out[rank] = (t.params.numpy().copy(), list(t.losses), seen)
    finally:
        dist.destroy_process_group()


def test_two_ranks_sum_gradients_and_stay_identical():
    world = 2
    port = _free_port()
    out = mp.Manager().dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn")
    p0, l0, s0 = out[0]
    p1, l1, s1 = out[1]
    base = np.arange(6, dtype=np.float32)
    expect = (1 + 3 + 2 + 4) * base  # views 0, 2 on rank 0 and 1, 3 on rank 1
    for seen in (s0, s1):
        for grads, screen, visible in seen:
            assert np.array_equal(grads, expect)
            assert np.array_equal(screen, np.full(6, 2.0, np.float32))
            assert np.array_equal(visible, np.full(6, 4, np.int32))
    assert np.array_equal(p0, p1)
    assert l0 == l1 == [1.5, 1.5]  # mean of views 0..3


@pytest.mark.gpu
def test_single_rank_split_step_matches_the_batched_step():
    """accumulate + apply on one GPU (a world of one) takes the same step as
    step_batch: same losses, parameters within the atomics' summation order."""
    import parallax_b200 as px
    from parallax_b200.data_parallel import device_tensors
    import oracle_lib as O

    params, rest = O.random_cloud(21, 8000, 3, log_scale_mean=-4.0)
    truth, _ = O.random_cloud(22, 8000, 3, log_scale_mean=-4.0)
    views = O.orbit_views(6, 96, 72, seed=5)
    images = [px.render_splats(px.GaussianCloud(truth, 3, rest), v.camera(),
                               px.RasterOptions(sh_degree=3))[0] for v in views]
    cfg = px.TrainConfig(iterations=50, sh_degree=3, sh_increase_interval=0,
                         densify_from_iteration=1000, densify_until_iteration=1000)
    pairs = [(v.camera(), im) for v, im in zip(views, images)]
    a = px.SplatTrainer(px.GaussianCloud(params, 3, rest), pairs, cfg)
    b = px.SplatTrainer(px.GaussianCloud(params, 3, rest), pairs, cfg)
    la, lb = [], []
    for s in range(3):
        ids = [(s + i) % 6 for i in range(3)]
        la.append(a.step_batch(3, ids))
        loss = b.accumulate(ids)
        bufs = device_tensors(b.gradient_buffers())
        assert len(bufs) == 3 and bufs[0].numel() == b.P * 8000
        b.apply(loss)
        lb.append(loss)
    assert np.allclose(la, lb, rtol=1e-5)
    assert np.abs(a.cloud_params() - b.cloud_params()).max() <= 1e-4
    assert a.state()["iteration"] == b.state()["iteration"] == 3

"""The data-parallel step over two ranks (gloo on CPU): one all-reduce of the
reduction block leaves every rank with the summed gradients, statistics and
loss, the ranks take identical optimiser steps, and their densify decisions --
made from the summed statistics by the reference's densifyAndPrune as the
oracle restates it (SplatDensify.cpp:28-109) -- give identical clouds. A
stand-in trainer with host buffers takes the place of the GPU trainer; the GPU
test drives the real one on one device."""
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
    """accumulate / apply on one host block laid out like the device trainer's
    reduction block: [gradients | screen gradient | visible counts (floats) |
    mean loss x views, views]. View v adds (v + 1) * base to the gradients,
    0.5 (g % 3) to the screen gradient of each gaussian g it sees (every other
    gaussian, offset by v) and 1 to their visible counts; its loss is v. Every
    `densify_every` steps apply() runs densifyAndPrune on the summed
    statistics."""

    def __init__(self, params, rest, densify_every=0, config=None):
        self.params = params.copy()
        self.rest = rest
        self.n = params.shape[1]
        self.block = torch.zeros(3 * self.n + 2, dtype=torch.float32)
        self.acc_screen = np.zeros(self.n, np.float32)
        self.acc_visible = np.zeros(self.n, np.int32)
        self.densify_every = densify_every
        self.config = config
        self.rng = 7
        self.iteration = 0
        self.losses, self.seen, self.counts = [], [], []

    def reduction_block(self):
        return self.block

    def accumulate(self, view_ids, graph=True):
        n = self.n
        base = torch.arange(n, dtype=torch.float32)
        for v in view_ids:
            sees = torch.from_numpy(((np.arange(n) + v) % 2 == 0).astype(np.float32))
            self.block[:n] += (v + 1) * base
            self.block[n:2 * n] += 0.5 * sees * (torch.arange(n) % 3).float()
            self.block[2 * n:3 * n] += sees
        self.block[3 * n] += float(np.mean(view_ids)) * len(view_ids)
        self.block[3 * n + 1] += len(view_ids)
        return float(np.mean(view_ids))

    def apply(self, loss):
        import oracle_lib as O

        n = self.n
        b = self.block.numpy()
        if np.isnan(loss):
            loss = float(b[3 * n] / b[3 * n + 1])
        self.seen.append((b[:n].copy(), b[n:2 * n].copy(), np.rint(b[2 * n:3 * n]).astype(np.int32)))
        self.params[0] -= 0.01 * b[:n]  # stands in for the optimiser
        self.acc_screen += b[n:2 * n]
        self.acc_visible += np.rint(b[2 * n:3 * n]).astype(np.int32)
        self.block.zero_()
        self.losses.append(loss)
        self.iteration += 1
        if self.densify_every and self.iteration % self.densify_every == 0:
            self.params, _, self.rng, counts = O.oracle_densify(
                self.params, self.rest, self.acc_screen, self.acc_visible, self.config, 2.5,
                600, self.rng)
            self.counts.append(counts)
            self.n = self.params.shape[1]
            self.block = torch.zeros(3 * self.n + 2, dtype=torch.float32)
            self.acc_screen = np.zeros(self.n, np.float32)
            self.acc_visible = np.zeros(self.n, np.int32)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _cloud():
    import oracle_lib as O

    return O.random_cloud(5, 400, 1, log_scale_mean=-3.0)


def _rank(rank, world, port, out):
    from parallax_b200._abi import TrainConfig

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        params, rest = _cloud()
        cfg = TrainConfig(densify_grad_threshold=0.3, max_gaussians=100000)
        t = HostTrainer(params, rest, densify_every=2, config=cfg)
        calls = []

        def reduce(tensors):
            calls.append(len(tensors))
            for x in tensors:
                dist.all_reduce(x, op=dist.ReduceOp.SUM)

        step = DataParallelStep(t, reduce=reduce, device="cpu")
        views = [[0, 2], [1, 3]][rank]
        for _ in range(3):
            step(views)
        out[rank] = (t.params.copy(), list(t.losses), t.seen, t.counts, calls)
    finally:
        dist.destroy_process_group()


def test_two_ranks_sum_one_block_densify_alike_and_stay_identical():
    world = 2
    port = _free_port()
    out = mp.Manager().dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn")
    p0, l0, s0, c0, calls0 = out[0]
    p1, l1, s1, c1, calls1 = out[1]
    assert calls0 == calls1 == [1, 1, 1]  # one collective per step
    n = 400
    base = np.arange(n, dtype=np.float32)
    expect = (1 + 3 + 2 + 4) * base  # views 0, 2 on rank 0 and 1, 3 on rank 1
    for seen in (s0, s1):
        grads, screen, visible = seen[0]
        assert np.array_equal(grads, expect)
        # each gaussian is seen by 2 of the 4 views
        assert np.array_equal(screen, (np.arange(n) % 3).astype(np.float32))
        assert np.array_equal(visible, np.full(n, 2, np.int32))
    assert l0 == l1 == [1.5, 1.5, 1.5]  # the mean over views 0..3, from the block
    # the densify step (after step 2) saw the summed statistics on both ranks
    assert c0 == c1 and len(c0) == 1
    assert np.array_equal(p0.view(np.uint32), p1.view(np.uint32))
    # and decided what one process with the whole batch decides
    import oracle_lib as O
    from parallax_b200._abi import TrainConfig

    params, rest = _cloud()
    params = params.copy()
    params[0] -= 0.01 * expect
    params[0] -= 0.01 * expect
    one, _, _, counts = O.oracle_densify(params, rest,
                                         2 * (np.arange(n) % 3).astype(np.float32),
                                         np.full(n, 4, np.int32),
                                         TrainConfig(densify_grad_threshold=0.3,
                                                     max_gaussians=100000), 2.5, 600, 7)
    assert counts == c0[0] and counts[0] + counts[1] > 0 and counts[0] + counts[1] < n
    one[0] -= 0.01 * (10 * np.arange(one.shape[1], dtype=np.float32))  # the third step
    assert np.array_equal(one.view(np.uint32), p0.view(np.uint32))


@pytest.mark.gpu
def test_single_rank_split_step_matches_the_batched_step():
    """accumulate + one reduction of the block + apply on one GPU (a world of
    one: the reduction is the identity) takes the same step as step_batch:
    same losses, parameters within the atomics' summation order; the block is
    one buffer of (P + 2) N + 2 floats and apply takes the loss from it."""
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
    reduced = []
    step = DataParallelStep(b, reduce=lambda ts: reduced.append([t.numel() for t in ts]))
    la, lb = [], []
    for s in range(3):
        ids = [(s + i) % 6 for i in range(3)]
        la.append(a.step_batch(3, ids))
        lb.append(step(ids))
    assert reduced == [[(b.P + 2) * 8000 + 2]] * 3
    bufs = device_tensors(b.gradient_buffers())
    assert [t.numel() for t in bufs] == [b.P * 8000, 8000, 8000]
    assert np.allclose(la, lb, rtol=1e-5)
    assert np.abs(a.cloud_params() - b.cloud_params()).max() <= 1e-4
    assert a.state()["iteration"] == b.state()["iteration"] == 3

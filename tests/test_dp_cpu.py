"""Data-parallel training host logic on CPU: two gloo ranks run the same per-step reductions the NCCL path runs
(hush_b200.dp), with a CPU stand-in for the device trainer (its gradient and loss accumulators are CPU tensors and its
step is Adam in float64)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from hush_b200.dp import DataParallel, finish_step

NW = 812


class FakeTrainer:
    """Same accumulator / step contract as hush_b200.train.Trainer, on the CPU."""

    def __init__(self, theta):
        self.theta = torch.as_tensor(theta, dtype=torch.float64).clone()
        self.grad = torch.zeros(NW, dtype=torch.float64)
        self.loss = torch.zeros(1, dtype=torch.float64)
        self.m = torch.zeros(NW, dtype=torch.float64)
        self.v = torch.zeros(NW, dtype=torch.float64)
        self.t = 0

    def add_frame(self, g, loss):
        self.grad += g
        self.loss += loss

    def accumulators(self):
        return self.grad, self.loss

    def loss_sum(self):
        v = float(self.loss.item())
        self.loss.zero_()
        return v

    def step(self, lr, clip=1.0, beta1=0.9, beta2=0.999, eps=1e-8):
        n = float(self.grad.norm())
        g = self.grad * (clip / n if clip > 0 and n > clip else 1.0)
        self.t += 1
        self.m = beta1 * self.m + (1 - beta1) * g
        self.v = beta2 * self.v + (1 - beta2) * g * g
        mh, vh = self.m / (1 - beta1 ** self.t), self.v / (1 - beta2 ** self.t)
        self.theta -= lr * mh / (vh.sqrt() + eps)
        self.grad.zero_()
        return n


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dp = DataParallel()
        out = {"rank": dp.rank, "world": dp.world}
        # disjoint window seeds
        rng = dp.seed_rng(7)
        out["seeds"] = [dp.window_seed(rng, 2048) for _ in range(200)]
        # averaging in place
        t = torch.full((NW,), float(rank + 1), dtype=torch.float64)
        dp.average_(t)
        out["avg"] = float(t[0]), float(t[-1])
        # broadcast of rank 0's initial weights
        th = torch.from_numpy(np.random.default_rng(100 + rank).normal(size=NW))
        dp.broadcast_(th)
        tr = FakeTrainer(th)
        # three steps on different per-rank gradients: the ranks must stay identical
        g_rng = np.random.default_rng(1000 + rank)
        local_sums = []
        for _ in range(3):
            gsum, lsum = np.zeros(NW), 0.0
            for _ in range(4):  # frames of the step
                g = g_rng.normal(size=NW) * 0.1
                lo = float(g_rng.uniform())
                tr.add_frame(torch.from_numpy(g), lo)
                gsum += g
                lsum += lo
            local_sums.append((gsum, lsum))
            loss, gn = finish_step(tr, dp, 4, 1e-2, 1.0)
            out.setdefault("loss", []).append(loss)
        out["theta"] = tr.theta.numpy().copy()
        out["local_sums"] = local_sums
        out["div"] = dp.max_divergence(tr.theta)
        q.put(out)
    finally:
        dist.destroy_process_group()


def test_data_parallel_step_keeps_ranks_identical():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = sorted([q.get(timeout=120) for _ in range(world)], key=lambda r: r["rank"])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    a, b = res
    assert a["world"] == b["world"] == 2
    # seeds: each rank in its residue class, inside the range, no overlap
    assert all(s % 2 == 0 and 0 <= s < 2048 for s in a["seeds"])
    assert all(s % 2 == 1 and 0 <= s < 2048 for s in b["seeds"])
    assert a["avg"] == b["avg"] == (1.5, 1.5)
    # identical weights after the steps, and equal to a single-process replay on the averaged gradients
    np.testing.assert_array_equal(a["theta"], b["theta"])
    assert a["div"] == b["div"] == 0.0
    np.testing.assert_allclose(a["loss"], b["loss"])
    th0 = torch.from_numpy(np.random.default_rng(100).normal(size=NW))
    replay = FakeTrainer(th0)
    for k in range(3):
        g = (a["local_sums"][k][0] + b["local_sums"][k][0]) / 2
        lo = (a["local_sums"][k][1] + b["local_sums"][k][1]) / 2
        replay.add_frame(torch.from_numpy(g), lo)
        assert replay.loss_sum() / 4 == pytest.approx(a["loss"][k])
        replay.step(1e-2, clip=1.0)
    np.testing.assert_allclose(replay.theta.numpy(), a["theta"], rtol=0, atol=1e-12)


def test_single_process_is_a_no_op():
    dp = DataParallel()
    assert (dp.rank, dp.world) == (0, 1)
    t = torch.ones(3)
    dp.average_(t)
    assert t.tolist() == [1.0, 1.0, 1.0]
    assert dp.max_divergence(t) == 0.0
    rng = dp.seed_rng(3)
    assert all(0 <= dp.window_seed(rng, 10) < 10 for _ in range(50))


def test_window_seeds_cover_each_residue_class_and_need_one_seed_per_rank():
    dp = DataParallel()
    for rank, world, n in ((0, 3, 10), (1, 3, 10), (2, 3, 10), (3, 4, 4)):
        dp.rank, dp.world = rank, world
        rng = np.random.default_rng(rank)
        got = {dp.window_seed(rng, n) for _ in range(400)}
        assert got == {s for s in range(n) if s % world == rank}
    dp.rank, dp.world = 2, 4
    with pytest.raises(ValueError, match="cannot give each of 4 ranks"):
        dp.window_seed(np.random.default_rng(0), 3)

"""world_size-2 gloo tests (CPU) of the multi-rank logic: VDF sharding, output
cell sharding + all-gather of Q, and the max-over-ranks timing reduction."""
import os
import socket

import numpy as np
import pytest

from dgv0d3v_direct_collision_b200.sharding import balanced_range, node_shard, vdf_shard


def test_balanced_ranges_cover_exactly():
    for n in (0, 1, 7, 256, 1000):
        for world in (1, 2, 3, 8):
            spans = [balanced_range(n, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from dgv0d3v_direct_collision_b200.sharding import gather_node_slices
        from oracle.oracle import Oracle
        o = Oracle(2, 3, 3.0)
        cap, A, xi, xi1 = o.synth_A(seed=21, support=1)
        o.set_A(cap, A, xi, xi1)
        f = o.maxwellian(0.6, 0.5, 0.0, 0.0, 1.0) + o.maxwellian(0.4, -0.7, 0.2, 0.0, 0.5)
        a, b = node_shard(o.Nc, o.P, world, rank)
        q = o.collide(f, nodes=np.arange(a, b))[a:b]
        full = gather_node_slices(torch.tensor(q), o.Nc, o.P).numpy()
        ref = o.collide(f)
        out[rank] = float(np.abs(full - ref).max() / np.abs(ref).max())
        # replicas: disjoint VDF shards, elapsed time reduced with MAX
        s0, s1 = vdf_shard(256, world, rank)
        t = torch.tensor([float(rank + 1)])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sizes = torch.tensor([float(s1 - s0)])
        dist.all_reduce(sizes)
        out[world + rank] = (float(t.item()), float(sizes.item()))
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_and_max():
    import torch.multiprocessing as mp
    port = _free_port()
    world = 2
    mgr = mp.get_context("spawn").Manager()  # no fork of this (threaded) process
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    assert out[0] == 0.0 and out[1] == 0.0  # bit-identical assembly
    for r in range(world):
        assert out[world + r] == (2.0, 256.0)


class _OracleCells:
    """The oracle behind the solver methods the sharded helpers call."""

    def __init__(self, o, kappa):
        self.o, self.Nc, self.P, self.kappa, self.projection = o, o.Nc, o.P, kappa, False

    def collide_cells(self, f, cell0, cell1, out=None, precision=None):
        import torch
        a, b = cell0 * self.P, cell1 * self.P
        return torch.tensor(self.o.collide(f.numpy(), nodes=np.arange(a, b))[a:b])


def _rk_worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from dgv0d3v_direct_collision_b200.sharding import sharded_rk_step
        from oracle.oracle import Oracle
        o = Oracle(2, 3, 3.0)
        cap, A, xi, xi1 = o.synth_A(seed=22, support=1)
        o.set_A(cap, A, xi, xi1)
        f = o.maxwellian(0.6, 0.5, 0.0, 0.0, 1.0) + o.maxwellian(0.4, -0.7, 0.2, 0.0, 0.5)
        kappa, dt = 0.8, 0.02
        got = sharded_rk_step(_OracleCells(o, kappa), torch.tensor(f), dt, order=4).numpy()
        ref, _ = o.rk_step(f, dt, 4, kappa=kappa)
        out[rank] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref - f))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_rk_step():
    """A single VDF split by output cells over 2 ranks, one all-gather per RK
    stage, reproduces the unsplit RK4 step."""
    import torch.multiprocessing as mp
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()  # no fork of this (threaded) process
    out = mgr.dict()
    mp.spawn(_rk_worker, args=(2, port, out), nprocs=2, join=True)
    assert out[0] < 1e-12 and out[1] < 1e-12

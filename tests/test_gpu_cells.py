"""dgv_collide_cells (Q on a range of output cells, one rank's share of a
single-VDF evaluation split by cells) against the whole-grid evaluation, and
the sharded RK step on a one-rank NCCL group against the library's step."""
import os
import socket

import numpy as np
import pytest
import torch

from conftest import max_rel_err, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    import dgv0d3v_direct_collision_b200 as dgv
    from oracle.oracle import Oracle
    s = dgv.DGVSolver(3, 5, 6.0, kappa=0.9)
    s.generate_synthetic_A(seed=11, support=1)
    o = Oracle(3, 5, 6.0)
    f = o.maxwellian(1.0, 1.5, 0, 0, 0.5) + o.maxwellian(1.0, -1.5, 0, 0, 0.5)
    return s, f


@pytest.mark.parametrize("precision,tol", [("f64", 1e-12), ("f32c", 1e-6)])
def test_cell_slices_assemble_q(c1, precision, tol):
    s, f = c1
    full = s.EvalCollisionPeriodicAPlus_DGV(f, precision="f64")
    cuts = [0, 17, 60, 61, s.Nc]  # uneven shares, one of a single cell
    parts = [s.collide_cells(f, a, b, precision=precision) for a, b in zip(cuts, cuts[1:])]
    got = np.concatenate(parts)
    assert got.shape == full.shape
    assert rel_err(got, full) < tol
    if precision == "f64":
        assert max_rel_err(got, full) < 1e-12


def test_cell_slices_batched_device(c1):
    s, f = c1
    fb = torch.tensor(np.stack([f, 0.3 * f]), device="cuda")
    full = s.EvalCollisionPeriodicAPlus_DGV(fb).cpu().numpy()
    part = s.collide_cells(fb, 40, 90).cpu().numpy()
    assert part.shape == (2, 50 * s.P)
    assert rel_err(part, full[:, 40 * s.P:90 * s.P]) < 1e-12


def test_cell_range_errors(c1, ):
    import dgv0d3v_direct_collision_b200 as dgv
    s, f = c1
    for a, b in [(-1, 3), (5, 5), (0, s.Nc + 1)]:
        with pytest.raises(dgv.DGVError):
            s.collide_cells(f, a, b)
    with pytest.raises(dgv.DGVError):
        s.collide_cells(f, 0, 4, precision="tc")
    assert np.all(np.isfinite(s.collide_cells(f, 0, 4)))  # context still usable


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def test_sharded_rk_step_one_rank_nccl(c1):
    import torch.distributed as dist
    from dgv0d3v_direct_collision_b200.sharding import sharded_rk_step
    s, f = c1
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        g = torch.tensor(f, device="cuda")
        got = sharded_rk_step(s, g, 0.01, order=2)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    ref = g.clone()
    s.TimeIntegratorORK_SH_DGV(ref, 0.01, order=2)
    assert rel_err((got - g).cpu().numpy(), (ref - g).cpu().numpy()) < 1e-12

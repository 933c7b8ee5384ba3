"""The torch.autograd wrappers on the device path: gradients of the
collision operator (the library's VJP) against the oracle, RK steps against
the library's own TimeIntegratorORK_SH_DGV, and the checkpointed trajectory
adjoint against central finite differences of the FP64 forward."""
import numpy as np
import pytest
import torch

from conftest import rel_err
from helpers import golden_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gsol(golden):
    import dgv0d3v_direct_collision_b200 as dgv
    s = dgv.DGVSolver(int(golden["s"]), int(golden["M"]), float(golden["L"]), kappa=float(golden["kappa"]))
    s.load_A(golden["capphi"], golden["A"], golden["A_xi"], golden["A_xi1"], one_based=True)
    return s


def test_collision_grad_is_the_vjp(gsol, golden):
    from dgv0d3v_direct_collision_b200.autograd import collision
    o = golden_oracle(golden)
    rng = np.random.default_rng(3)
    v = rng.standard_normal(o.N)
    f = torch.tensor(golden["f0"], device="cuda", requires_grad=True)
    q = collision(f, gsol)
    assert rel_err(q.detach().cpu().numpy(), golden["q0"]) < 1e-12
    (q * torch.tensor(v, device="cuda")).sum().backward()
    assert rel_err(f.grad.cpu().numpy(), o.vjp(golden["f0"], v)) < 1e-12


def test_batched_and_tensor_core_forward(gsol, golden):
    from dgv0d3v_direct_collision_b200.autograd import collision
    f0 = torch.tensor(golden["f0"], device="cuda")
    f = torch.stack([f0, 0.5 * f0]).requires_grad_(True)
    q = collision(f, gsol, precision="tc")
    assert rel_err(q[0].detach().cpu().numpy(), golden["q0"]) < 1e-6
    q.sum().backward()
    g = f.grad.cpu().numpy()
    assert rel_err(g[1], 0.5 * g[0]) < 1e-12  # J(f) is linear in f (and the scaling exact)
    # the tensor-core forward's backward is the tensor-core VJP of the batch
    o = golden_oracle(golden)
    assert rel_err(g[0], o.vjp(golden["f0"], np.ones(o.N))) < 1e-6


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_rk_step_matches_library_step(gsol, golden, order):
    from dgv0d3v_direct_collision_b200.autograd import rk_step
    dt = 0.01
    f0 = golden["f0"]
    g = torch.tensor(f0, device="cuda")
    ref = g.clone()
    gsol.TimeIntegratorORK_SH_DGV(ref, dt, order=order)
    out = rk_step(g, gsol, dt, order)
    assert rel_err((out - g).cpu().numpy(), (ref - g).cpu().numpy()) < 1e-12


def test_trajectory_adjoint_vs_finite_differences(gsol, golden):
    from dgv0d3v_direct_collision_b200.autograd import rk_trajectory
    rng = np.random.default_rng(5)
    dt, n = 0.02, 3
    f0 = torch.tensor(golden["f0"], device="cuda")
    w = torch.tensor(rng.standard_normal(f0.numel()), device="cuda")
    d = torch.tensor(rng.standard_normal(f0.numel()), device="cuda") * f0.abs().max() * 1e-2
    f = f0.clone().requires_grad_(True)
    (w * rk_trajectory(f, gsol, dt, n, order=4)).sum().backward()
    eps = 1e-4
    with torch.no_grad():
        lp = (w * rk_trajectory(f0 + eps * d, gsol, dt, n, order=4)).sum().item()
        lm = (w * rk_trajectory(f0 - eps * d, gsol, dt, n, order=4)).sum().item()
    fd = (lp - lm) / (2 * eps)
    ad = float((f.grad * d).sum())
    assert abs(ad - fd) <= 1e-7 * max(1.0, abs(fd))

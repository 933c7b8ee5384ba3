"""The autograd wrappers' adjoint logic, on the CPU: a dense bilinear
operator Q_i = sum_jk T_ijk f_j f_k stands in for the library (same method
names), and torch.autograd.gradcheck compares the wrappers' backward (VJP
calls, the RK discrete adjoint with recomputed stages) with finite
differences."""
import pytest
import torch

from dgv0d3v_direct_collision_b200.autograd import RK_TABLEAUX, collision, rk_step, rk_trajectory


class DenseBilinear:
    def __init__(self, n, seed=0, kappa=0.7):
        g = torch.Generator().manual_seed(seed)
        self.T = torch.randn(n, n, n, generator=g, dtype=torch.float64) / n
        self.kappa = kappa
        self.projection = False

    def collide(self, f, out, precision=None):
        out.copy_(torch.einsum("ijk,...j,...k->...i", self.T, f, f))
        return out

    def vjp(self, f, v, out):
        out.copy_(torch.einsum("i,ijk,k->j", v, self.T, f) + torch.einsum("i,ijk,j->k", v, self.T, f))
        return out


@pytest.fixture(scope="module")
def op():
    return DenseBilinear(7)


def test_collision_gradcheck(op):
    f = torch.randn(2, 7, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda x: collision(x, op, scale=0.3), (f,))


@pytest.mark.parametrize("order", sorted(RK_TABLEAUX))
def test_rk_step_gradcheck(op, order):
    f = torch.randn(7, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda x: rk_step(x, op, 0.05, order), (f,))


def test_rk_step_matches_explicit_stages(op):
    """RK4 written out as in the reference (k4 reuses ft2)."""
    f = torch.randn(7, dtype=torch.float64)
    h = op.kappa * 0.05
    F = lambda x: h * op.collide(x, torch.empty_like(x))
    k1 = F(f); k2 = F(f + k1 / 2); k3 = F(f + k1 / 4 + k2 / 4); k4 = F(f - k2 + 2 * k3)
    ref = f + k1 / 6 + k3 * 2 / 3 + k4 / 6
    assert torch.allclose(rk_step(f, op, 0.05, 4), ref, rtol=1e-14, atol=1e-14)


def test_trajectory_gradcheck(op):
    f = torch.randn(7, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda x: rk_trajectory(x, op, 0.05, 3, order=2), (f,))


def test_projection_is_refused(op):
    p = DenseBilinear(7)
    p.projection = True
    with pytest.raises(ValueError):
        collision(torch.zeros(7, dtype=torch.float64), p)

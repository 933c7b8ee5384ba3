"""The batched adjoint on the tensor cores (dgv_vjp_batched, DGV_PREC_TC: the
block form's G = f(c2) W1 and G = f(c1) W2 contracted with c = 2v/w) against
the oracle's VJP (the adjoint of collision_mod.f90:213-216), the FP64 device
VJP, central differences of the FP64 operator, and the reference's linearised
operator 2 fmA^T v at a Maxwellian (collision_mod.f90:448-449, 357).

Tolerance: 1e-6 norm-wise relative, as for the tensor-core forward (split
fp16 operands, FP32 accumulation, compensated block sums)."""
import numpy as np
import pytest

from conftest import rel_err
from helpers import golden_oracle, mixture_vdf

pytestmark = pytest.mark.gpu

TOLTC = 1e-6


@pytest.fixture(scope="module")
def c1():
    """The 15^3 grid (s=3, M=5, [-6,6]^3) with seeded synthetic A on both sides."""
    import dgv0d3v_direct_collision_b200 as m
    from oracle.oracle import Oracle
    o = Oracle(3, 5, 6.0)
    o.set_A(*o.synth_A(seed=11, support=1))
    s = m.DGVSolver(3, 5, 6.0)
    s.generate_synthetic_A(seed=11, support=1)
    yield {"oracle": o, "solver": s}
    s.close()


def test_vjp_tc_golden_s2M3(golden):
    """8 nodes per cell, one VDF (tile of 32 VDFs x 4 cells), host arrays."""
    import dgv0d3v_direct_collision_b200 as m
    s = m.DGVSolver(int(golden["s"]), int(golden["M"]), float(golden["L"]), kappa=float(golden["kappa"]))
    s.load_A(golden["capphi"], golden["A"], golden["A_xi"], golden["A_xi1"], one_based=True)
    o = golden_oracle(golden)
    rng = np.random.default_rng(3)
    v = rng.standard_normal(o.N)
    g = s.vjp(golden["f0"], v, precision="tc")
    assert rel_err(g, o.vjp(golden["f0"], v)) < TOLTC


@pytest.mark.parametrize("nb", [1, 37, 150, 300])
def test_vjp_tc_batched_vs_f64_and_oracle(c1, nb):
    """Tiles of 32, 64 and 128 VDFs (300: the second CTA of a row tile has one
    VDF tile); densities over four decades; every VDF against the FP64
    device VJP, two against the oracle."""
    o, s = c1["oracle"], c1["solver"]
    rng = np.random.default_rng(nb)
    fs = np.stack([mixture_vdf(o.u, o.v, o.w, rng, normalise_w=o.gwts) * 10.0 ** rng.uniform(-2, 2)
                   for _ in range(nb)])
    vs = rng.standard_normal((nb, o.N))
    import torch
    f_d = torch.tensor(fs, device="cuda")
    v_d = torch.tensor(vs, device="cuda")
    g_tc = s.vjp(f_d, v_d, precision="tc").cpu().numpy()
    g64 = s.vjp(f_d, v_d, precision="f64").cpu().numpy()
    for k in range(nb):
        assert rel_err(g_tc[k], g64[k]) < TOLTC, k
    for k in {0, nb - 1}:
        assert rel_err(g_tc[k], o.vjp(fs[k], vs[k])) < TOLTC, k
        assert rel_err(g64[k], o.vjp(fs[k], vs[k])) < 1e-12, k


def test_vjp_tc_central_differences(c1):
    """<g, d> against (<v, Q(f + eps d)> - <v, Q(f - eps d)>) / (2 eps) with the
    FP64 operator, eps = 1e-6 (exact up to rounding: Q is quadratic)."""
    o, s = c1["oracle"], c1["solver"]
    rng = np.random.default_rng(21)
    fs = np.stack([mixture_vdf(o.u, o.v, o.w, rng, normalise_w=o.gwts) for _ in range(4)])
    vs = rng.standard_normal((4, o.N))
    g = s.vjp(fs, vs, precision="tc")
    eps = 1e-6
    for k in range(4):
        for _ in range(2):
            d = rng.standard_normal(o.N) * fs[k]
            qp = s.EvalCollisionPeriodicAPlus_DGV(fs[k] + eps * d)
            qm = s.EvalCollisionPeriodicAPlus_DGV(fs[k] - eps * d)
            fd = (vs[k] @ qp - vs[k] @ qm) / (2 * eps)
            assert abs(g[k] @ d - fd) <= TOLTC * np.abs(g[k] * d).sum(), (k, g[k] @ d, fd)


def test_vjp_tc_equals_linearized_operator_at_maxwellian(c1):
    """J^T v at a unit Maxwellian equals 2 fmA^T v, the reference's linearised
    operator (PrepareFMA_DGV collision_mod.f90:377-464, EvalCollisionLinear
    :346-359), on the 15^3 grid."""
    o, s = c1["oracle"], c1["solver"]
    fm = o.maxwellian(1.0, 0.0, 0.0, 0.0, 1.0)
    rng = np.random.default_rng(8)
    vs = rng.standard_normal((3, o.N))
    fmA = o.prepare_fma(fm)
    g = s.vjp(np.stack([fm] * 3), vs, precision="tc")
    for k in range(3):
        assert rel_err(g[k], 2.0 * fmA.T @ vs[k]) < TOLTC


def test_derivative_precisions_refused_or_served(c1):
    """dgv_vjp serves FP64 and tensor cores; FP32-compensated is refused.
    dgv_jvp / dgv_apply_linear compute in FP64 only and refuse the others
    instead of silently running FP64."""
    from dgv0d3v_direct_collision_b200 import _lib
    o, s = c1["oracle"], c1["solver"]
    L = _lib.load()
    f = o.maxwellian(1.0, 0.3, 0.0, 0.0, 1.0)
    v = np.random.default_rng(2).standard_normal(o.N)
    g = np.zeros(o.N)
    assert L.dgv_vjp(s._h, f.ctypes.data, v.ctypes.data, g.ctypes.data, _lib.DGV_PREC_F32C) == _lib.DGV_EUNSUP
    assert L.dgv_vjp(s._h, f.ctypes.data, v.ctypes.data, g.ctypes.data, _lib.DGV_PREC_TC) == 0
    assert rel_err(g, o.vjp(f, v)) < TOLTC
    for prec in (_lib.DGV_PREC_F32C, _lib.DGV_PREC_TC):
        assert L.dgv_jvp(s._h, f.ctypes.data, v.ctypes.data, g.ctypes.data, prec) == _lib.DGV_EUNSUP
    s.PrepareFMA_DGV(f)
    assert L.dgv_apply_linear(s._h, v.ctypes.data, g.ctypes.data, _lib.DGV_PREC_TC) == _lib.DGV_EUNSUP

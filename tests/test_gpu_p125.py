"""Grids of 5 Gauss nodes per cell and axis (P = 125 basis functions per
cell, the node count of the 45^3 configuration): the CUDA-core kernels serve
them in slices of 25 basis functions per CTA.  Grid: s=5, M=3 on [-5,5]^3
(N = 3375, 4.27 M pairs, 533 M records), seeded synthetic A-arrays.

Against: the oracle's EvalCollisionPeriodicAPlus_DGV (collision_mod.f90:143-229)
at every cell for three basis functions (the oracle holds the records of one
basis function at a time); the sliced adjoint and mixed-terms (JVP) kernels
against central differences of the FP64 operator.  The tensor-core forms
serve at most 32 nodes per cell and refuse the grid."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

S, M, L, SEED = 5, 3, 5.0, 11


@pytest.fixture(scope="module")
def p125():
    import dgv0d3v_direct_collision_b200 as m
    s = m.DGVSolver(S, M, L)
    s.generate_synthetic_A(seed=SEED, support=1)
    rng = np.random.default_rng(3)
    u, v, w = s.nodes_u, s.nodes_v, s.nodes_w
    fs = np.stack([np.exp(-((u - c[0]) ** 2 + (v - c[1]) ** 2 + (w - c[2]) ** 2) / T) / (np.pi * T) ** 1.5
                   for c, T in [(rng.uniform(-1, 1, 3), rng.uniform(0.6, 1.4)) for _ in range(3)]])
    yield {"solver": s, "fs": fs}
    s.close()


def test_p125_f64_and_f32c_vs_oracle(p125):
    from oracle.oracle import Oracle
    s, fs = p125["solver"], p125["fs"]
    assert s.P == 125
    q64 = s.EvalCollisionPeriodicAPlus_DGV(fs)
    q32 = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="f32c")
    o = Oracle(S, M, L)
    for p in (0, 62, 124):
        o.set_A(*o.synth_A(seed=SEED, support=1, p_only=p))
        nodes = np.arange(o.Nc) * o.P + p
        for k in range(len(fs)):
            ref = o.collide(fs[k], nodes=nodes)[nodes]
            assert rel_err(q64[k][nodes], ref) < 1e-12, (p, k)
            assert np.abs(q64[k][nodes] - ref).max() <= 1e-12 * np.abs(ref).max(), (p, k)
            assert rel_err(q32[k][nodes], ref) < 1e-6, (p, k)


def test_p125_adjoint_and_jvp_vs_central_differences(p125):
    s, fs = p125["solver"], p125["fs"]
    rng = np.random.default_rng(8)
    f = fs[0]
    v = rng.standard_normal(s.N)
    d = rng.standard_normal(s.N) * f
    eps = 1e-6
    qp = s.EvalCollisionPeriodicAPlus_DGV(f + eps * d)
    qm = s.EvalCollisionPeriodicAPlus_DGV(f - eps * d)
    jd_fd = (qp - qm) / (2 * eps)                   # exact up to rounding: Q is quadratic
    g = s.vjp(f, v)
    assert abs(g @ d - v @ jd_fd) <= 1e-8 * np.abs(g * d).sum()
    jd = s.jvp(f, d)
    assert rel_err(jd, jd_fd) < 1e-8


def test_p125_tensor_cores_refused(p125):
    from dgv0d3v_direct_collision_b200 import _lib
    s, fs = p125["solver"], p125["fs"]
    with pytest.raises(_lib.DGVError) as ei:
        s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    assert ei.value.code == _lib.DGV_EUNSUP

"""CPU tests of the oracle (the checker) against the golden vectors of the
independent pure-Python restatement and against the reference's own
invariants.  No GPU needed."""
import numpy as np
import pytest

from conftest import max_rel_err, rel_err
from helpers import golden_oracle
from oracle.oracle import Oracle, gauss_legendre


def test_gauss_legendre_matches_numpy():
    for n in range(1, 11):
        x, w = gauss_legendre(n)
        xr, wr = np.polynomial.legendre.leggauss(n)
        assert np.allclose(x, xr, rtol=0, atol=2e-15)
        assert np.allclose(w, wr, rtol=0, atol=2e-15)


def test_grid_nodes_and_canonical_cell(golden):
    o = Oracle(int(golden["s"]), int(golden["M"]), float(golden["L"]))
    assert o.N == len(golden["nodes_u"])
    assert o.ccell == int(golden["ccell"])
    for k in ("u", "v", "w"):
        assert np.allclose(getattr(o, k), golden["nodes_" + k], rtol=0, atol=1e-14)
    assert np.allclose(o.gwts, golden["nodes_gwts"], rtol=1e-13, atol=0)
    # weights integrate 1 over the box exactly
    assert abs(o.gwts.sum() - (2 * float(golden["L"])) ** 3) < 1e-12


@pytest.mark.parametrize("M,expect", [(5, (2, 2, 2)), (4, (2, 2, 2)), (2, (1, 1, 1))])
def test_canonical_cell_ties_go_right(M, expect):
    """v=0 on a grid line belongs to the cell to its right (finduiviwi's
    `u >= ugrid(ui) - eps` loop, dgvtools_mod.f90:312-315)."""
    o = Oracle(2, M, 3.0)
    cu, cv, cw = expect
    assert o.ccell == (cu * M + cv) * M + cw


def test_shift_tables_match_golden(golden):
    o = golden_oracle(golden)
    t = o.shift_tables()
    assert np.array_equal(t["Ashift"], golden["Ashift"])
    assert np.array_equal(t["phican"], golden["phican"])
    assert np.array_equal(t["dui"], golden["dui"])


def test_q_matches_golden(golden):
    o = golden_oracle(golden)
    q = o.collide(golden["f0"])
    assert rel_err(q, golden["q0"]) < 1e-13
    assert max_rel_err(q, golden["q0"]) < 1e-13


def test_three_q_routines_agree(golden):
    """APlus (collision_mod.f90:143-229) == A-variant (:29-129); IphiDGV
    (dgvtools_mod.f90:847-877) equals Q on canonical-cell nodes."""
    o = golden_oracle(golden)
    f = golden["f0"]
    q = o.collide(f)
    assert max_rel_err(o.collide_a(f), q) < 1e-14
    can = np.arange(o.ccell * o.P, (o.ccell + 1) * o.P)
    assert max_rel_err(o.iphi(f)[can], q[can]) < 1e-14


def test_node_subset_evaluation(golden):
    o = golden_oracle(golden)
    f = golden["f0"]
    q = o.collide(f)
    sub = np.array([0, 5, 17, 100, 215])
    qs = o.collide(f, nodes=sub)
    assert np.array_equal(qs[sub], q[sub])


def test_mixed_terms_and_linear_operator(golden):
    o = golden_oracle(golden)
    f, fm = golden["f0"], golden["fm"]
    df = f - fm
    mt = o.mixed_terms(df, fm)
    assert rel_err(mt, golden["mixed"]) < 1e-13
    fmA = o.prepare_fma(fm)
    assert rel_err(o.eval_linear(fmA, df), mt) < 1e-13


def test_vjp_is_transpose_of_linear_operator(golden):
    """J = dQ/df at fm has J[i,k] = 2 fmA(k,i) (collision_mod.f90:357)."""
    o = golden_oracle(golden)
    fm = golden["fm"]
    rng = np.random.default_rng(3)
    v = rng.standard_normal(o.N)
    fmA = o.prepare_fma(fm)          # row i holds column i of the Fortran array
    J = 2.0 * fmA                    # J[i, k]
    assert rel_err(o.vjp(fm, v), J.T @ v) < 1e-13


def test_vjp_central_difference(golden):
    o = golden_oracle(golden)
    f = golden["f0"]
    rng = np.random.default_rng(4)
    v = rng.standard_normal(o.N)
    dfd = rng.standard_normal(o.N)
    eps = 1e-6
    fd = (v @ o.collide(f + eps * dfd) - v @ o.collide(f - eps * dfd)) / (2 * eps)
    assert abs(o.vjp(f, v) @ dfd - fd) <= 1e-8 * max(1.0, abs(fd))


def test_time_integrators_match_golden(golden):
    o = golden_oracle(golden)
    dt = float(golden["dt"])
    f = golden["f0"].copy()
    for k in range(3):
        f, _ = o.rk_step(f, dt, 2)
        assert rel_err(f, golden["rk2_traj"][k]) < 1e-14
    f4, _ = o.rk_step(golden["f0"], dt, 4)
    assert rel_err(f4, golden["rk4_1"]) < 1e-14
    f, hist = o.prepare_ab(golden["f0"], dt, 2)
    for k in range(2):
        f, hist = o.ab_step(f, hist, dt, 2)
        assert rel_err(f, golden["ab2_traj"][k]) < 1e-14


@pytest.mark.parametrize("order", [1, 3, 5])
def test_rk_orders_converge(golden, order):
    """Halving dt reduces the one-step error like dt^(order+1)."""
    o = golden_oracle(golden)
    f0 = golden["f0"]

    def step(dt):
        f, _ = o.rk_step(f0, dt, order)
        return f

    ref = f0.copy()
    for _ in range(16):
        ref, _ = o.rk_step(ref, 0.2 / 16, 5)
    e1 = np.linalg.norm(step(0.2) - ref)
    half = f0.copy()
    for _ in range(2):
        half, _ = o.rk_step(half, 0.1, order)
    e2 = np.linalg.norm(half - ref)
    assert e2 < e1


def test_ab_orders_start_up(golden):
    o = golden_oracle(golden)
    dt = float(golden["dt"])
    for order in range(1, 6):
        f, hist = o.prepare_ab(golden["f0"], dt, order)
        f, hist = o.ab_step(f, hist, dt, order)
        assert np.all(np.isfinite(f))


def test_moments_and_maxwellian(golden):
    o = golden_oracle(golden)
    assert np.allclose(o.moments(golden["f0"]), golden["moments0"], rtol=1e-13, atol=1e-15)
    fm = o.maxwellian(0.7, 0.0, 0.0, 0.0, 1.0)
    assert rel_err(fm, golden["fm"]) < 1e-14


def test_projection_removes_invariant_moments(golden):
    o = golden_oracle(golden)
    q = o.collide(golden["f0"])
    qp = o.project(q)
    psi = [np.ones(o.N), o.u, o.v, o.w, o.u ** 2 + o.v ** 2 + o.w ** 2]
    for p in psi:
        scale = np.sum(np.abs(o.gwts * p * q))
        assert abs(np.sum(o.gwts * p * qp)) <= 1e-13 * scale
    # projecting twice changes nothing
    assert rel_err(o.project(qp), qp) < 1e-14


def test_synthetic_records_match_golden(golden):
    o = Oracle(int(golden["s"]), int(golden["M"]), float(golden["L"]))
    capphi, A, xi, xi1 = o.synth_A(seed=int(golden["seed"]), support=1)
    assert np.array_equal(capphi, golden["capphi"])
    assert np.array_equal(xi + 1, golden["A_xi"]) and np.array_equal(xi1 + 1, golden["A_xi1"])
    assert max_rel_err(A, golden["A"]) < 1e-13


def test_synthetic_structure_is_p_independent_and_subset_of_prefilter():
    o = Oracle(2, 3, 3.0)
    c1, A1, x1, y1 = o.synth_A(seed=5, support=1)
    c0, A0, x0, y0 = o.synth_A(seed=5, support=0)
    n1 = c1[o.ccell * o.P]
    assert np.all(c1[o.ccell * o.P:(o.ccell + 1) * o.P] == n1)
    s1 = set(zip(x1[:n1], y1[:n1]))
    s0 = set(zip(x0[:c0[o.ccell * o.P]], y0[:c0[o.ccell * o.P]]))
    assert s1 < s0
    # every record has xi < xi1 (SetA_DGV's i3 = i2+1..ni)
    assert np.all(x1 < y1)


@pytest.mark.parametrize("mode", [1, 2, 3, 4, 5])
def test_seta_collision_invariant_known_answer(mode):
    """With phi replaced by a collision invariant the SetA integrand
    phi(xi')+phi(xi1')-phi(xi)-phi(xi1) vanishes (dgvtools_mod.f90:267-274,
    972-973): every A-record must be ~0."""
    o = Oracle(2, 2, 3.0)
    i1 = o.ccell * o.P + 3
    rng = np.random.default_rng(mode)
    pairs = rng.integers(0, o.N, size=(12, 2))
    for i2, i3 in pairs:
        if i2 == i3:
            continue
        val = o.seta_pair_integral(i1, int(min(i2, i3)), int(max(i2, i3)), 1e-5, 1e-5, mode)
        assert abs(val) < 1e-10


def test_seta_lagrange_basis_is_nonzero_and_partition_of_unity():
    """With the Lagrange basis restored the integrals are O(1); the sum over
    the canonical cell's basis functions equals the integral for the cell's
    indicator function (partition of unity, Lagrange interpolation of 1)."""
    o = Oracle(2, 2, 3.0)
    i2, i3 = 0, o.N - 1
    vals = [o.seta_pair_integral(o.ccell * o.P + p, i2, i3, 1e-6, 1e-6, 0) for p in range(o.P)]
    assert max(abs(v) for v in vals) > 1e-3

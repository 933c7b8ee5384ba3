"""Parity of the sm_100a path (through the C-ABI) with the oracle and the golden
vectors.  Tolerances: plain FP64 path <= 1e-12 norm-wise and max-relative
against FP64 references; FP32-compensated path <= 1e-6 norm-wise."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, max_rel_err, rel_err
from helpers import golden_oracle, mixture_vdf

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-6


@pytest.fixture(scope="module")
def dgv():
    import dgv0d3v_direct_collision_b200 as m
    return m


@pytest.fixture(scope="module")
def gsolver(dgv, golden):
    s = dgv.DGVSolver(int(golden["s"]), int(golden["M"]), float(golden["L"]), kappa=float(golden["kappa"]))
    s.load_A(golden["capphi"], golden["A"], golden["A_xi"], golden["A_xi1"], one_based=True)
    return s


@pytest.fixture(scope="module")
def c1():
    """The 15^3 grid (s=3, M=5, [-6,6]^3) with seeded synthetic A on both sides."""
    import dgv0d3v_direct_collision_b200 as m
    from oracle.oracle import Oracle
    o = Oracle(3, 5, 6.0)
    cap, A, xi, xi1 = o.synth_A(seed=11, support=1)
    o.set_A(cap, A, xi, xi1)
    s = m.DGVSolver(3, 5, 6.0)
    s.generate_synthetic_A(seed=11, support=1)
    f = o.maxwellian(1.0, 1.5, 0, 0, 0.5) + o.maxwellian(1.0, -1.5, 0, 0, 0.5)
    return {"oracle": o, "solver": s, "f": f, "ref": (cap, A, xi, xi1)}


def test_grid_identical_to_oracle(dgv):
    from oracle.oracle import Oracle
    for args in [(3, 5, 6.0), (2, 3, 3.0), (3, 9, 7.0)]:
        o = Oracle(*args)
        s = dgv.DGVSolver(*args)
        assert s.ccell == o.ccell
        for a, b in [(s.nodes_u, o.u), (s.nodes_v, o.v), (s.nodes_w, o.w), (s.nodes_gwts, o.gwts)]:
            assert np.array_equal(a, b)


def test_q_golden_f64(gsolver, golden):
    q = gsolver.EvalCollisionPeriodicAPlus_DGV(golden["f0"])
    assert rel_err(q, golden["q0"]) < TOL64
    assert max_rel_err(q, golden["q0"]) < TOL64


def test_q_golden_f32c(gsolver, golden):
    q = gsolver.EvalCollisionPeriodicAPlus_DGV(golden["f0"], precision="f32c")
    assert rel_err(q, golden["q0"]) < TOL32


def test_spatial_oper(gsolver, golden):
    dt = 0.37
    fcol = gsolver.SpatialOperSH_DGV(golden["f0"], dt)
    assert rel_err(fcol, golden["q0"] * (float(golden["kappa"]) * dt)) < TOL64


def test_rk_and_ab_trajectories_golden(gsolver, golden):
    dt = float(golden["dt"])
    f = golden["f0"].copy()
    for k in range(3):  # call 1 eager, call 2 captures a CUDA graph, call 3 replays it
        gsolver.TimeIntegratorORK_SH_DGV(f, dt, order=2)
        assert rel_err(f, golden["rk2_traj"][k]) < TOL64
    f = golden["f0"].copy()
    gsolver.TimeIntegratorORK_SH_DGV(f, dt, order=4)
    assert rel_err(f, golden["rk4_1"]) < TOL64
    f = golden["f0"].copy()
    gsolver.PrepareMTS_SH_DGV(f, dt, order=2)
    for k in range(2):
        gsolver.TimeIntegratorMTS_SH_DGV(f, dt)
        assert rel_err(f, golden["ab2_traj"][k]) < TOL64


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_rk_orders_vs_oracle(gsolver, golden, order):
    o = golden_oracle(golden)
    dt = 0.05
    f_ref, r_ref = o.rk_step(golden["f0"], dt, order, kappa=float(golden["kappa"]))
    f = golden["f0"].copy()
    r = gsolver.TimeIntegratorORK_SH_DGV(f, dt, order=order)
    assert rel_err(f, f_ref) < TOL64
    assert rel_err(r, r_ref) < TOL64


@pytest.mark.parametrize("order", [1, 3, 4, 5])
def test_ab_orders_vs_oracle(gsolver, golden, order):
    o = golden_oracle(golden)
    dt = 0.02
    f_ref, hist = o.prepare_ab(golden["f0"], dt, order)
    f = golden["f0"].copy()
    gsolver.PrepareMTS_SH_DGV(f, dt, order=order)
    assert rel_err(f, f_ref) < TOL64
    for _ in range(3):
        f_ref, hist = o.ab_step(f_ref, hist, dt, order)
        gsolver.TimeIntegratorMTS_SH_DGV(f, dt)
        assert rel_err(f, f_ref) < TOL64


def test_jvp_and_linear_operator_golden(gsolver, golden):
    df = golden["f0"] - golden["fm"]
    mt = gsolver.EvalCollisionPeriodicMixedTermsA_DGV(df, golden["fm"])
    assert rel_err(mt, golden["mixed"]) < TOL64
    gsolver.PrepareFMA_DGV(golden["fm"])
    assert rel_err(gsolver.EvalCollisionLinear(df), golden["mixed"]) < TOL64


def test_vjp_vs_oracle_and_fd(gsolver, golden):
    o = golden_oracle(golden)
    rng = np.random.default_rng(7)
    v = rng.standard_normal(o.N)
    f = golden["f0"]
    g = gsolver.vjp(f, v)
    assert rel_err(g, o.vjp(f, v)) < TOL64
    d = rng.standard_normal(o.N)
    eps = 1e-6
    fd = (v @ o.collide(f + eps * d) - v @ o.collide(f - eps * d)) / (2 * eps)
    assert abs(g @ d - fd) <= 1e-8 * max(1.0, abs(fd))


def test_two_input_calls_first_on_a_fresh_context(dgv, golden):
    """VJP and JVP stage two host arrays; as the first call on a new context
    the staging buffer grows while they are staged."""
    o = golden_oracle(golden)
    rng = np.random.default_rng(11)
    f, v = golden["f0"], rng.standard_normal(o.N)
    for which in ("vjp", "jvp"):
        s = dgv.DGVSolver(int(golden["s"]), int(golden["M"]), float(golden["L"]), kappa=float(golden["kappa"]))
        s.load_A(golden["capphi"], golden["A"], golden["A_xi"], golden["A_xi1"], one_based=True)
        if which == "vjp":
            assert rel_err(s.vjp(f, v), o.vjp(f, v)) < TOL64
        else:
            assert rel_err(s.jvp(f, v), o.mixed_terms(f, v)) < TOL64


def test_vjp_equals_linearized_operator_at_maxwellian(gsolver, golden):
    """J^T v at fm equals 2 fmA v, the reference's linearized operator
    (collision_mod.f90:448-449, 357), within 1e-8."""
    o = golden_oracle(golden)
    fm = golden["fm"]
    rng = np.random.default_rng(8)
    v = rng.standard_normal(o.N)
    fmA = o.prepare_fma(fm)
    assert rel_err(gsolver.vjp(fm, v), 2.0 * fmA.T @ v) < 1e-8


def test_moments_maxwellian(gsolver, golden):
    o = golden_oracle(golden)
    m = np.array(gsolver.MassCheckRec(golden["f0"]))
    assert np.allclose(m, golden["moments0"], rtol=1e-13, atol=1e-15)
    for args in [(1.0, 0.0, 0.0, 0.0, 1.0), (0.4, 1.2, -0.3, 0.5, 2.0)]:
        assert rel_err(gsolver.maxwelveldist(*args), o.maxwellian(*args)) < 1e-14


def test_projection(gsolver, golden):
    o = golden_oracle(golden)
    q = gsolver.EvalCollisionPeriodicAPlus_DGV(golden["f0"])
    qp = gsolver.project(q.copy())
    assert rel_err(qp, o.project(q)) < 1e-13
    psi = [np.ones(o.N), o.u, o.v, o.w, o.u ** 2 + o.v ** 2 + o.w ** 2]
    for p in psi:
        assert abs(np.sum(o.gwts * p * qp)) <= 1e-12 * np.sum(np.abs(o.gwts * p * q))
    gsolver.set_projection(True)
    try:
        q2 = gsolver.EvalCollisionPeriodicAPlus_DGV(golden["f0"])
    finally:
        gsolver.set_projection(False)
    assert rel_err(q2, qp) < 1e-14


def test_batched_equals_single(gsolver, golden):
    rng = np.random.default_rng(9)
    o = golden_oracle(golden)
    fs = np.stack([mixture_vdf(o.u, o.v, o.w, rng, normalise_w=o.gwts) for _ in range(5)])
    qb = gsolver.EvalCollisionPeriodicAPlus_DGV(fs)
    for k in range(5):
        assert max_rel_err(qb[k], o.collide(fs[k])) < TOL64
    qb32 = gsolver.EvalCollisionPeriodicAPlus_DGV(fs, precision="f32c")
    for k in range(5):
        assert rel_err(qb32[k], qb[k]) < TOL32


def test_chunk_count_does_not_change_results(gsolver, golden):
    q0 = gsolver.EvalCollisionPeriodicAPlus_DGV(golden["f0"])
    for n in (1, 3, 64):
        gsolver.set_nchunks(n)
        q = gsolver.EvalCollisionPeriodicAPlus_DGV(golden["f0"])
        assert max_rel_err(q, q0) < 1e-14
    gsolver.set_nchunks(0)


def test_torch_device_tensors(gsolver, golden):
    torch = pytest.importorskip("torch")
    f = torch.tensor(golden["f0"], dtype=torch.float64, device="cuda")
    q = gsolver.EvalCollisionPeriodicAPlus_DGV(f)
    assert isinstance(q, torch.Tensor) and q.is_cuda
    assert rel_err(q.cpu().numpy(), golden["q0"]) < TOL64
    ft = f.clone()
    gsolver.TimeIntegratorORK_SH_DGV(ft, float(golden["dt"]), order=2)
    assert rel_err(ft.cpu().numpy(), golden["rk2_traj"][0]) < TOL64


def test_errors_are_reported_not_fatal(dgv, golden):
    s = dgv.DGVSolver(2, 3, 3.0)
    with pytest.raises(dgv.DGVError) as e:
        s.EvalCollisionPeriodicAPlus_DGV(golden["f0"])
    assert e.value.code == 6  # DGV_ESTATE: no A-arrays
    bad_xi = golden["A_xi"].copy()
    bad_xi[3] = 10 ** 6
    with pytest.raises(dgv.DGVError) as e:
        s.load_A(golden["capphi"], golden["A"], bad_xi, golden["A_xi1"])
    assert e.value.code == 2  # DGV_ERANGE
    cap = golden["capphi"].copy()
    cap[0] += 1
    with pytest.raises(dgv.DGVError) as e:
        s.load_A(cap, golden["A"], golden["A_xi"], golden["A_xi1"])
    assert e.value.code == 1  # DGV_EINVAL
    with pytest.raises(dgv.DGVError):
        s.TimeIntegratorMTS_SH_DGV(golden["f0"].copy(), 0.01)  # no start-up yet
    with pytest.raises(dgv.DGVError):
        s.TimeIntegratorORK_SH_DGV(golden["f0"].copy(), 0.01, order=6)
    # the context stays usable after the errors
    s.load_A(golden["capphi"], golden["A"], golden["A_xi"], golden["A_xi1"])
    assert rel_err(s.EvalCollisionPeriodicAPlus_DGV(golden["f0"]), golden["q0"]) < TOL64


def test_export_round_trip(gsolver, golden):
    cap, A, xi, xi1 = gsolver.export_A()
    ref = sorted(zip(np.repeat(np.arange(len(golden["capphi"])), golden["capphi"]),
                     golden["A_xi"] - 1, golden["A_xi1"] - 1, golden["A"]))
    got = sorted(zip(np.repeat(np.arange(len(cap)), cap), xi, xi1, A))
    assert len(ref) == len(got)
    for a, b in zip(ref, got):
        assert a[:3] == b[:3] and a[3] == b[3]


# --- the 15^3 configuration (s=3, M=5, [-6,6]^3, N=3375) --------------------
def test_synthetic_layout_matches_oracle(c1):
    s, (cap, A, xi, xi1) = c1["solver"], c1["ref"]
    info = s.A_info()
    assert info["records"] == len(A)
    cap2, A2, xi2, xi12 = s.export_A()
    assert np.array_equal(cap2, cap)
    P, ccell = s.P, s.ccell
    for p in (0, 13, 26):
        k = ccell * P + p
        lo = int(cap[:k].sum())
        r = np.lexsort((xi1[lo:lo + cap[k]], xi[lo:lo + cap[k]]))
        lo2 = int(cap2[:k].sum())
        r2 = np.lexsort((xi12[lo2:lo2 + cap2[k]], xi2[lo2:lo2 + cap2[k]]))
        assert np.array_equal(xi[lo:][r], xi2[lo2:][r2])
        assert np.array_equal(xi1[lo:][r], xi12[lo2:][r2])
        assert np.array_equal(A[lo:][r], A2[lo2:][r2])  # bit-identical values


def test_q_15cubed_f64_and_f32c(c1):
    o, s, f = c1["oracle"], c1["solver"], c1["f"]
    q_ref = o.collide(f)
    q = s.EvalCollisionPeriodicAPlus_DGV(f)
    assert rel_err(q, q_ref) < TOL64
    assert max_rel_err(q, q_ref) < TOL64
    q32 = s.EvalCollisionPeriodicAPlus_DGV(f, precision="f32c")
    assert rel_err(q32, q_ref) < TOL32


def test_rk2_step_15cubed(c1):
    o, s, f = c1["oracle"], c1["solver"], c1["f"]
    f_ref, _ = o.rk_step(f, 0.01, 2)
    g = f.copy()
    s.TimeIntegratorORK_SH_DGV(g, 0.01, order=2)
    assert rel_err(g, f_ref) < TOL64


def test_load_A_reference_layout_15cubed(c1, dgv):
    """The drop-in upload of reference-layout arrays (1-based) gives the same Q
    as the device generator."""
    cap, A, xi, xi1 = c1["ref"]
    s = dgv.DGVSolver(3, 5, 6.0)
    s.load_A(cap, A, xi + 1, xi1 + 1, one_based=True)
    q = s.EvalCollisionPeriodicAPlus_DGV(c1["f"])
    q2 = c1["solver"].EvalCollisionPeriodicAPlus_DGV(c1["f"])
    assert max_rel_err(q, q2) < 1e-14


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLDEN, "physA_s2M2.npz")),
                    reason="physical A fixture not generated")
def test_physical_A_parity_and_conservation(dgv):
    from oracle.oracle import Oracle
    d = dict(np.load(os.path.join(GOLDEN, "physA_s2M2.npz")))
    o = Oracle(int(d["s"]), int(d["M"]), float(d["L"]))
    o.set_A(d["capphi"], d["A"], d["A_xi"], d["A_xi1"], one_based=True)
    s = dgv.DGVSolver(int(d["s"]), int(d["M"]), float(d["L"]))
    s.load_A(d["capphi"], d["A"], d["A_xi"], d["A_xi1"], one_based=True)
    f = o.maxwellian(0.3, 0.2, 0.0, -0.1, 1.0) + o.maxwellian(0.25, -0.4, 0.3, 0.0, 0.5)
    q_ref = o.collide(f)
    q = s.EvalCollisionPeriodicAPlus_DGV(f)
    assert rel_err(q, q_ref) < TOL64
    s.set_projection(True)
    qp = s.EvalCollisionPeriodicAPlus_DGV(f, precision="f32c")
    s.set_projection(False)
    for p in [np.ones(o.N), o.u, o.v, o.w, o.u ** 2 + o.v ** 2 + o.w ** 2]:
        assert abs(np.sum(o.gwts * p * qp)) <= 1e-12 * np.sum(np.abs(o.gwts * p * q))
    assert rel_err(qp, o.project(q_ref)) < TOL32

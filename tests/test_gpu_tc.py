"""Parity of the chunk form of the tensor-core collision path (DGV_PREC_TC
with DGV_OPT_TCFORM = 1: products per pair on the CUDA cores, tcgen05 with
split-fp16 operands) with the oracle, the golden vectors and the FP64 device
path.  The block form (the default) is covered in test_gpu_tc2.py.
Tolerance: 1e-6 norm-wise relative error, the bound the batched
reduced-precision path is held to."""
import numpy as np
import pytest

from conftest import max_rel_err, rel_err
from helpers import mixture_vdf

pytestmark = pytest.mark.gpu

TOLTC = 1e-6


@pytest.fixture(scope="module")
def dgv():
    import dgv0d3v_direct_collision_b200 as m
    return m


@pytest.fixture(scope="module")
def gsolver(dgv, golden):
    s = dgv.DGVSolver(int(golden["s"]), int(golden["M"]), float(golden["L"]), kappa=float(golden["kappa"]))
    s.load_A(golden["capphi"], golden["A"], golden["A_xi"], golden["A_xi1"], one_based=True)
    s.set_tc_form(1)
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
    s.set_tc_form(1)
    return {"oracle": o, "solver": s}


def test_tc_golden(gsolver, golden):
    q = gsolver.EvalCollisionPeriodicAPlus_DGV(golden["f0"], precision="tc")
    assert rel_err(q, golden["q0"]) < TOLTC


def test_tc_15cubed_vs_oracle(c1):
    o, s = c1["oracle"], c1["solver"]
    f = o.maxwellian(1.0, 1.5, 0, 0, 0.5) + o.maxwellian(1.0, -1.5, 0, 0, 0.5)
    q_ref = o.collide(f)
    q = s.EvalCollisionPeriodicAPlus_DGV(f, precision="tc")
    assert rel_err(q, q_ref) < TOLTC


@pytest.mark.parametrize("nb", [37, 150])
def test_tc_batched_ragged(c1, nb):
    """Batches that are not a multiple of the VDF tile (37: tiles of 64 VDFs
    x 2 cells; 150: tiles of 128 VDFs x 1 cell), each VDF with its own scale
    (densities over four decades), against the FP64 device path."""
    o, s = c1["oracle"], c1["solver"]
    rng = np.random.default_rng(5)
    fs = np.stack([mixture_vdf(o.u, o.v, o.w, rng, normalise_w=o.gwts) * 10.0 ** rng.uniform(-2, 2)
                   for _ in range(nb)])
    q64 = s.EvalCollisionPeriodicAPlus_DGV(fs)
    qtc = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    for k in range(fs.shape[0]):
        assert rel_err(qtc[k], q64[k]) < TOLTC, k
    # one VDF alone (tiles of 32 VDFs x 4 cells) agrees with its batched result
    q1 = s.EvalCollisionPeriodicAPlus_DGV(fs[3], precision="tc")
    assert rel_err(q1, q64[3]) < TOLTC


def test_tc_conservation_with_projection(c1):
    o, s = c1["oracle"], c1["solver"]
    rng = np.random.default_rng(9)
    f = mixture_vdf(o.u, o.v, o.w, rng, normalise_w=o.gwts)
    q = s.EvalCollisionPeriodicAPlus_DGV(f)
    s.set_projection(True)
    try:
        qp = s.EvalCollisionPeriodicAPlus_DGV(f, precision="tc")
    finally:
        s.set_projection(False)
    for p in [np.ones(o.N), o.u, o.v, o.w, o.u ** 2 + o.v ** 2 + o.w ** 2]:
        assert abs(np.sum(o.gwts * p * qp)) <= 1e-12 * np.sum(np.abs(o.gwts * p * q))
    assert rel_err(qp, o.project(q)) < TOLTC


def test_tc_rk2_step(c1):
    o, s = c1["oracle"], c1["solver"]
    f = o.maxwellian(1.0, 1.5, 0, 0, 0.5) + o.maxwellian(1.0, -1.5, 0, 0, 0.5)
    f_ref, _ = o.rk_step(f, 0.01, 2)
    g = f.copy()
    s.TimeIntegratorORK_SH_DGV(g, 0.01, order=2, precision="tc")
    assert rel_err(g - f, f_ref - f) < TOLTC


def test_tc_rejects_more_than_32_nodes_per_cell(dgv):
    s = dgv.DGVSolver(4, 3, 3.0)  # 64 nodes per cell
    cap = np.zeros(s.N, np.int32)
    k0 = s.ccell * s.P
    cap[k0] = 1
    s.load_A(cap, np.array([0.5]), np.array([k0 + 1], np.int32), np.array([k0 + 2], np.int32), one_based=True)
    with pytest.raises(dgv.DGVError):
        s.EvalCollisionPeriodicAPlus_DGV(np.ones(s.N), precision="tc")
    assert s.A_info()["records"] == 1  # the context stays usable

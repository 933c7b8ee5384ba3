"""Parity of the block form of the tensor-core path (DGV_OPT_TCFORM = 2:
G = f(c2) W on the tensor core, contraction with f(c1) on the CUDA cores)
with the oracle, the golden vectors, the FP64 device path and the chunk form.
Tolerance: 1e-6 norm-wise relative error, as for the chunk form."""
import numpy as np
import pytest

from conftest import rel_err
from helpers import mixture_vdf

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
    s.set_tc_form(2)
    return {"oracle": o, "solver": s}


def test_tc2_golden(golden):
    import dgv0d3v_direct_collision_b200 as m
    s = m.DGVSolver(int(golden["s"]), int(golden["M"]), float(golden["L"]), kappa=float(golden["kappa"]))
    s.load_A(golden["capphi"], golden["A"], golden["A_xi"], golden["A_xi1"], one_based=True)
    s.set_tc_form(2)  # s = 2: 8 nodes per cell, one column group
    q = s.EvalCollisionPeriodicAPlus_DGV(golden["f0"], precision="tc")
    assert rel_err(q, golden["q0"]) < TOLTC


def test_tc2_15cubed_vs_oracle(c1):
    o, s = c1["oracle"], c1["solver"]
    f = o.maxwellian(1.0, 1.5, 0, 0, 0.5) + o.maxwellian(1.0, -1.5, 0, 0, 0.5)
    q = s.EvalCollisionPeriodicAPlus_DGV(f, precision="tc")
    assert rel_err(q, o.collide(f)) < TOLTC


@pytest.mark.parametrize("nb", [37, 150, 300])
def test_tc2_batched_ragged(c1, nb):
    """37: tiles of 64 VDFs x 2 cells, one tile; 150: two tiles of 128 (one
    pair); 300: three tiles (the second CTA of a row tile has one); densities
    over four decades; against the FP64 device path and the chunk form."""
    o, s = c1["oracle"], c1["solver"]
    rng = np.random.default_rng(5)
    fs = np.stack([mixture_vdf(o.u, o.v, o.w, rng, normalise_w=o.gwts) * 10.0 ** rng.uniform(-2, 2)
                   for _ in range(nb)])
    q64 = s.EvalCollisionPeriodicAPlus_DGV(fs)
    q2 = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    s.set_tc_form(1)
    try:
        q1 = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    finally:
        s.set_tc_form(2)
    for k in range(nb):
        assert rel_err(q2[k], q64[k]) < TOLTC, k
        assert rel_err(q2[k], q1[k]) < 2 * TOLTC, k
    # one VDF alone (tiles of 32 VDFs x 4 cells)
    assert rel_err(s.EvalCollisionPeriodicAPlus_DGV(fs[3], precision="tc"), q64[3]) < TOLTC


def test_tc2_projection_and_rk_step(c1):
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
    # RK2 steps through the captured graph (eager, capture, replay)
    import torch
    g = torch.from_numpy(f.copy()).cuda()
    ref = f.copy()
    for _ in range(3):
        ref, _ = o.rk_step(ref, 0.01, 2)
        s.TimeIntegratorORK_SH_DGV(g, 0.01, order=2, precision="tc")
        assert rel_err(g.cpu().numpy() - f, ref - f) < TOLTC


def test_tc2_one_tile_per_cta(c1):
    """DGV_OPT_TCTILES = 1: each CTA serves one VDF tile with two alternating
    accumulators; same results as two tiles per CTA."""
    o, s = c1["oracle"], c1["solver"]
    rng = np.random.default_rng(17)
    fs = np.stack([mixture_vdf(o.u, o.v, o.w, rng, normalise_w=o.gwts) for _ in range(150)])
    q2 = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    s.set_tc_tiles_per_cta(1)
    try:
        q1 = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    finally:
        s.set_tc_tiles_per_cta(2)
    q64 = s.EvalCollisionPeriodicAPlus_DGV(fs[:8])
    for k in range(8):
        assert rel_err(q1[k], q64[k]) < TOLTC, k
    assert rel_err(q1, q2) < 1e-9  # same per-row arithmetic, only the CTA split differs


def test_tc_plan_matches_launches(c1):
    """dgv_tc_plan: the launches of one evaluation equal those the kernel
    timer counts, and the issued tensor work exceeds the algorithmic work
    (dense tiles, three split products)."""
    o, s = c1["oracle"], c1["solver"]
    fs = np.stack([o.maxwellian(1.0, 0.3 * k, 0, 0, 0.8) for k in range(40)])
    s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")  # settles the tuned launch choice
    plan = s.tc_plan(40)
    s.set_kernel_timing(True)
    s.kernel_stats(reset=True)
    s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    st = s.kernel_stats(reset=True)
    s.set_kernel_timing(False)
    assert st["launches"] == plan["launches"] > 0
    assert plan["items"] > 0
    assert plan["tensor_flop"] > 3.0 * s.A_info()["record_shifts"] * 40


def test_tc2_launch_size_option(c1):
    """DGV_OPT_TCSETMB: more or fewer block records per launch changes the
    number of launches, not the result."""
    o, s = c1["oracle"], c1["solver"]
    fs = np.stack([o.maxwellian(1.0, 0.2 * k, 0, 0, 0.7) for k in range(20)])
    s.set_tc_persistent(False)  # one launch per set of records
    q48 = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    n48 = s.tc_plan(20)["launches"]
    s.set_tc_set_mb(8)
    try:
        q8 = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
        n8 = s.tc_plan(20)["launches"]
    finally:
        s.set_tc_set_mb(48)
    assert n8 > n48
    assert rel_err(q8, q48) < 1e-10  # only the grouping of compensated partial sums differs


def test_tc2_autotuned_launch_choice():
    """The first evaluation of a batch class times VDF tiles per CTA x records
    per launch and keeps the fastest; the results equal those of the fixed
    default choice (only the grouping of compensated partial sums differs)."""
    import dgv0d3v_direct_collision_b200 as m
    from dgv0d3v_direct_collision_b200 import _lib
    s = m.DGVSolver(3, 5, 6.0)
    s.generate_synthetic_A(seed=11, support=1)
    rng = np.random.default_rng(23)
    fs = np.stack([mixture_vdf(s.nodes_u, s.nodes_v, s.nodes_w, rng, normalise_w=s.nodes_gwts) for _ in range(150)])
    q_tuned = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    q_again = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    assert np.array_equal(q_tuned, q_again)  # the choice is kept: same launches, same sums
    L = _lib.load()
    assert L.dgv_set_option(s._h, _lib.DGV_OPT_TCAUTOTUNE, 0) == 0
    q_fixed = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    assert rel_err(q_tuned, q_fixed) < 1e-10
    s.close()

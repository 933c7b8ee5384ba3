"""Run modes of SpatialOperSH_DGV (spat_oper_mod.f90:28-68) chosen by
CheckSolutionMode_DGV (:195-272), device against the oracle: the same
sequence of VDFs -- far from, near and very near their local Maxwellian --
drives both state machines through modes 0 -> 1 -> 2 -> 1 -> 0, and an RK2
trajectory with the modes on matches step by step.  Physical A-arrays of the
s=2, M=2 grid (fixture made by the oracle's SetA)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err

pytestmark = pytest.mark.gpu

FIX = os.path.join(GOLDEN, "physA_s2M2.npz")


@pytest.fixture(scope="module")
def sides():
    import dgv0d3v_direct_collision_b200 as dgv
    from oracle.oracle import Oracle
    d = dict(np.load(FIX))
    o = Oracle(int(d["s"]), int(d["M"]), float(d["L"]))
    o.set_A(d["capphi"], d["A"], d["A_xi"], d["A_xi1"], one_based=True)
    s = dgv.DGVSolver(int(d["s"]), int(d["M"]), float(d["L"]), kappa=0.7)
    s.load_A(d["capphi"], d["A"], d["A_xi"], d["A_xi1"], one_based=True)
    fm = o.maxwellian(0.6, 0.1, 0.0, 0.0, 1.0)
    bump = o.maxwellian(0.3, -0.8, 0.4, 0.0, 1.0)
    vdfs = {"far": fm + 0.8 * bump, "mid": fm + 0.1 * bump, "near": fm + 0.002 * bump}
    l1 = {}
    for k, f in vdfs.items():  # relative L1 distance to the local Maxwellian
        r = o.regime(0.0, 0.0)
        o.spatial_oper_regime(r, f, 0.01)
        l1[k] = r.last_L1
    assert l1["near"] < l1["mid"] < l1["far"]
    levels = (np.sqrt(l1["mid"] * l1["far"]), np.sqrt(l1["near"] * l1["mid"]))
    return o, s, vdfs, levels


@pytest.mark.skipif(not os.path.exists(FIX), reason="fixture missing")
def test_mode_sequence_matches_oracle(sides):
    o, s, vdfs, (decomp, linear) = sides
    reg = o.regime(decomp, linear)
    s.set_regime(decomp, linear)
    seen = []
    for name in ["far", "mid", "near", "near", "mid", "far"]:
        f = vdfs[name]
        ref = o.spatial_oper_regime(reg, f, 0.01, kappa=0.7)
        got = s.SpatialOperSH_DGV(f, 0.01)
        mode, l1 = s.regime_info()
        assert mode == reg.mode, name
        assert abs(l1 - reg.last_L1) <= 1e-12 * reg.last_L1
        assert rel_err(got, ref) < 1e-12, (name, mode)
        seen.append(mode)
    assert seen == [0, 1, 2, 2, 1, 0]
    s.set_regime(0.0, 0.0)
    assert rel_err(s.SpatialOperSH_DGV(vdfs["mid"], 0.01), o.spatial_oper(vdfs["mid"], 0.01, kappa=0.7)) < 1e-12


@pytest.mark.skipif(not os.path.exists(FIX), reason="fixture missing")
def test_rk2_trajectory_with_modes(sides):
    o, s, vdfs, (decomp, linear) = sides
    reg = o.regime(decomp, linear)
    s.set_regime(decomp, linear)
    f_ref = vdfs["mid"].copy()
    f_dev = vdfs["mid"].copy()
    modes = []
    for _ in range(6):
        f_ref, _ = o.rk_step_regime(reg, f_ref, 0.05, 2, kappa=0.7)
        s.TimeIntegratorORK_SH_DGV(f_dev, 0.05, order=2)
        assert s.regime_info()[0] == reg.mode
        assert rel_err(f_dev, f_ref) < 1e-12
        modes.append(reg.mode)
    s.set_regime(0.0, 0.0)
    assert 1 in modes or 2 in modes

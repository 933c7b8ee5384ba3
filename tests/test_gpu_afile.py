"""Operator files through a context: the loaded A-arrays written with
dgv_write_A_file and read into a new context with dgv_read_A_files give the
same Q; so does the chunked form."""
import numpy as np
import pytest

from conftest import max_rel_err, rel_err

pytestmark = pytest.mark.gpu


def test_write_read_round_trip(tmp_path, golden):
    import dgv0d3v_direct_collision_b200 as dgv
    from dgv0d3v_direct_collision_b200.afile import read_A_arrays, write_A_arrays
    mk = lambda: dgv.DGVSolver(int(golden["s"]), int(golden["M"]), float(golden["L"]), kappa=float(golden["kappa"]))
    s = mk()
    s.load_A(golden["capphi"], golden["A"], golden["A_xi"], golden["A_xi1"], one_based=True)
    p = str(tmp_path / "op_Aarrs.dat")
    s.write_A_file(p, max_subrecord=100000)
    t = mk()
    t.read_A_files(p)
    q0 = s.EvalCollisionPeriodicAPlus_DGV(golden["f0"])
    assert max_rel_err(t.EvalCollisionPeriodicAPlus_DGV(golden["f0"]), q0) < 1e-14
    assert rel_err(q0, golden["q0"]) < 1e-12
    # the same operator as two chunk files
    cap, A, xi, xi1 = read_A_arrays(p, s.N)
    h = s.N // 2
    r = int(cap[:h].sum())
    c1, c2 = cap.copy(), cap.copy()
    c1[h:] = 0
    c2[:h] = 0
    write_A_arrays(str(tmp_path / "a_Aarrs.dat"), c1, A[:r], xi[:r], xi1[:r])
    write_A_arrays(str(tmp_path / "b_Aarrs.dat"), c2, A[r:], xi[r:], xi1[r:])
    u = mk()
    u.read_A_files([str(tmp_path / "a_Aarrs.dat"), str(tmp_path / "b_Aarrs.dat")])
    assert max_rel_err(u.EvalCollisionPeriodicAPlus_DGV(golden["f0"]), q0) < 1e-14
    with pytest.raises(dgv.DGVError):
        u.read_A_files(str(tmp_path / "missing_Aarrs.dat"))

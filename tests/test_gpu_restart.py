"""Solution files (WriteSol_DGV / RestartSolutionDGV, readwrite.f90:1756-1796,
2389-2513) on the device: an Adams-Bashforth run is written mid-way, restarted
in a fresh context and continued; it matches the uninterrupted run and the
oracle continuing from the file's f and frhs1..frhs(rkmts-1).  Golden
A-arrays, FP64 path, tolerance 1e-12 norm-wise."""
import numpy as np
import pytest

from conftest import rel_err
from helpers import golden_oracle

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def _solver(golden):
    import dgv0d3v_direct_collision_b200 as dgv
    s = dgv.DGVSolver(int(golden["s"]), int(golden["M"]), float(golden["L"]), kappa=float(golden["kappa"]))
    s.load_A(golden["capphi"], golden["A"], golden["A_xi"], golden["A_xi1"], one_based=True)
    return s


@pytest.mark.parametrize("order", [2, 3, 5])
def test_restart_continues_the_run(golden, tmp_path, order):
    from dgv0d3v_direct_collision_b200.afile import read_solution_arrays, solution_file_name
    dt = 0.02
    a = _solver(golden)
    f = golden["f0"].copy()
    a.PrepareMTS_SH_DGV(f, dt, order=order)
    for _ in range(2):
        a.TimeIntegratorMTS_SH_DGV(f, dt)
    path = str(tmp_path / solution_file_name("golden_", "0.1000"))
    a.WriteSol_DGV(path, f, 0.1, dt)

    sol = read_solution_arrays(path)
    assert sol["rkmts"] == order and sol["e_time"] == 0.1 and sol["dt"] == dt
    np.testing.assert_array_equal(sol["f"], f)

    b = _solver(golden)
    g, t, dtr = b.RestartSolutionDGV(path)
    assert (t, dtr) == (0.1, dt) and b.rkmts == order
    np.testing.assert_array_equal(g, f)

    o = golden_oracle(golden)
    hist = np.zeros(5 * o.N)
    hist[:(order - 1) * o.N] = sol["frhs"].ravel()
    f_ref = sol["f"].copy()
    for _ in range(3):
        a.TimeIntegratorMTS_SH_DGV(f, dt)
        b.TimeIntegratorMTS_SH_DGV(g, dt)
        f_ref, hist = o.ab_step(f_ref, hist, dt, order, kappa=float(golden["kappa"]))
        assert rel_err(g, f) < TOL64
        assert rel_err(g, f_ref) < TOL64


def test_restart_into_device_memory_and_errors(golden, tmp_path):
    import torch

    import dgv0d3v_direct_collision_b200 as dgv
    dt = 0.01
    a = _solver(golden)
    f = golden["f0"].copy()
    a.PrepareMTS_SH_DGV(f, dt, order=3)
    a.TimeIntegratorMTS_SH_DGV(f, dt)
    path = str(tmp_path / "dev_sol.dat")
    fd = torch.from_numpy(f).cuda()
    a.WriteSol_DGV(path, fd, 0.5, dt)  # from device memory

    b = _solver(golden)
    gd = torch.zeros(b.N, dtype=torch.float64, device="cuda")
    b.RestartSolutionDGV(path, gd)  # into device memory
    np.testing.assert_array_equal(gd.cpu().numpy(), f)
    a.TimeIntegratorMTS_SH_DGV(fd, dt)
    b.TimeIntegratorMTS_SH_DGV(gd, dt)
    assert rel_err(gd.cpu().numpy(), fd.cpu().numpy()) < TOL64

    # a file of another grid is refused, as RestartSolutionDGV refuses m /= size(f,1)
    other = dgv.DGVSolver(2, 4, 4.0)  # N = 512, the golden grid has 216
    with pytest.raises(dgv.DGVError):
        other.RestartSolutionDGV(path)
    with pytest.raises(dgv.DGVError):
        b.RestartSolutionDGV(str(tmp_path / "missing_sol.dat"))
    # a context that has not prepared a multistep run writes rkmts = 1
    c = _solver(golden)
    c.WriteSol_DGV(str(tmp_path / "rk_sol.dat"), golden["f0"], 0.0, dt)
    from dgv0d3v_direct_collision_b200.afile import read_solution_arrays
    assert read_solution_arrays(str(tmp_path / "rk_sol.dat"))["rkmts"] == 1

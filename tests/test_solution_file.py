"""The reference's solution files (WriteSol_DGV / RestartSolutionDGV,
readwrite.f90:1756-1796, 2389-2513) through the library's context-free file
routines, on the CPU: a file built byte by byte here (records (e_time, dt),
(rkmts), (N), (f, f1..f(rkmts-1), frhs1..frhs(rkmts-1)), gfortran sequential
framing) is read back, the writer's output is parsed here for every rkmts,
and damaged files are refused."""
import struct

import numpy as np
import pytest

from dgv0d3v_direct_collision_b200 import DGVError
from dgv0d3v_direct_collision_b200.afile import read_solution_arrays, solution_file_name, write_solution_arrays


def _record(payload: bytes):
    return struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload))


def _records(data: bytes):
    out, pos = [], 0
    while pos < len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        assert n >= 0
        out.append(data[pos + 4:pos + 4 + n])
        (t,) = struct.unpack_from("<i", data, pos + 4 + n)
        assert t == n
        pos += n + 8
    return out


def _file_bytes(e_time, dt, arrays):
    k = (len(arrays) + 1) // 2
    N = len(arrays[0])
    return (_record(struct.pack("<dd", e_time, dt)) + _record(struct.pack("<i", k)) + _record(struct.pack("<i", N))
            + _record(b"".join(np.asarray(a, "<f8").tobytes() for a in arrays)))


def test_file_name():
    # trim(Adjustl(base))//"_time"//trim(Adjustl(suff))//"_sol.dat"
    assert solution_file_name("run/mix_", "  0.5000E-01 ") == "run/mix__time0.5000E-01_sol.dat"


@pytest.mark.parametrize("rkmts", [1, 2, 3, 4, 5])
def test_hand_built_file_reads(tmp_path, rkmts):
    rng = np.random.default_rng(rkmts)
    N = 343
    arrays = [rng.standard_normal(N) for _ in range(2 * rkmts - 1)]
    p = tmp_path / "s_sol.dat"
    p.write_bytes(_file_bytes(0.125 * rkmts, 1e-3, arrays))
    s = read_solution_arrays(str(p))
    assert s["rkmts"] == rkmts and s["e_time"] == 0.125 * rkmts and s["dt"] == 1e-3
    np.testing.assert_array_equal(s["f"], arrays[0])
    assert s["f_prev"].shape == (rkmts - 1, N) and s["frhs"].shape == (rkmts - 1, N)
    for j in range(rkmts - 1):
        np.testing.assert_array_equal(s["f_prev"][j], arrays[1 + j])
        np.testing.assert_array_equal(s["frhs"][j], arrays[rkmts + j])


@pytest.mark.parametrize("rkmts", [1, 3, 5])
def test_writer_layout(tmp_path, rkmts):
    rng = np.random.default_rng(10 + rkmts)
    N = 125
    f = rng.standard_normal(N)
    frhs = [rng.standard_normal(N) for _ in range(rkmts - 1)]
    p = tmp_path / "w_sol.dat"
    write_solution_arrays(str(p), f, 2.5, 0.01, frhs=frhs)
    recs = _records(p.read_bytes())
    assert len(recs) == 4
    assert struct.unpack("<dd", recs[0]) == (2.5, 0.01)
    assert struct.unpack("<i", recs[1]) == (rkmts,)
    assert struct.unpack("<i", recs[2]) == (N,)
    body = np.frombuffer(recs[3], "<f8").reshape(2 * rkmts - 1, N)
    np.testing.assert_array_equal(body[0], f)
    np.testing.assert_array_equal(body[1:rkmts], 0.0)  # f1..f4 unused by the multistep formulas
    for j in range(rkmts - 1):
        np.testing.assert_array_equal(body[rkmts + j], frhs[j])


def test_damaged_files_are_refused(tmp_path):
    rng = np.random.default_rng(0)
    arrays = [rng.standard_normal(64) for _ in range(3)]
    good = _file_bytes(1.0, 0.1, arrays)
    cases = {
        "truncated": good[:-20],
        "bad_order": good.replace(_record(struct.pack("<i", 2)), _record(struct.pack("<i", 7)), 1),
        "short_body": _file_bytes(1.0, 0.1, arrays[:2]).replace(_record(struct.pack("<i", 1)),
                                                                  _record(struct.pack("<i", 2)), 1),
        "bad_marker": good[:-4] + struct.pack("<i", 12345),
    }
    for name, data in cases.items():
        p = tmp_path / f"{name}.dat"
        p.write_bytes(data)
        with pytest.raises(DGVError):
            read_solution_arrays(str(p))
    with pytest.raises(DGVError):
        read_solution_arrays(str(tmp_path / "missing.dat"))

"""The reference's operator files (WriteAarraysDGV / ReadAarraysDGV /
ReadAarraysChnksDGV, readwrite.f90:1066-1484) through the library's file
routines, on the CPU: a file written byte by byte here (gfortran sequential
framing) is read back, the writer's output is parsed here, records split into
subrecords round-trip, chunked operators join, and damaged files are refused."""
import struct

import numpy as np
import pytest

from conftest import GOLDEN
from dgv0d3v_direct_collision_b200 import DGVError
from dgv0d3v_direct_collision_b200.afile import aoperator_file_name, read_A_arrays, write_A_arrays


def _record(payload: bytes, maxsub=None):
    """gfortran framing: head < 0 = more subrecords follow, tail < 0 = continuation"""
    if maxsub is None or len(payload) <= maxsub:
        return struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload))
    parts = [payload[i:i + maxsub] for i in range(0, len(payload), maxsub)]
    out = []
    for k, p in enumerate(parts):
        head = -len(p) if k + 1 < len(parts) else len(p)
        tail = -len(p) if k > 0 else len(p)
        out += [struct.pack("<i", head), p, struct.pack("<i", tail)]
    return b"".join(out)


def _file_bytes(cap, A, xi, xi1, maxsub=None):
    phi = np.repeat(np.arange(1, len(cap) + 1, dtype=np.int32), cap)
    body = (np.asarray(cap, "<i4").tobytes() + np.asarray(A, "<f8").tobytes() + np.asarray(xi, "<i4").tobytes()
            + np.asarray(xi1, "<i4").tobytes() + phi.astype("<i4").tobytes())
    return _record(struct.pack("<ii", len(cap), len(A))) + _record(body, maxsub)


@pytest.fixture(scope="module")
def gA(golden):
    return golden["capphi"].astype(np.int32), golden["A"], golden["A_xi"].astype(np.int32), golden["A_xi1"].astype(np.int32)


def test_reads_a_file_written_here(tmp_path, gA):
    cap, A, xi, xi1 = gA
    p = tmp_path / "op_Aarrs.dat"
    p.write_bytes(_file_bytes(cap, A, xi, xi1))
    c2, A2, x2, y2 = read_A_arrays(str(p), len(cap))
    assert np.array_equal(c2, cap) and np.array_equal(A2, A) and np.array_equal(x2, xi) and np.array_equal(y2, xi1)


@pytest.mark.parametrize("maxsub", [0, 4096, 1000, 13])  # 13: ~2e5 subrecords, an odd split
def test_writer_bytes_and_round_trip(tmp_path, gA, maxsub):
    cap, A, xi, xi1 = gA
    p = str(tmp_path / "w_Aarrs.dat")
    write_A_arrays(p, cap, A, xi, xi1, max_subrecord=maxsub)
    raw = open(p, "rb").read()
    assert raw == _file_bytes(cap, A, xi, xi1, maxsub or None)
    c2, A2, x2, y2 = read_A_arrays(p, len(cap))
    assert np.array_equal(c2, cap) and np.array_equal(A2, A) and np.array_equal(x2, xi) and np.array_equal(y2, xi1)


def test_chunked_operator_joins(tmp_path, gA):
    """Chunks cover increasing node ranges; A_capphi of each chunk is zero
    outside its range; reading adds them and concatenates the records."""
    cap, A, xi, xi1 = gA
    N = len(cap)
    ends = np.cumsum(cap)
    starts = ends - cap
    paths = []
    for k, (a, b) in enumerate([(0, N // 3), (N // 3, N // 2), (N // 2, N)]):
        c = np.zeros(N, np.int32)
        c[a:b] = cap[a:b]
        r0, r1 = (starts[a] if a < N else len(A)), (ends[b - 1] if b > 0 else 0)
        p = tmp_path / aoperator_file_name("op", 0, 2, 2, 2, 1, 3, 3, 3, chunk=k)
        p.write_bytes(_file_bytes(c, A[r0:r1], xi[r0:r1], xi1[r0:r1]))
        paths.append(str(p))
    c2, A2, x2, y2 = read_A_arrays(paths, N)
    assert np.array_equal(c2, cap) and np.array_equal(A2, A) and np.array_equal(x2, xi) and np.array_equal(y2, xi1)


def test_file_names_follow_the_reference():
    assert aoperator_file_name("B", 1, 3, 3, 3, 1, 9, 9, 9) == "B1kc3su3sv3sw1NXU9MuUU9MvVU9MwWU_Aarrs.dat"
    assert aoperator_file_name("B", 1, 3, 3, 3, 1, 9, 9, 9, chunk=7, directory="d/") == \
        "d/Bch007_1kc3su3sv3sw1NXU9MuUU9MvVU9MwWU_Aarrs.dat"


def test_damaged_files_are_refused(tmp_path, gA):
    cap, A, xi, xi1 = gA
    good = _file_bytes(cap, A, xi, xi1)
    cases = {
        "truncated": good[:-7],
        "markers": good[:-4] + struct.pack("<i", 12345),
        "wrong_sizes": _record(struct.pack("<ii", len(cap), len(A) + 1)) + good[16:],
    }
    for name, raw in cases.items():
        p = tmp_path / f"{name}_Aarrs.dat"
        p.write_bytes(raw)
        with pytest.raises(DGVError):
            read_A_arrays(str(p), len(cap))
    # records out of node order: A_phi contradicts A_capphi
    bad = bytearray(good)
    phi_off = 8 + 8 + 4 + 4 * len(cap) + 20 * len(A) - 4 * len(A)
    struct.pack_into("<i", bad, phi_off, 2)  # first record claims node 2
    p = tmp_path / "phi_Aarrs.dat"
    p.write_bytes(bytes(bad))
    with pytest.raises(DGVError):
        read_A_arrays(str(p), len(cap))
    with pytest.raises(DGVError):
        read_A_arrays(str(tmp_path / "missing_Aarrs.dat"), len(cap))

"""The reference's A-array files on the host: names and contents.

`aoperator_file_name` builds the names MakeBaseNameAoperDGV /
MakeBaseNameAoperChnksDGV give the operator files (readwrite.f90:2148-2280,
uniform meshes); `read_A_arrays` / `write_A_arrays` read and write their
contents through the library's file routines (no GPU needed).  A context
loads files directly with `DGVSolver.read_A_files`.

`solution_file_name`, `read_solution_arrays` and `write_solution_arrays` do
the same for the solution files of WriteSol_DGV / RestartSolutionDGV
(readwrite.f90:1756-1796, 2389-2513); a context writes and restarts from
them with `DGVSolver.WriteSol_DGV` / `DGVSolver.RestartSolutionDGV`.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def aoperator_file_name(base: str, k_c: int, su: int, sv: int, sw: int, N: int, Mu: int, Mv: int, Mw: int,
                        chunk: int | None = None, directory: str = "") -> str:
    """'<dir><base>[chNNN_]<k_c>kc<su>su<sv>sv<sw>sw<N>NXU<Mu>MuUU<Mv>MvVU<Mw>MwWU_Aarrs.dat'
    (uniform x and velocity meshes; chunk numbers start at 0)."""
    name = directory + base
    if chunk is not None:
        name += "ch%03d_" % chunk
    name += f"{k_c}kc{su}su{sv}sv{sw}sw{N}NXU{Mu}MuUU{Mv}MvVU{Mw}MwWU"
    return name + "_Aarrs.dat"


def solution_file_name(base: str, suff: str) -> str:
    """'<base>_time<suff>_sol.dat' (WriteSol_DGV, readwrite.f90:1768-1769;
    base is what MakeBaseNameDGV builds for the run)."""
    return base.strip() + "_time" + suff.strip() + "_sol.dat"


def read_solution_arrays(path: str) -> dict:
    """e_time, dt, rkmts, f, f_prev (f1..f(rkmts-1)) and frhs
    (frhs1..frhs(rkmts-1)) of a solution file."""
    L = _lib.load()
    N = C.c_int32(); r = C.c_int32(); t = C.c_double(); dt = C.c_double()
    if L.dgv_read_solution_arrays(path.encode(), C.byref(N), C.byref(r), C.byref(t), C.byref(dt), None):
        raise _lib.DGVError(_lib.DGV_EINVAL, L.dgv_file_error().decode())
    arr = np.zeros((2 * r.value - 1, N.value))
    if L.dgv_read_solution_arrays(path.encode(), None, None, None, None, arr.ctypes.data_as(C.c_void_p)):
        raise _lib.DGVError(_lib.DGV_EINVAL, L.dgv_file_error().decode())
    k = r.value
    return {"e_time": t.value, "dt": dt.value, "rkmts": k, "f": arr[0], "f_prev": arr[1:k], "frhs": arr[k:]}


def write_solution_arrays(path: str, f, e_time: float, dt: float, f_prev=(), frhs=()):
    """Write a solution file; rkmts = 1 + len(frhs), f_prev zero-filled when
    shorter (the multistep formulas never read f1..f4)."""
    L = _lib.load()
    f = np.ascontiguousarray(f, np.float64).ravel()
    k = 1 + len(frhs)
    arr = np.zeros((2 * k - 1, f.size))
    arr[0] = f
    for j, a in enumerate(f_prev):
        arr[1 + j] = a
    for j, a in enumerate(frhs):
        arr[k + j] = a
    if L.dgv_write_solution_arrays(path.encode(), f.size, k, float(e_time), float(dt), arr.ctypes.data_as(C.c_void_p)):
        raise _lib.DGVError(_lib.DGV_EINVAL, L.dgv_file_error().decode())


def _paths(paths):
    if isinstance(paths, (str, bytes)):
        paths = [paths]
    enc = [p.encode() if isinstance(p, str) else p for p in paths]
    return (C.c_char_p * len(enc))(*enc), len(enc)


def read_A_arrays(paths, N: int):
    """(capphi, A, A_xi, A_xi1) of an operator file or of the chunk files of
    one operator, indices 1-based as stored."""
    L = _lib.load()
    arr, n = _paths(paths)
    nnz = C.c_int64()
    if L.dgv_read_A_arrays(arr, n, N, C.byref(nnz), None, None, None, None):
        raise _lib.DGVError(_lib.DGV_EINVAL, L.dgv_file_error().decode())
    cap = np.zeros(N, np.int32)
    A = np.zeros(nnz.value)
    xi = np.zeros(nnz.value, np.int32)
    xi1 = np.zeros(nnz.value, np.int32)
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)
    if L.dgv_read_A_arrays(arr, n, N, C.byref(nnz), ptr(cap), ptr(A), ptr(xi), ptr(xi1)):
        raise _lib.DGVError(_lib.DGV_EINVAL, L.dgv_file_error().decode())
    return cap, A, xi, xi1


def write_A_arrays(path: str, capphi, A, A_xi, A_xi1, max_subrecord: int = 0):
    """Write one operator file; A_xi / A_xi1 1-based."""
    L = _lib.load()
    cap = np.ascontiguousarray(capphi, np.int32)
    A = np.ascontiguousarray(A, np.float64)
    xi = np.ascontiguousarray(A_xi, np.int32)
    xi1 = np.ascontiguousarray(A_xi1, np.int32)
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)
    if L.dgv_write_A_arrays(path.encode(), len(cap), len(A), ptr(cap), ptr(A), ptr(xi), ptr(xi1), max_subrecord):
        raise _lib.DGVError(_lib.DGV_EINVAL, L.dgv_file_error().decode())

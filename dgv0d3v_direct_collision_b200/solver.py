"""Host-side mirror of the reference's collision/time-stepping interface.

`DGVSolver` wraps one C-ABI context (include/dgv_b200.h).  Its methods carry the
names of the Fortran routines they replace, take the same arguments (minus the
module globals, which live in the context) and fail the way the reference
fails -- by raising instead of `stop`:

    EvalCollisionPeriodicAPlus_DGV(f)        collision_mod.f90:143-229
    EvalCollisionPeriodicMixedTermsA_DGV(f, fm)  collision_mod.f90:244-332
    PrepareFMA_DGV(fm) / EvalCollisionLinear(f)  collision_mod.f90:377-464, 346-359
    SpatialOperSH_DGV(f, dt)                 spat_oper_mod.f90:28-68 (run_mode 0)
    TimeIntegratorORK_SH_DGV(f, dt)          time_integr_mod.f90:26-152
    PrepareMTS_SH_DGV(f, dt)                 time_integr_mod.f90:443-569
    TimeIntegratorMTS_SH_DGV(f, dt)          time_integr_mod.f90:314-364
    MassCheckRec(f)                          dgvtools_mod.f90:1437-1458
    maxwelveldist(T, u0, v0, w0, n)          distributions_mod.f90:83-95

Arrays may be numpy arrays (host memory, copied through the library's staging
buffers) or CUDA torch tensors (used in place).  All arithmetic runs in the
library's sm_100a kernels.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from ._lib import (DGVError, GridDesc, DGV_PREC_F64, DGV_PREC_F32C, DGV_PREC_TC, DGV_OPT_PROJECT,
                   DGV_OPT_NCHUNKS, DGV_OPT_KTIMING, DGV_OPT_TCFORM, DGV_OPT_TCTILES, DGV_OPT_TCSETMB)

PRECISIONS = {"f64": DGV_PREC_F64, "f32c": DGV_PREC_F32C, "tc": DGV_PREC_TC}


def _ptr(a):
    """Data pointer of a numpy array or a torch tensor."""
    if isinstance(a, np.ndarray):
        if not a.flags.c_contiguous:
            raise ValueError("arrays must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)}")


def _check_f64(a):
    dt = getattr(a, "dtype", None)
    if isinstance(a, np.ndarray):
        if dt != np.float64:
            raise TypeError("arrays must be float64")
    elif str(dt) != "torch.float64":
        raise TypeError("tensors must be float64")


class DGVSolver:
    """One uniform velocity grid with its A-arrays on one GPU."""

    def __init__(self, s: int = 3, M: int = 5, L: float = 6.0, *, su=None, sv=None, sw=None,
                 Mu=None, Mv=None, Mw=None, bounds=None, kappa: float = 1.0, device: int = 0,
                 precision: str = "f64", rkmts: int = 2):
        self._lib = _lib.load()
        su = su or s; sv = sv or s; sw = sw or s
        Mu = Mu or M; Mv = Mv or M; Mw = Mw or M
        b = bounds or (-L, L, -L, L, -L, L)
        self.desc = GridDesc(su, sv, sw, Mu, Mv, Mw, *b, kappa)
        h = C.c_void_p()
        rc = self._lib.dgv_ctx_create(C.byref(self.desc), device, C.byref(h))
        if rc != 0:
            raise DGVError(rc, "dgv_ctx_create failed (grid or device)")
        self._h = h
        N = C.c_int64(); P = C.c_int32(); Nc = C.c_int32(); cc = C.c_int32()
        self._lib.dgv_grid_info(h, C.byref(N), C.byref(P), C.byref(Nc), C.byref(cc))
        self.N, self.P, self.Nc, self.ccell = N.value, P.value, Nc.value, cc.value
        self.nodes_u = np.zeros(self.N); self.nodes_v = np.zeros(self.N)
        self.nodes_w = np.zeros(self.N); self.nodes_gwts = np.zeros(self.N)
        self._lib.dgv_nodes(h, _ptr(self.nodes_u), _ptr(self.nodes_v), _ptr(self.nodes_w),
                            _ptr(self.nodes_gwts))
        self.precision = precision
        self.rkmts = rkmts
        self.device = device
        self.kappa = float(kappa)
        self.projection = False
        self.tc_form = 2

    # -- plumbing ------------------------------------------------------------
    def _check(self, rc: int):
        if rc != 0:
            msg = self._lib.dgv_last_error(self._h)
            raise DGVError(rc, msg.decode() if msg else "")

    def _prec(self, precision: Optional[str]) -> int:
        p = precision or self.precision
        if p not in PRECISIONS:
            raise ValueError(f"precision must be one of {list(PRECISIONS)}")
        return PRECISIONS[p]

    @staticmethod
    def _like(f):
        if isinstance(f, np.ndarray):
            return np.zeros_like(f, dtype=np.float64)
        import torch
        return torch.zeros_like(f, dtype=torch.float64)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.dgv_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int):
        self._check(self._lib.dgv_set_stream(self._h, stream_ptr))

    def set_async(self, flag: bool):
        self._check(self._lib.dgv_set_async(self._h, int(flag)))

    def set_projection(self, on: bool):
        self._check(self._lib.dgv_set_option(self._h, DGV_OPT_PROJECT, int(on)))
        self.projection = bool(on)

    def set_regime(self, decomp_lev: float, linear_lev: float):
        """Run modes of SpatialOperSH_DGV (CheckSolutionMode_DGV); decomp_lev = 0 switches them off."""
        self._check(self._lib.dgv_set_regime(self._h, float(decomp_lev), float(linear_lev)))

    def regime_info(self):
        """(run_mode, last relative L1 distance of f to its local Maxwellian)"""
        m, l1 = C.c_int32(), C.c_double()
        self._check(self._lib.dgv_regime_info(self._h, C.byref(m), C.byref(l1)))
        return m.value, l1.value

    def set_nchunks(self, n: int):
        self._check(self._lib.dgv_set_option(self._h, DGV_OPT_NCHUNKS, int(n)))

    def set_tc_form(self, form: int):
        """Tensor-core form: 2 (default) = dense cell-pair blocks (grids of 8
        or 27 nodes per cell; others use the chunk form), 1 = pair chunks."""
        self._check(self._lib.dgv_set_option(self._h, DGV_OPT_TCFORM, int(form)))
        self.tc_form = int(form)

    def set_tc_tiles_per_cta(self, n: int):
        """Block form: VDF tiles (of up to 128) per CTA, 2 or 1."""
        self._check(self._lib.dgv_set_option(self._h, DGV_OPT_TCTILES, int(n)))

    def tc_plan(self, nvdf: int):
        """Launches, work items and issued tensor FLOPs of one tensor-core
        evaluation of nvdf VDFs in the current form."""
        l = C.c_int64(); it = C.c_int64(); fl = C.c_double()
        self._check(self._lib.dgv_tc_plan(self._h, int(nvdf), C.byref(l), C.byref(it), C.byref(fl)))
        return {"launches": l.value, "items": it.value, "tensor_flop": fl.value}

    def get_option(self, option: int) -> int:
        """The current value of a DGV_OPT_* option (dgv_get_option)."""
        v = C.c_int64(0)
        self._check(self._lib.dgv_get_option(self._h, int(option), C.byref(v)))
        return int(v.value)

    def set_tc_set_mb(self, mb: int):
        """Block form: megabytes of block records per kernel launch."""
        self._check(self._lib.dgv_set_option(self._h, DGV_OPT_TCSETMB, int(mb)))

    def release_layouts(self, f32: bool = False, tc_chunk: bool = False, tc_block: bool = False,
                        tc_adjoint: bool = False) -> int:
        """Frees device layouts that are not needed (dgv_release_layouts):
        the FP32 rows, the chunk-form or block-form tensor-core records, or
        only the block-form adjoint's second record set.  Each is rebuilt on
        its next use.  Returns the change in the device's free memory."""
        from ._lib import DGV_LAYOUT_F32, DGV_LAYOUT_TC_ADJ, DGV_LAYOUT_TC_BLOCK, DGV_LAYOUT_TC_CHUNK
        mask = ((DGV_LAYOUT_F32 if f32 else 0) | (DGV_LAYOUT_TC_CHUNK if tc_chunk else 0) |
                (DGV_LAYOUT_TC_BLOCK if tc_block else 0) | (DGV_LAYOUT_TC_ADJ if tc_adjoint else 0))
        freed = C.c_int64()
        self._check(self._lib.dgv_release_layouts(self._h, mask, C.byref(freed)))
        return freed.value

    def set_tc_persistent(self, on: bool):
        """Block form: one persistent launch over all block sets (1) or one
        launch per set (0) -- the same results bit for bit
        (DGV_OPT_TCPERSIST; setting it switches the launch tuning off)."""
        from ._lib import DGV_OPT_TCPERSIST
        self._check(self._lib.dgv_set_option(self._h, DGV_OPT_TCPERSIST, int(on)))

    def set_f_global(self, on: bool):
        """CUDA-core kernels gather f from a local-major copy in global memory
        instead of staging it in shared memory (DGV_OPT_FGLOBAL; grids whose f
        does not fit in shared memory use it in any case)."""
        from ._lib import DGV_OPT_FGLOBAL
        self._check(self._lib.dgv_set_option(self._h, DGV_OPT_FGLOBAL, int(on)))

    def set_kernel_timing(self, on: bool):
        """Time the collision kernel's launches with CUDA events on the
        context stream (read back with kernel_stats)."""
        self._check(self._lib.dgv_set_option(self._h, DGV_OPT_KTIMING, int(on)))

    def kernel_stats(self, reset: bool = True):
        """(device ms, launches) of the collision kernel and the number of
        this library's kernel launches, summed since the last reset."""
        ms, nl, na = C.c_double(), C.c_int64(), C.c_int64()
        self._check(self._lib.dgv_kernel_stats(self._h, C.byref(ms), C.byref(nl), C.byref(na), int(reset)))
        return {"ms": ms.value, "launches": nl.value, "all_launches": na.value}

    # -- A-arrays -------------------------------------------------------------
    def load_A(self, capphi, A, xi, xi1, one_based: bool = True):
        """A-arrays in the reference layout (ReadAarraysDGV, readwrite.f90:1066-1118)."""
        capphi = np.ascontiguousarray(capphi, np.int32)
        A = np.ascontiguousarray(A, np.float64)
        xi = np.ascontiguousarray(xi, np.int32)
        xi1 = np.ascontiguousarray(xi1, np.int32)
        if capphi.shape != (self.N,):
            raise ValueError(f"A_capphi must have {self.N} entries")
        if not (len(A) == len(xi) == len(xi1)):
            raise ValueError("A, A_xi, A_xi1 lengths differ")
        self._check(self._lib.dgv_load_A(self._h, len(A), _ptr(capphi), _ptr(A), _ptr(xi),
                                         _ptr(xi1), int(one_based)))

    ReadAarraysDGV = load_A

    def generate_synthetic_A(self, seed: int = 1, Trad: float = float("inf"), support: int = 1):
        self._check(self._lib.dgv_generate_A_synthetic(self._h, seed, Trad, support))

    def SetA_DGV(self, Trad: float = float("inf"), ErrChi: float = 1e-4, ErrEps: float = 1e-4,
                 min_sens: float = 0.0, basis_mode: int = 0):
        """Compute the A-arrays of every canonical basis function on the GPU
        (the reference's SetA_DGV precompute) and load them."""
        self._check(self._lib.dgv_compute_A(self._h, float(Trad), float(ErrChi), float(ErrEps),
                                            float(min_sens), int(basis_mode)))

    compute_A = SetA_DGV

    def read_A_files(self, paths):
        """Load an operator file (or the chunk files of one operator) in the
        reference's format (ReadAarraysDGV / ReadAarraysChnksDGV)."""
        from .afile import _paths
        arr, n = _paths(paths)
        self._check(self._lib.dgv_read_A_files(self._h, arr, n))

    def write_A_file(self, path: str, max_subrecord: int = 0):
        """Write the loaded A-arrays as one operator file (WriteAarraysDGV)."""
        self._check(self._lib.dgv_write_A_file(self._h, path.encode(), int(max_subrecord)))

    def A_info(self):
        nr = C.c_int64(); npairs = C.c_int64(); nb = C.c_int64(); rs = C.c_double()
        self._check(self._lib.dgv_A_info(self._h, C.byref(nr), C.byref(npairs), C.byref(nb),
                                         C.byref(rs)))
        return {"records": nr.value, "pairs": npairs.value, "blocks": nb.value,
                "record_shifts": rs.value}

    def export_A(self):
        """Loaded A-arrays back in the reference layout (0-based indices)."""
        n = C.c_int64()
        self._check(self._lib.dgv_export_A(self._h, C.byref(n), None, None, None, None))
        capphi = np.zeros(self.N, np.int32)
        A = np.zeros(n.value); xi = np.zeros(n.value, np.int32); xi1 = np.zeros(n.value, np.int32)
        self._check(self._lib.dgv_export_A(self._h, C.byref(n), _ptr(capphi), _ptr(A), _ptr(xi),
                                           _ptr(xi1)))
        return capphi, A, xi, xi1

    # -- collision operator ---------------------------------------------------
    def EvalCollisionPeriodicAPlus_DGV(self, f, fc=None, precision=None):
        _check_f64(f)
        nb = int(np.prod(f.shape)) // self.N
        if nb * self.N != int(np.prod(f.shape)):
            raise ValueError(f"f must hold a multiple of {self.N} values")
        fc = self._like(f) if fc is None else fc
        self._check(self._lib.dgv_collide_batched(self._h, nb, _ptr(f), _ptr(fc), self._prec(precision)))
        return fc

    collide = EvalCollisionPeriodicAPlus_DGV

    def collide_cells(self, f, cell0: int, cell1: int, out=None, precision=None):
        """Q on output cells [cell0, cell1) only (one rank's share of a sharded
        evaluation): returns (..., (cell1-cell0)*P) in node order."""
        _check_f64(f)
        nb = int(np.prod(f.shape)) // self.N
        if nb * self.N != int(np.prod(f.shape)):
            raise ValueError(f"f must hold a multiple of {self.N} values")
        shape = tuple(f.shape[:-1]) + ((cell1 - cell0) * self.P,)
        if out is None:
            if isinstance(f, np.ndarray):
                out = np.zeros(shape)
            else:
                import torch
                out = torch.zeros(shape, dtype=torch.float64, device=f.device)
        self._check(self._lib.dgv_collide_cells(self._h, nb, _ptr(f), _ptr(out), int(cell0), int(cell1),
                                                self._prec(precision)))
        return out

    def EvalCollisionPeriodicMixedTermsA_DGV(self, f, fm, fc=None):
        """2/w sum A (fm(xi) f(xi1) + f(xi) fm(xi1)): the JVP of Q at fm along f."""
        _check_f64(f); _check_f64(fm)
        fc = self._like(f) if fc is None else fc
        self._check(self._lib.dgv_jvp(self._h, _ptr(fm), _ptr(f), _ptr(fc), DGV_PREC_F64))
        return fc

    def jvp(self, f, df, out=None):
        return self.EvalCollisionPeriodicMixedTermsA_DGV(df, f, out)

    def vjp(self, f, v, out=None, precision="f64"):
        """g = J(f)^T v for one VDF or a batch [nb, N] (dgv_vjp_batched);
        precision "f64" (FP64 kernel per VDF) or "tc" (block form on the
        tensor cores, all VDFs in one pass)."""
        _check_f64(f); _check_f64(v)
        if tuple(f.shape) != tuple(v.shape) or f.shape[-1] != self.N:
            raise ValueError("vjp: f and v must have the same shape [..., N]")
        out = self._like(f) if out is None else out
        nb = int(np.prod(f.shape)) // self.N
        self._check(self._lib.dgv_vjp_batched(self._h, nb, _ptr(f), _ptr(v), _ptr(out), self._prec(precision)))
        return out

    def PrepareFMA_DGV(self, fm):
        _check_f64(fm)
        self._check(self._lib.dgv_prepare_linear(self._h, _ptr(fm)))

    def EvalCollisionLinear(self, f, fc=None):
        _check_f64(f)
        fc = self._like(f) if fc is None else fc
        self._check(self._lib.dgv_apply_linear(self._h, _ptr(f), _ptr(fc), DGV_PREC_F64))
        return fc

    def SpatialOperSH_DGV(self, f, dt, fcol=None, precision=None):
        _check_f64(f)
        fcol = self._like(f) if fcol is None else fcol
        self._check(self._lib.dgv_spatial_oper(self._h, _ptr(f), _ptr(fcol), dt, self._prec(precision)))
        return fcol

    def project(self, q):
        nb = int(np.prod(q.shape)) // self.N
        self._check(self._lib.dgv_project(self._h, _ptr(q), nb))
        return q

    # -- time integration ----------------------------------------------------
    def TimeIntegratorORK_SH_DGV(self, f, dt, frhs1=None, order=None, precision=None):
        """One RK step in place on f, one VDF [N] or a batch [nb, N]
        (dgv_step_rk_batched: each stage's Q of the batch in one call);
        returns frhs1 (first-stage right side / dt)."""
        _check_f64(f)
        if f.shape[-1] != self.N:
            raise ValueError("TimeIntegratorORK_SH_DGV: last axis must have N entries")
        frhs1 = self._like(f) if frhs1 is None else frhs1
        nb = int(np.prod(f.shape)) // self.N
        if nb == 1:
            self._check(self._lib.dgv_step_rk(self._h, _ptr(f), _ptr(frhs1), dt, order or self.rkmts,
                                              self._prec(precision)))
        else:
            self._check(self._lib.dgv_step_rk_batched(self._h, nb, _ptr(f), _ptr(frhs1), dt, order or self.rkmts,
                                                      self._prec(precision)))
        return frhs1

    def PrepareMTS_SH_DGV(self, f, dt, order=None, precision=None):
        _check_f64(f)
        self._check(self._lib.dgv_prepare_ab(self._h, _ptr(f), dt, order or self.rkmts,
                                             self._prec(precision)))

    def TimeIntegratorMTS_SH_DGV(self, f, dt, precision=None):
        _check_f64(f)
        self._check(self._lib.dgv_step_ab(self._h, _ptr(f), dt, self._prec(precision)))

    def WriteSol_DGV(self, path: str, f, e_time: float, dt: float):
        """Write f and the Adams-Bashforth history in the reference's solution
        file format (WriteSol_DGV; name it with afile.solution_file_name)."""
        _check_f64(f)
        self._check(self._lib.dgv_write_solution(self._h, path.encode(), _ptr(f), float(e_time), float(dt)))

    def RestartSolutionDGV(self, path: str, f=None):
        """Read a solution file into f (a new host array when None) and the
        Adams-Bashforth history; returns (f, e_time, dt).  rkmts becomes the
        file's order, as RestartSolutionDGV sets it."""
        f = np.zeros(self.N) if f is None else f
        _check_f64(f)
        t = C.c_double(); dt = C.c_double()
        self._check(self._lib.dgv_read_solution(self._h, path.encode(), _ptr(f), C.byref(t), C.byref(dt)))
        r = C.c_int32()
        if self._lib.dgv_read_solution_arrays(path.encode(), None, C.byref(r), None, None, None) == 0:
            self.rkmts = r.value
        return f, t.value, dt.value

    # -- moments and equilibrium ----------------------------------------------
    def MassCheckRec(self, f):
        _check_f64(f)
        out = np.zeros(5)
        self._check(self._lib.dgv_moments(self._h, _ptr(f), _ptr(out)))
        return tuple(out)

    def maxwelveldist(self, T, u0, v0, w0, n, out=None):
        out = np.zeros(self.N) if out is None else out
        self._check(self._lib.dgv_maxwellian(self._h, T, u0, v0, w0, n, _ptr(out)))
        return out


def collide_group(members, precision: Optional[str] = None, stream_ptr: int = 0):
    """Q of a mixed batch over several grids in one call: members is a list
    of (solver, f, q) with f, q device tensors [nb, N] of that solver's grid
    (all solvers on one device).  Repeated calls with the same members replay
    one captured CUDA graph (dgv_collide_group)."""
    if not members:
        raise ValueError("need at least one member")
    n = len(members)
    s0 = members[0][0]
    ctxs = (C.c_void_p * n)(*[m[0]._h.value for m in members])
    nbs, fs, qs = (C.c_int32 * n)(), (C.c_void_p * n)(), (C.c_void_p * n)()
    for i, (s, f, q) in enumerate(members):
        _check_f64(f); _check_f64(q)
        nb = int(np.prod(f.shape)) // s.N
        if nb < 1 or nb * s.N != int(np.prod(f.shape)) or int(np.prod(q.shape)) != nb * s.N:
            raise ValueError(f"member {i}: f and q must hold nb x {s.N} values")
        nbs[i], fs[i], qs[i] = nb, _ptr(f), _ptr(q)
    s0._check(s0._lib.dgv_collide_group(n, ctxs, nbs, fs, qs, s0._prec(precision), stream_ptr or None))
    return [m[2] for m in members]

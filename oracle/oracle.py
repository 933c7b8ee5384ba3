"""ctypes wrapper around oracle/libdgv_oracle.so.

TEST INFRASTRUCTURE ONLY.  The oracle is the CPU FP64 restatement of the
reference's collision hot path (collision_mod.f90, time_integr_mod.f90,
spat_oper_mod.f90, dgvtools_mod.f90, miscset.f90, distributions_mod.f90).  It
may be imported by tests/, by __graft_entry__.smoke() and by bench.py's CPU
baseline leg only -- the product package never imports it.

Parity status: unpinned against reference outputs (the Fortran reference cannot
be compiled in this environment and ships no golden vectors); pinned by the
reference-derived invariants listed in oracle/dgv_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libdgv_oracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


class GridDesc(C.Structure):
    _fields_ = [("su", C.c_int32), ("sv", C.c_int32), ("sw", C.c_int32),
                ("Mu", C.c_int32), ("Mv", C.c_int32), ("Mw", C.c_int32),
                ("u_L", C.c_double), ("u_R", C.c_double), ("v_L", C.c_double),
                ("v_R", C.c_double), ("w_L", C.c_double), ("w_R", C.c_double)]


def build():
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.check_call(["make", "-s", "-C", _HERE], stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp = C.c_void_p
        L.dgvo_create.restype = vp
        L.dgvo_create.argtypes = [C.POINTER(GridDesc)]
        L.dgvo_destroy.argtypes = [vp]
        for name, rt in [("dgvo_num_nodes", C.c_int64), ("dgvo_nodes_per_cell", C.c_int32),
                         ("dgvo_num_cells", C.c_int32), ("dgvo_canonical_cell", C.c_int32)]:
            getattr(L, name).restype = rt
            getattr(L, name).argtypes = [vp]
        L.dgvo_get_nodes.argtypes = [vp, _dp, _dp, _dp, _dp, _ip, _ip, _ip, _ip]
        L.dgvo_get_cells.argtypes = [vp, _ip, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp]
        L.dgvo_gauss_legendre.argtypes = [C.c_int, _dp, _dp]
        L.dgvo_find_cell.restype = C.c_int32
        L.dgvo_find_cell.argtypes = [vp, C.c_double, C.c_double, C.c_double]
        L.dgvo_set_A.restype = C.c_int
        L.dgvo_set_A.argtypes = [vp, _ip, C.c_int64, _dp, _ip, _ip, C.c_int]
        L.dgvo_get_shift_tables.argtypes = [vp, _ip, _ip, _ip, _ip, _lp]
        L.dgvo_collide_aplus.argtypes = [vp, _dp, _dp, C.c_void_p, C.c_int64, C.c_int]
        L.dgvo_collide_a.argtypes = [vp, _dp, _dp]
        L.dgvo_iphi.argtypes = [vp, _dp, C.c_double, _dp]
        L.dgvo_mixed_terms.argtypes = [vp, _dp, _dp, _dp, C.c_int]
        L.dgvo_prepare_fma.argtypes = [vp, _dp, _dp]
        L.dgvo_eval_linear.argtypes = [vp, _dp, _dp, _dp]
        L.dgvo_vjp.argtypes = [vp, _dp, _dp, _dp, C.c_int]
        L.dgvo_spatial_oper.argtypes = [vp, _dp, _dp, C.c_double, C.c_double, C.c_int]
        L.dgvo_regime_create.restype = vp
        L.dgvo_regime_create.argtypes = [vp, C.c_double, C.c_double]
        L.dgvo_regime_free.argtypes = [vp]
        L.dgvo_regime_mode.restype = C.c_int
        L.dgvo_regime_mode.argtypes = [vp, C.POINTER(C.c_double)]
        L.dgvo_spatial_oper_regime.argtypes = [vp, vp, _dp, _dp, C.c_double, C.c_double, C.c_int]
        L.dgvo_rk_step_regime.restype = C.c_int
        L.dgvo_rk_step_regime.argtypes = [vp, vp, C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_int]
        L.dgvo_rk_step.restype = C.c_int
        L.dgvo_rk_step.argtypes = [vp, C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_int]
        L.dgvo_ab_step.restype = C.c_int
        L.dgvo_ab_step.argtypes = [vp, C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_int]
        L.dgvo_prepare_ab.restype = C.c_int
        L.dgvo_prepare_ab.argtypes = [vp, C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_int]
        L.dgvo_moments.argtypes = [vp, _dp, _dp]
        L.dgvo_maxwellian.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double,
                                      C.c_double, _dp]
        L.dgvo_project_conservative.argtypes = [vp, _dp]
        L.dgvo_seta.restype = C.c_int64
        L.dgvo_seta.argtypes = [vp, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
                                C.c_int, C.c_int, C.POINTER(C.POINTER(C.c_double)),
                                C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.POINTER(C.c_int32))]
        L.dgvo_seta_pair_integral.restype = C.c_double
        L.dgvo_seta_pair_integral.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                              C.c_double, C.c_int]
        L.dgvo_synth_A.restype = C.c_int64
        L.dgvo_synth_A.argtypes = [vp, C.c_uint64, C.c_double, C.c_int, C.c_int32,
                                   C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.POINTER(C.c_double)),
                                   C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.POINTER(C.c_int32))]
        L.dgvo_synth_value.restype = C.c_double
        L.dgvo_synth_value.argtypes = [C.c_uint64, C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                       C.c_double, C.c_double]
        L.dgvo_free.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def gauss_legendre(n: int):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().dgvo_gauss_legendre(n, x, w)
    return x, w


def _take(ptr, n, dtype):
    """Copy a malloc'd C array into numpy and free it."""
    if n == 0:
        out = np.zeros(0, dtype=dtype)
    else:
        ctype = C.c_double if dtype == np.float64 else C.c_int32
        buf = C.cast(ptr, C.POINTER(ctype * n)).contents
        out = np.frombuffer(buf, dtype=dtype).copy()
    lib().dgvo_free(C.cast(ptr, C.c_void_p))
    return out


class Oracle:
    """One uniform velocity grid plus (optionally) A-arrays, in the reference layout."""

    def __init__(self, s=3, M=5, L=6.0, su=None, sv=None, sw=None, Mu=None, Mv=None, Mw=None,
                 bounds=None):
        su = su or s; sv = sv or s; sw = sw or s
        Mu = Mu or M; Mv = Mv or M; Mw = Mw or M
        b = bounds or (-L, L, -L, L, -L, L)
        self.desc = GridDesc(su, sv, sw, Mu, Mv, Mw, *b)
        self._h = lib().dgvo_create(C.byref(self.desc))
        if not self._h:
            raise ValueError("invalid grid")
        L_ = lib()
        self.N = L_.dgvo_num_nodes(self._h)
        self.P = L_.dgvo_nodes_per_cell(self._h)
        self.Nc = L_.dgvo_num_cells(self._h)
        self.ccell = L_.dgvo_canonical_cell(self._h)
        N = self.N
        self.u = np.zeros(N); self.v = np.zeros(N); self.w = np.zeros(N); self.gwts = np.zeros(N)
        self.pcell = np.zeros(N, np.int32); self.ui = np.zeros(N, np.int32)
        self.vi = np.zeros(N, np.int32); self.wi = np.zeros(N, np.int32)
        L_.dgvo_get_nodes(self._h, self.u, self.v, self.w, self.gwts, self.pcell, self.ui,
                          self.vi, self.wi)
        self.has_A = False

    def __del__(self):
        try:
            if self._h:
                lib().dgvo_destroy(self._h)
        except Exception:
            pass

    # --- A arrays ----------------------------------------------------------
    def set_A(self, capphi, A, xi, xi1, one_based=False):
        capphi = np.ascontiguousarray(capphi, np.int32)
        A = np.ascontiguousarray(A, np.float64)
        xi = np.ascontiguousarray(xi, np.int32)
        xi1 = np.ascontiguousarray(xi1, np.int32)
        rc = lib().dgvo_set_A(self._h, capphi, len(A), A, xi, xi1, int(one_based))
        if rc != 0:
            raise ValueError(f"dgvo_set_A failed with code {rc}")
        self.capphi, self.A, self.xi, self.xi1 = capphi, A, (xi - int(one_based)), (xi1 - int(one_based))
        self.has_A = True

    def shift_tables(self):
        N = self.N
        out = [np.zeros(N, np.int32) for _ in range(4)] + [np.zeros(N, np.int64)]
        lib().dgvo_get_shift_tables(self._h, *out)
        return dict(zip(["dui", "dvi", "dwi", "phican", "Ashift"], out))

    def synth_A(self, seed=1, Trad=np.inf, support=1, p_only=-1):
        cp = C.POINTER(C.c_int32)(); ap = C.POINTER(C.c_double)()
        xp = C.POINTER(C.c_int32)(); x1p = C.POINTER(C.c_int32)()
        nnz = lib().dgvo_synth_A(self._h, seed, Trad, support, p_only, C.byref(cp), C.byref(ap),
                                 C.byref(xp), C.byref(x1p))
        capphi = _take(cp, self.N, np.int32)
        A = _take(ap, nnz, np.float64)
        xi = _take(xp, nnz, np.int32)
        xi1 = _take(x1p, nnz, np.int32)
        return capphi, A, xi, xi1

    def seta(self, i1, Trad=np.inf, ErrChi=1e-4, ErrEps=1e-4, min_sens=0.0, basis_mode=0,
             nthreads=0):
        ap = C.POINTER(C.c_double)(); xp = C.POINTER(C.c_int32)(); x1p = C.POINTER(C.c_int32)()
        n = lib().dgvo_seta(self._h, i1, Trad, ErrChi, ErrEps, min_sens, basis_mode, nthreads,
                            C.byref(ap), C.byref(xp), C.byref(x1p))
        return _take(ap, n, np.float64), _take(xp, n, np.int32), _take(x1p, n, np.int32)

    def seta_pair_integral(self, i1, i2, i3, ErrChi=1e-4, ErrEps=1e-4, basis_mode=0):
        return lib().dgvo_seta_pair_integral(self._h, i1, i2, i3, ErrChi, ErrEps, basis_mode)

    # --- collision operator -------------------------------------------------
    def collide(self, f, nodes=None, nthreads=0):
        f = np.ascontiguousarray(f, np.float64)
        fc = np.zeros(self.N)
        if nodes is None:
            lib().dgvo_collide_aplus(self._h, f, fc, None, 0, nthreads)
        else:
            nodes = np.ascontiguousarray(nodes, np.int64)
            lib().dgvo_collide_aplus(self._h, f, fc, nodes.ctypes.data, len(nodes), nthreads)
        return fc

    def collide_a(self, f):
        fc = np.zeros(self.N)
        lib().dgvo_collide_a(self._h, np.ascontiguousarray(f, np.float64), fc)
        return fc

    def iphi(self, f, kappa=1.0):
        out = np.zeros(self.N)
        lib().dgvo_iphi(self._h, np.ascontiguousarray(f, np.float64), kappa, out)
        return out

    def mixed_terms(self, f, fm, nthreads=0):
        fc = np.zeros(self.N)
        lib().dgvo_mixed_terms(self._h, np.ascontiguousarray(f, np.float64),
                               np.ascontiguousarray(fm, np.float64), fc, nthreads)
        return fc

    def prepare_fma(self, fm):
        fmA = np.zeros(self.N * self.N)
        lib().dgvo_prepare_fma(self._h, np.ascontiguousarray(fm, np.float64), fmA)
        return fmA.reshape(self.N, self.N)  # row i = column i of the Fortran array

    def eval_linear(self, fmA, f):
        fc = np.zeros(self.N)
        lib().dgvo_eval_linear(self._h, np.ascontiguousarray(fmA.reshape(-1), np.float64),
                               np.ascontiguousarray(f, np.float64), fc)
        return fc

    def vjp(self, f, v, nthreads=0):
        g = np.zeros(self.N)
        lib().dgvo_vjp(self._h, np.ascontiguousarray(f, np.float64),
                       np.ascontiguousarray(v, np.float64), g, nthreads)
        return g

    def spatial_oper(self, f, dt, kappa=1.0, nthreads=0):
        out = np.zeros(self.N)
        lib().dgvo_spatial_oper(self._h, np.ascontiguousarray(f, np.float64), out, dt, kappa,
                                nthreads)
        return out

    def rk_step(self, f, dt, order, kappa=1.0, nthreads=0):
        f = np.array(f, np.float64, copy=True)
        frhs1 = np.zeros(self.N)
        rc = lib().dgvo_rk_step(self._h, order, f, frhs1, dt, kappa, nthreads)
        if rc:
            raise ValueError("bad order")
        return f, frhs1

    # --- run modes of SpatialOperSH_DGV (spat_oper_mod.f90:28-68, 195-272) ----
    def regime(self, decomp_lev, linear_lev):
        """A run-mode state (CheckSolutionMode_DGV); pass it to spatial_oper_regime / rk_step_regime."""
        return _Regime(self, decomp_lev, linear_lev)

    def spatial_oper_regime(self, reg, f, dt, kappa=1.0, nthreads=0):
        fcol = np.zeros(self.N)
        lib().dgvo_spatial_oper_regime(self._h, reg._h, np.ascontiguousarray(f, np.float64), fcol, dt, kappa,
                                       nthreads)
        return fcol

    def rk_step_regime(self, reg, f, dt, order, kappa=1.0, nthreads=0):
        f = np.array(f, np.float64, copy=True)
        frhs1 = np.zeros(self.N)
        if lib().dgvo_rk_step_regime(self._h, reg._h, order, f, frhs1, dt, kappa, nthreads):
            raise ValueError("bad order")
        return f, frhs1

    def prepare_ab(self, f, dt, order, kappa=1.0, nthreads=0):
        f = np.array(f, np.float64, copy=True)
        frhs = np.zeros(5 * self.N)
        lib().dgvo_prepare_ab(self._h, order, f, frhs, dt, kappa, nthreads)
        return f, frhs

    def ab_step(self, f, frhs, dt, order, kappa=1.0, nthreads=0):
        f = np.array(f, np.float64, copy=True)
        frhs = np.array(frhs, np.float64, copy=True)
        lib().dgvo_ab_step(self._h, order, f, frhs, dt, kappa, nthreads)
        return f, frhs

    def moments(self, f):
        out = np.zeros(5)
        lib().dgvo_moments(self._h, np.ascontiguousarray(f, np.float64), out)
        return out

    def maxwellian(self, T=1.0, u0=0.0, v0=0.0, w0=0.0, n=1.0):
        f = np.zeros(self.N)
        lib().dgvo_maxwellian(self._h, T, u0, v0, w0, n, f)
        return f

    def project(self, q):
        q = np.array(q, np.float64, copy=True)
        lib().dgvo_project_conservative(self._h, q)
        return q

    def find_cell(self, u, v, w):
        return lib().dgvo_find_cell(self._h, u, v, w)


def synth_value(seed, p, i2, i3, w2, w3, dsph):
    return lib().dgvo_synth_value(seed, p, i2, i3, w2, w3, dsph)


class _Regime:
    def __init__(self, o, decomp_lev, linear_lev):
        self._h = lib().dgvo_regime_create(o._h, decomp_lev, linear_lev)

    @property
    def mode(self):
        return lib().dgvo_regime_mode(self._h, None)

    @property
    def last_L1(self):
        x = C.c_double()
        lib().dgvo_regime_mode(self._h, C.byref(x))
        return x.value

    def __del__(self):
        if getattr(self, "_h", None):
            lib().dgvo_regime_free(self._h)
            self._h = None

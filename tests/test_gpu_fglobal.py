"""f read from global memory by the CUDA-core kernels (FP64, FP32-compensated,
mixed terms, FP64 adjoint): grids whose f does not fit in shared memory, and
DGV_OPT_FGLOBAL forcing the same variant on any grid.

The variant changes only where the gathers f[o + D] read from (a local-major
copy in global memory instead of shared memory), not the order of any sum:
FP64, FP32-compensated and mixed-terms results are bit-identical to the
shared-memory kernels; the adjoint (FP64 atomics) agrees within 1e-13.

The grid s=3, M=11 on [-7,7]^3 (35 937 nodes, 287 KB of f in FP64: more than
a CTA's shared memory) is checked against the oracle's
EvalCollisionPeriodicAPlus_DGV (collision_mod.f90:143-229) on sampled nodes,
with seeded synthetic A-arrays."""
import numpy as np
import pytest

from conftest import rel_err
from helpers import mixture_vdf

pytestmark = pytest.mark.gpu


def _pair(s):
    rng = np.random.default_rng(4)
    f = np.stack([mixture_vdf(s.nodes_u, s.nodes_v, s.nodes_w, rng, normalise_w=s.nodes_gwts) for _ in range(3)])
    d = rng.standard_normal(f.shape) * f
    return f, d


@pytest.mark.parametrize("grid", [(3, 5, 6.0), (2, 4, 5.0), (5, 3, 5.0)])
def test_fglobal_forced_equals_shared(grid):
    import dgv0d3v_direct_collision_b200 as m
    s = m.DGVSolver(*grid)
    try:
        s.generate_synthetic_A(seed=11, support=1)
        # a fixed number of block chunks: small batches otherwise time their
        # chunk count, and a different partition sums in a different order
        s.set_nchunks(64)
        f, d = _pair(s)
        rng = np.random.default_rng(9)
        v = rng.standard_normal(s.N)
        base = {p: s.EvalCollisionPeriodicAPlus_DGV(f, precision=p) for p in ("f64", "f32c")}
        jv = s.jvp(f[0], d[0])
        vj = s.vjp(f[0], v)
        s.set_f_global(True)
        assert s.get_option(10) == 1
        for p in ("f64", "f32c"):
            q = s.EvalCollisionPeriodicAPlus_DGV(f, precision=p)
            assert np.array_equal(q, base[p]), p
        assert np.array_equal(s.jvp(f[0], d[0]), jv)
        assert rel_err(s.vjp(f[0], v), vj) < 1e-13
        s.set_f_global(False)
        assert np.array_equal(s.EvalCollisionPeriodicAPlus_DGV(f, precision="f64"), base["f64"])
    finally:
        s.close()


def test_f_larger_than_shared_memory_vs_oracle():
    """33^3 grid (s=3, M=11, [-7,7]^3): 35 937 nodes, 287 KB of f in FP64.
    The oracle holds the records of one basis function at a time; nodes of
    basis functions 0 and 26 are compared (sampled cells: corners, centre,
    seeded interior cells)."""
    import dgv0d3v_direct_collision_b200 as m
    from oracle.oracle import Oracle
    S, M, L = 3, 11, 7.0
    s = m.DGVSolver(S, M, L)
    o = Oracle(S, M, L)
    try:
        assert s.N == 35937 and s.N * 8 > 232448   # FP64 f: more than 227 KB
        s.generate_synthetic_A(seed=5, support=1)
        rng = np.random.default_rng(12)
        f = mixture_vdf(s.nodes_u, s.nodes_v, s.nodes_w, rng, normalise_w=s.nodes_gwts)
        q64 = s.EvalCollisionPeriodicAPlus_DGV(f)
        cells = np.unique(np.concatenate([[0, M - 1, M * M - 1, s.Nc - 1, (s.Nc - 1) // 2],
                                          rng.integers(0, s.Nc, 10)]))
        for p in (0, 26):
            o.set_A(*o.synth_A(seed=5, support=1, p_only=p))
            nodes = cells * s.P + p
            ref = o.collide(f, nodes=nodes)[nodes]
            assert rel_err(q64[nodes], ref) < 1e-12, p
            assert np.abs(q64[nodes] - ref).max() <= 1e-12 * np.abs(ref).max(), p
        # the adjoint and the mixed terms on the same grid: <g, d> = <v, J d>
        d = rng.standard_normal(s.N) * f
        v = rng.standard_normal(s.N)
        jd = s.jvp(f, d)
        g = s.vjp(f, v)
        assert abs(g @ d - v @ jd) <= 1e-10 * (np.abs(g * d).sum() + np.abs(v * jd).sum())
        # FP32-compensated (f fits in shared memory in FP32) against FP64
        q32 = s.EvalCollisionPeriodicAPlus_DGV(f, precision="f32c")
        assert rel_err(q32, q64) < 1e-6
    finally:
        s.close()

"""The benchmark configuration itself against the oracle: the 27^3 grid (s=3,
M=9, [-7,7]^3) with the benchmark's seeded synthetic A-arrays, compared with
the oracle's restatement of EvalCollisionPeriodicAPlus_DGV
(collision_mod.f90:143-229) on a seeded sample of output nodes.

A full oracle evaluation at 27^3 takes minutes per VDF, so the oracle
evaluates only sampled nodes: the 8 corner cells, the 6 face-centre cells,
the centre cell and 9 seeded interior cells, at basis functions 0 and 26 (all
24 cells) and 13 (8 cells).  The oracle holds the records of one basis
function at a time (its records are only read by the nodes of that basis
function, collision_mod.f90:186-188), ~0.9 GB per basis function.

Tolerances: plain FP64 path 1e-12 (norm-wise and max-relative over the
sample); tensor-core path (batch of 256, both VDF tiles sampled) 1e-6
norm-wise and 2e-6 max-relative, without the conservation projection (it
needs the whole Q)."""
import numpy as np
import pytest

from helpers import mixture_vdf

pytestmark = pytest.mark.gpu

S, M, L = 3, 9, 7.0
SEED_A = 20260101
VDFS = (0, 1, 130, 255)


def _sample_cells(M, seed=7):
    cells = set()
    for u in (0, M - 1):
        for v in (0, M - 1):
            for w in (0, M - 1):
                cells.add((u, v, w))
    c = M // 2
    for ax in range(3):
        for e in (0, M - 1):
            x = [c, c, c]
            x[ax] = e
            cells.add(tuple(x))
    cells.add((c, c, c))
    rng = np.random.default_rng(seed)
    while len(cells) < 24:
        cells.add(tuple(int(t) for t in rng.integers(1, M - 1, 3)))
    return sorted((u * M + v) * M + w for (u, v, w) in cells)


@pytest.fixture(scope="module")
def pin27():
    import dgv0d3v_direct_collision_b200 as m
    from oracle.oracle import Oracle
    s = m.DGVSolver(S, M, L)
    s.generate_synthetic_A(seed=SEED_A, support=1)
    o = Oracle(S, M, L)
    rng = np.random.default_rng(1000)
    fs = np.stack([mixture_vdf(o.u, o.v, o.w, rng, normalise_w=o.gwts) for _ in range(256)])
    cells = np.array(_sample_cells(M))
    plan = [(0, cells), (26, cells), (13, cells[::3])]
    ref = {}  # (vdf, node) -> Q
    for p, cs in plan:
        o.set_A(*o.synth_A(seed=SEED_A, support=1, p_only=p))
        nodes = cs * o.P + p
        for k in VDFS:
            q = o.collide(fs[k], nodes=nodes)
            for n in nodes:
                ref[(k, int(n))] = q[n]
    nodes = np.array(sorted({n for (_, n) in ref}))
    yield {"solver": s, "fs": fs, "nodes": nodes, "ref": np.array([[ref[(k, n)] for n in nodes] for k in VDFS])}
    s.close()


def _errs(got, ref):
    d = got - ref
    return (float(np.linalg.norm(d) / np.linalg.norm(ref)), float(np.abs(d).max() / np.abs(ref).max()))


def test_f64_27cubed_sampled_nodes(pin27):
    s, fs, nodes, ref = pin27["solver"], pin27["fs"], pin27["nodes"], pin27["ref"]
    q = s.EvalCollisionPeriodicAPlus_DGV(fs[list(VDFS)], precision="f64")
    for i, k in enumerate(VDFS):
        norm, mx = _errs(q[i][nodes], ref[i])
        assert norm <= 1e-12 and mx <= 1e-12, (k, norm, mx)


def test_tc_27cubed_batch256_sampled_nodes(pin27):
    s, fs, nodes, ref = pin27["solver"], pin27["fs"], pin27["nodes"], pin27["ref"]
    q = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    errs = []
    for i, k in enumerate(VDFS):
        norm, mx = _errs(q[k][nodes], ref[i])
        errs.append((k, norm, mx))
        assert norm <= 1e-6 and mx <= 2e-6, (k, norm, mx)
    print("27^3 tensor-core vs oracle (vdf, norm, max):", errs)

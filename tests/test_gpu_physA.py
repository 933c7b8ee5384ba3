"""The collision paths on physical A-arrays: the s=3, M=3 grid on [-4,4]^3
(5.36 million records, 27 basis functions per cell) computed on the device by
dgv_compute_A (SetA_DGV, dgvtools_mod.f90:377-681, ErrChi = ErrEps = 1e-3; its
parity with the oracle's SetA is tested in test_gpu_seta.py), exported and
loaded into the oracle, so that both sides evaluate the same operator.

Physical operators have the gain/loss cancellation that seeded synthetic
values lack: near equilibrium ||Q|| is ~21x smaller than the norm of the
per-node sums of |A f f| (the collision-term scale T, computed by the oracle
with |A| and |f|; on this coarse grid Q(Maxwellian) itself is 4.7% of T).

Tolerances:
  FP64 path                         <= 1e-12 of ||Q|| (norm-wise and max)
  tensor cores, mixture and bimodal <= 1e-6 of ||Q|| (norm-wise and max)
  tensor cores, near equilibrium    <= 1e-7 of ||T|| and <= 2e-6 of ||Q||:
      the split-fp16 operands carry 22 bits, so the error is a fixed
      fraction (~5e-8, measured) of the collision terms and grows relative
      to Q with the cancellation ratio ||T|| / ||Q||
  conservation with the projection  <= 1e-12 of the invariant-weighted T
  tensor-core adjoint               <= 1e-6 of ||J^T v|| against the oracle"""
import numpy as np
import pytest

from conftest import rel_err
from helpers import mixture_vdf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def phys():
    import dgv0d3v_direct_collision_b200 as m
    from oracle.oracle import Oracle
    s = m.DGVSolver(3, 3, 4.0)
    s.SetA_DGV(ErrChi=1e-3, ErrEps=1e-3)
    cap, A, xi, xi1 = s.export_A()
    o = Oracle(3, 3, 4.0)
    o.set_A(cap, A, xi, xi1)
    oa = Oracle(3, 3, 4.0)  # |A|: the collision-term scale
    oa.set_A(cap, np.abs(A), xi, xi1)
    rng = np.random.default_rng(3)
    fM = o.maxwellian(1.0, 0.0, 0.0, 0.0, 1.0)
    cases = {
        "near_eq": fM * (1.0 + 1e-3 * rng.standard_normal(o.N)),
        "maxwellian": fM,
        "bimodal": o.maxwellian(0.5, 1.2, 0.0, 0.0, 0.5) + o.maxwellian(0.5, -1.2, 0.0, 0.0, 0.5),
        "mixture": mixture_vdf(o.u, o.v, o.w, rng, normalise_w=o.gwts),
    }
    fs = np.stack(list(cases.values()))
    ref = {k: o.collide(f) for k, f in cases.items()}
    scale = {k: oa.collide(np.abs(f)) for k, f in cases.items()}
    yield {"solver": s, "oracle": o, "cases": cases, "fs": fs, "ref": ref, "scale": scale, "rng": rng}
    s.close()


def _max_rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_physical_f64_vs_oracle(phys):
    s, fs = phys["solver"], phys["fs"]
    q = s.EvalCollisionPeriodicAPlus_DGV(fs)
    for i, k in enumerate(phys["cases"]):
        assert rel_err(q[i], phys["ref"][k]) <= 1e-12, k
        assert _max_rel(q[i], phys["ref"][k]) <= 1e-12, k


@pytest.mark.parametrize("batch", [4, 130])
def test_physical_tc_vs_oracle(phys, batch):
    """The four cases alone (tile of 32 VDFs x 4 cells) and in a batch of 130
    (tiles of 128 VDFs on one cell)."""
    s, o, fs = phys["solver"], phys["oracle"], phys["fs"]
    if batch > len(fs):
        rng = np.random.default_rng(batch)
        fs = np.concatenate([fs, np.stack([mixture_vdf(o.u, o.v, o.w, rng, normalise_w=o.gwts)
                                           for _ in range(batch - len(fs))])])
    q = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    report = {}
    for i, k in enumerate(phys["cases"]):
        ref, sc = phys["ref"][k], phys["scale"][k]
        e_q, e_t = rel_err(q[i], ref), float(np.linalg.norm(q[i] - ref) / np.linalg.norm(sc))
        report[k] = (e_q, _max_rel(q[i], ref), e_t, float(np.linalg.norm(sc) / np.linalg.norm(ref)))
        if k in ("bimodal", "mixture"):
            assert e_q <= 1e-6 and _max_rel(q[i], ref) <= 1e-6, (k, report[k])
        else:
            assert e_t <= 1e-7 and e_q <= 2e-6, (k, report[k])
    print("physical A, tensor cores (norm, max, of term scale, cancellation):", report)


def test_physical_tc_projection_conserves(phys):
    s, o, fs = phys["solver"], phys["oracle"], phys["fs"]
    s.set_projection(True)
    try:
        qp = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    finally:
        s.set_projection(False)
    for i, k in enumerate(phys["cases"]):
        sc = phys["scale"][k]
        for psi in [np.ones(o.N), o.u, o.v, o.w, o.u ** 2 + o.v ** 2 + o.w ** 2]:
            assert abs(np.sum(o.gwts * psi * qp[i])) <= 1e-12 * np.sum(np.abs(o.gwts * psi * sc)), k
        if k in ("bimodal", "mixture"):
            assert rel_err(qp[i], o.project(phys["ref"][k])) <= 1e-6, k


def test_physical_tc_adjoint_vs_oracle(phys):
    s, o, fs = phys["solver"], phys["oracle"], phys["fs"]
    vs = phys["rng"].standard_normal(fs.shape)
    g = s.vjp(fs, vs, precision="tc")
    for i, k in enumerate(phys["cases"]):
        assert rel_err(g[i], o.vjp(fs[i], vs[i])) <= 1e-6, k

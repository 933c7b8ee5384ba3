"""The block decomposition the tensor-core kernel uses, restated in numpy on
the CPU and checked against the oracle's EvalCollisionPeriodicAPlus_DGV
(collision_mod.f90:143-229).  Records of the canonical basis functions are
grouped by the cells (c1, c2) of their two velocities; each group is a dense
matrix W[l2, l1, p] (0 where there is no record), and for an output cell D
whose shifted cells c1 + D - cc and c2 + D - cc lie in the grid

    Q[D, p] = 2/w * sum_blocks sum_l1 f(c1 + D - cc, l1) * (F2 W)[l1, p],
    F2[l2] = f(c2 + D - cc, l2),

which is G = F2 W on the tensor core followed by the contraction with f(c1)
on the CUDA cores.  Exact in FP64 (1e-13)."""
import numpy as np
import pytest


def _cell3(c, M):
    return np.stack([c // (M * M), (c // M) % M, c % M], axis=-1)


@pytest.mark.parametrize("s,M,L,seed", [(2, 3, 3.0, 3), (2, 4, 4.0, 7)])
def test_block_form_equals_oracle(s, M, L, seed):
    from oracle.oracle import Oracle
    o = Oracle(s, M, L)
    cap, A, xi, xi1 = o.synth_A(seed=seed, support=1)
    o.set_A(cap, A, xi, xi1)
    P, Nc = o.P, o.Nc
    phi = np.repeat(np.arange(o.N), cap)            # canonical node of each record
    p = phi % P
    assert np.all(phi // P == o.ccell)
    c1, l1 = xi // P, xi % P
    c2, l2 = xi1 // P, xi1 % P
    # dense W per cell pair
    blocks = {}
    for k in range(len(A)):
        key = (int(c1[k]), int(c2[k]))
        W = blocks.setdefault(key, np.zeros((P, P, P)))  # [l2, l1, p]
        W[l2[k], l1[k], p[k]] += A[k]
    rng = np.random.default_rng(seed)
    f = o.maxwellian(0.7, 0.5, -0.3, 0.2, 0.8) + 0.3 * o.maxwellian(0.5, -0.6, 0.4, 0.0, 0.6)
    f = f * (1.0 + 0.05 * rng.standard_normal(o.N))
    fc = f.reshape(Nc, P)
    cc = _cell3(np.array(o.ccell), M)
    D3 = _cell3(np.arange(Nc), M)
    q = np.zeros((Nc, P))
    for (a, b), W in blocks.items():
        s1 = _cell3(np.array(a), M) + D3 - cc        # shifted cells for every output cell D
        s2 = _cell3(np.array(b), M) + D3 - cc
        ok = np.all((s1 >= 0) & (s1 < M) & (s2 >= 0) & (s2 < M), axis=1)
        if not ok.any():
            continue
        i1 = (s1[ok, 0] * M + s1[ok, 1]) * M + s1[ok, 2]
        i2 = (s2[ok, 0] * M + s2[ok, 1]) * M + s2[ok, 2]
        G = np.einsum("dk,klp->dlp", fc[i2], W)      # F2 W: [D, l1, p]
        q[ok] += np.einsum("dl,dlp->dp", fc[i1], G)  # contraction with f(c1)
    q = 2.0 * q.ravel() / o.gwts
    ref = o.collide(f)
    assert np.linalg.norm(q - ref) / np.linalg.norm(ref) < 1e-13
    # the blocks are dense enough that the W matrices are the sensible unit
    fill = np.mean([np.count_nonzero(W.any(axis=2)) / (P * P) for W in blocks.values()])
    assert 0.0 < fill <= 1.0


@pytest.mark.parametrize("s,M,L,seed", [(2, 3, 3.0, 5)])
def test_block_form_adjoint_equals_oracle_vjp(s, M, L, seed):
    """The adjoint in the same block form: with c = 2 v / w per output node,
    g(c1 + D, l1) += sum_p c[D, p] G[D, l1, p]   (G = F2 W, the forward's
    tensor-core product) and g(c2 + D, l2) += (W (f1 x c))[l2], both scattered
    to the shifted cells.  Equals the oracle's VJP (the adjoint of
    collision_mod.f90:213-216) to 1e-13."""
    from oracle.oracle import Oracle
    o = Oracle(s, M, L)
    cap, A, xi, xi1 = o.synth_A(seed=seed, support=1)
    o.set_A(cap, A, xi, xi1)
    P, Nc = o.P, o.Nc
    p = np.repeat(np.arange(o.N), cap) % P
    blocks = {}
    for k in range(len(A)):
        W = blocks.setdefault((int(xi[k] // P), int(xi1[k] // P)), np.zeros((P, P, P)))
        W[xi1[k] % P, xi[k] % P, p[k]] += A[k]
    rng = np.random.default_rng(seed)
    f = o.maxwellian(0.7, 0.4, 0.1, -0.2, 0.9) * (1.0 + 0.05 * rng.standard_normal(o.N))
    v = rng.standard_normal(o.N)
    fc = f.reshape(Nc, P)
    cq = (2.0 * v / o.gwts).reshape(Nc, P)
    cc = _cell3(np.array(o.ccell), M)
    D3 = _cell3(np.arange(Nc), M)
    g = np.zeros((Nc, P))
    for (a, b), W in blocks.items():
        s1 = _cell3(np.array(a), M) + D3 - cc
        s2 = _cell3(np.array(b), M) + D3 - cc
        ok = np.all((s1 >= 0) & (s1 < M) & (s2 >= 0) & (s2 < M), axis=1)
        if not ok.any():
            continue
        i1 = (s1[ok, 0] * M + s1[ok, 1]) * M + s1[ok, 2]
        i2 = (s2[ok, 0] * M + s2[ok, 1]) * M + s2[ok, 2]
        G = np.einsum("dk,klp->dlp", fc[i2], W)
        np.add.at(g, i1, np.einsum("dlp,dp->dl", G, cq[ok]))
        np.add.at(g, i2, np.einsum("klp,dl,dp->dk", W, fc[i1], cq[ok]))
    g = g.ravel()
    ref = o.vjp(f, v)
    assert np.linalg.norm(g - ref) / np.linalg.norm(ref) < 1e-13


@pytest.mark.parametrize("s,M,L,seed", [(2, 3, 3.0, 5), (3, 3, 4.0, 9)])
def test_adjoint_kernel_schedule_equals_oracle_vjp(s, M, L, seed):
    """The schedule of the tensor-core adjoint kernel, restated: a CTA owns a
    target cell T; each block (c1 <= c2) gives two items per valid output
    cell D of its box (the per-axis bounds of the device layout), each with
    records compacted to one of the block's node masks:
      pass 1: T = D + (c1 - cc) (linear indices), side = c(D), operand
              f(D + c2 - cc), records W[n = rank(l1)*P + p, k = l2] (the
              collision operator's own), mask of the nodes l1;
      pass 2: T = D + (c2 - cc), side = c(D), operand f(D + c1 - cc),
              records W2[n = rank(l2)*P + p, k = l1], mask of the nodes l2;
    per row, node l of the mask gets sum_p side[p] * (f W^T)[rank(l)*P + p],
    added to g(T, l).  Equals the oracle's VJP to 1e-13."""
    from oracle.oracle import Oracle
    o = Oracle(s, M, L)
    cap, A, xi, xi1 = o.synth_A(seed=seed, support=1)
    o.set_A(cap, A, xi, xi1)
    P, Nc, cc = o.P, o.Nc, o.ccell
    p = np.repeat(np.arange(o.N), cap) % P
    assert np.all(xi < xi1)
    blocks = {}
    for k in range(len(A)):
        W = blocks.setdefault((int(xi[k] // P), int(xi1[k] // P)), np.zeros((P, P, P)))
        W[xi1[k] % P, xi[k] % P, p[k]] += A[k]
    rng = np.random.default_rng(seed)
    f = o.maxwellian(0.7, 0.4, 0.1, -0.2, 0.9) * (1.0 + 0.05 * rng.standard_normal(o.N))
    v = rng.standard_normal(o.N)
    fc = f.reshape(Nc, P)
    cq = (2.0 * v / o.gwts).reshape(Nc, P)
    c3 = _cell3(np.array(cc), M)
    g = np.zeros((Nc, P))
    partial = 0
    for (a, b), W in blocks.items():
        assert a <= b
        e1, e2 = _cell3(np.array(a), M), _cell3(np.array(b), M)
        lo = np.maximum(0, c3 - np.minimum(e1, e2))
        hi = np.minimum(M - 1, c3 + M - 1 - np.maximum(e1, e2))
        if np.any(hi < lo):
            continue
        present = W.any(axis=2)                       # [l2, l1]
        m1, m2 = np.nonzero(present.any(axis=0))[0], np.nonzero(present.any(axis=1))[0]
        partial += (len(m1) < P) + (len(m2) < P)
        W1 = W[:, m1, :].transpose(1, 2, 0).reshape(len(m1) * P, P)   # [rank(l1)*P + p, l2]
        W2 = W[m2, :, :].transpose(0, 2, 1).reshape(len(m2) * P, P)   # [rank(l2)*P + p, l1]
        o1, o2 = a - cc, b - cc
        for u in range(lo[0], hi[0] + 1):
            for vv in range(lo[1], hi[1] + 1):
                for w in range(lo[2], hi[2] + 1):
                    D = (u * M + vv) * M + w
                    for T, opnd, Wr, nodes in ((D + o1, D + o2, W1, m1), (D + o2, D + o1, W2, m2)):
                        G = (Wr @ fc[opnd]).reshape(len(nodes), P)  # [rank, p]
                        for r, l in enumerate(nodes):
                            g[T, l] += cq[D] @ G[r]
    ref = o.vjp(f, v)
    assert partial > 0  # some blocks use only part of their nodes
    assert np.linalg.norm(g.ravel() - ref) / np.linalg.norm(ref) < 1e-13

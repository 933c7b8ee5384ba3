"""Shared helpers for the test modules (imports stay cheap on CPU-only hosts)."""
import numpy as np


def golden_oracle(g):
    """Oracle on the golden grid with the golden A-arrays loaded."""
    from oracle.oracle import Oracle
    o = Oracle(int(g["s"]), int(g["M"]), float(g["L"]))
    o.set_A(g["capphi"], g["A"], g["A_xi"], g["A_xi1"], one_based=True)
    return o


def mixture_vdf(nodes_u, nodes_v, nodes_w, rng, kmax=4, normalise_w=None):
    """Seeded mixture of 1..kmax Maxwellians: weights ~ Dirichlet(1), bulk
    velocities ~ U[-2,2]^3, temperatures ~ U[0.5,2]; normalised to density 1
    with the quadrature weights when given."""
    k = int(rng.integers(1, kmax + 1))
    wts = rng.dirichlet(np.ones(k))
    f = np.zeros_like(nodes_u)
    for j in range(k):
        u0 = rng.uniform(-2, 2, 3)
        T = rng.uniform(0.5, 2.0)
        r2 = (nodes_u - u0[0]) ** 2 + (nodes_v - u0[1]) ** 2 + (nodes_w - u0[2]) ** 2
        f += wts[j] * np.exp(-r2 / T) / (np.pi * T) ** 1.5
    if normalise_w is not None:
        f /= float(np.sum(f * normalise_w))
    return f

"""Generates tests/golden/physA_s2M2.npz: physical A-arrays on a tiny grid.

Runs the oracle's restatement of SetA_DGV (dgvtools_mod.f90:377-681 with the
Lagrange basis of :254-287 restored) for every basis function of the canonical
cell of the grid s=2, M=2 on [-3,3]^3, and stores the records in the reference
layout (1-based A_xi/A_xi1, A_capphi per node).  ErrChi = ErrEps = 1e-5,
min_sens = 1e-14, Trad = infinity.  Takes a few minutes on 8 cores.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from oracle.oracle import Oracle  # noqa: E402

S, M, L = 2, 2, 3.0
ERR, MIN_SENS = 1e-5, 1e-14


def main(out=os.path.join(HERE, "physA_s2M2.npz")):
    o = Oracle(S, M, L)
    capphi = np.zeros(o.N, np.int32)
    As, xs, x1s = [], [], []
    t0 = time.time()
    for p in range(o.P):
        i1 = o.ccell * o.P + p
        A, xi, xi1 = o.seta(i1, ErrChi=ERR, ErrEps=ERR, min_sens=MIN_SENS)
        capphi[i1] = len(A)
        As.append(A); xs.append(xi + 1); x1s.append(xi1 + 1)
        print(f"basis function {p}: {len(A)} records, {time.time() - t0:.0f}s", flush=True)
    np.savez_compressed(out, s=S, M=M, L=L, err=ERR, min_sens=MIN_SENS, capphi=capphi,
                        A=np.concatenate(As), A_xi=np.concatenate(xs).astype(np.int32),
                        A_xi1=np.concatenate(x1s).astype(np.int32))


if __name__ == "__main__":
    main()

"""Golden RK trajectories of the oracle (the CPU restatement of
TimeIntegratorORK_SH_DGV, time_integr_mod.f90:26-152, around
EvalCollisionPeriodicAPlus_DGV, collision_mod.f90:143-229) for the parity
tests of the batched RK steps.  Test infrastructure: runs the oracle only.

  c1: the 15^3 grid (s=3, M=5, [-6,6]^3), seeded synthetic A-arrays
      (seed 11, support 1), kappa = 1, f0 = two Maxwellians (densities
      0.5/0.5, bulk velocities +/-1.5 along u, temperature 1); RK2 with
      dt = 0.01 for 100 steps; f after steps 1, 10, 50 and 100 and Q(f0).
  c2: the 21^3 grid (s=3, M=7, [-6,6]^3), synthetic A (seed 20260101,
      support 1), kappa = 0.1, f0 = the seeded 1-4 Maxwellian mixture of
      the benchmark's generator (seed 5); RK4 with dt = 0.005, 5 steps (a
      full oracle evaluation at 21^3 takes ~2 minutes on 8 cores); f after
      steps 1 and 5.

Usage: python tests/golden/make_rk_trajectory.py c1|c2  (writes
tests/golden/rk_<case>.npz)."""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def mixture(o, seed):
    """1-4 Maxwellians, weights ~ Dirichlet(1), bulk velocities ~ U[-2,2]^3,
    temperatures ~ U[0.5,2], normalised to density 1 (the benchmark's
    generator)."""
    rng = np.random.default_rng(seed)
    k = int(rng.integers(1, 5))
    wts = rng.dirichlet(np.ones(k))
    f = np.zeros(o.N)
    for j in range(k):
        c = rng.uniform(-2, 2, 3)
        T = rng.uniform(0.5, 2.0)
        f += wts[j] * np.exp(-((o.u - c[0]) ** 2 + (o.v - c[1]) ** 2 + (o.w - c[2]) ** 2) / T) / (np.pi * T) ** 1.5
    return f / float(np.sum(f * o.gwts))


def main(case):
    from oracle.oracle import Oracle
    t0 = time.time()
    if case == "c1":
        grid, seed_a, kappa, dt, order, steps, keep = (3, 5, 6.0), 11, 1.0, 0.01, 2, 100, (1, 10, 50, 100)
        o = Oracle(*grid)
        f = o.maxwellian(1.0, 1.5, 0.0, 0.0, 0.5) + o.maxwellian(1.0, -1.5, 0.0, 0.0, 0.5)
    else:
        grid, seed_a, kappa, dt, order, steps, keep = (3, 7, 6.0), 20260101, 0.1, 0.005, 4, 5, (1, 5)
        o = Oracle(*grid)
        f = mixture(o, 5)
    o.set_A(*o.synth_A(seed=seed_a, support=1))
    out = {"s": grid[0], "M": grid[1], "L": grid[2], "seed_A": seed_a, "kappa": kappa, "dt": dt,
           "order": order, "f0": f.copy(), "q0": o.collide(f)}
    for k in range(1, steps + 1):
        f, _ = o.rk_step(f, dt, order, kappa=kappa)
        if k in keep:
            out[f"f{k}"] = f.copy()
        print(f"{case}: step {k}/{steps} after {time.time() - t0:.0f} s", flush=True)
    out["steps_kept"] = np.array(keep)
    np.savez_compressed(os.path.join(HERE, f"rk_{case}.npz"), **out)


if __name__ == "__main__":
    main(sys.argv[1])

"""Mixed-grid batch in one call (dgv_collide_group): two grids, several VDFs
each, evaluated through one fork/join over the contexts' streams -- eager
first call, captured second call, replays after -- against separate calls and
the oracle (FP64 <= 1e-12, tensor cores <= 1e-6 norm-wise per VDF), replays
following new input values, and launch counts of replays; on the tensor cores
the captured graph holds three kernels for both grids: the f preparation, one
persistent collision kernel and the final step."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def grids():
    import dgv0d3v_direct_collision_b200 as dgv
    from oracle.oracle import Oracle
    out = []
    for (s, M, L, seed) in [(3, 5, 6.0, 11), (3, 3, 4.0, 5)]:
        o = Oracle(s, M, L)
        o.set_A(*o.synth_A(seed=seed, support=1))
        sol = dgv.DGVSolver(s, M, L)
        sol.generate_synthetic_A(seed=seed, support=1)
        out.append((o, sol))
    return out


def _vdfs(o, rng, nb):
    f = np.zeros((nb, o.N))
    for b in range(nb):
        u = rng.uniform(-1.5, 1.5, 3)
        f[b] = o.maxwellian(0.6, *u, 0.7) + o.maxwellian(0.4, *(-u), 1.0)
    return f


@pytest.mark.parametrize("precision,tol", [("f64", 1e-12), ("tc", 1e-6)])
def test_group_matches_oracle_and_replays(grids, precision, tol):
    import torch

    from dgv0d3v_direct_collision_b200 import collide_group
    rng = np.random.default_rng(3)
    nbs = [3, 2]
    fs = [torch.from_numpy(_vdfs(o, rng, nb)).cuda() for (o, _), nb in zip(grids, nbs)]
    qs = [torch.zeros_like(f) for f in fs]
    members = [(sol, f, q) for (_, sol), f, q in zip(grids, fs, qs)]
    for sol in (m[0] for m in members):
        sol.set_kernel_timing(True)
        sol.kernel_stats(reset=True)
    counts = []
    for call in range(4):
        if call == 3:  # new values in the same buffers: the replay reads them
            for (o, _), f, nb in zip(grids, fs, nbs):
                f.copy_(torch.from_numpy(_vdfs(o, rng, nb)))
        collide_group(members, precision=precision)
        counts.append([m[0].kernel_stats(reset=True)["all_launches"] for m in members])
        for (o, sol), f, q in zip(grids, fs, qs):
            fh, qh = f.cpu().numpy(), q.cpu().numpy()
            sep = sol.collide(fh, precision=precision)
            assert rel_err(qh, sep) < 1e-13
            for b in range(fh.shape[0]):
                assert rel_err(qh[b], o.collide(fh[b])) < tol, (call, b)
            sol.kernel_stats(reset=True)  # drop the separate call's launches
    for sol in (m[0] for m in members):
        sol.set_kernel_timing(False)
    # replays count what their capture counted.  (The separate calls with host
    # arrays grow the members' staging buffers, which releases the group's
    # graph once, so call 1 runs eagerly again and call 2 captures.)
    assert counts[2] == counts[3] and sum(counts[3]) > 0
    if precision == "tc":
        # for both grids together: one preparation of the f tiles, one
        # persistent collision kernel and one final kernel, counted on the
        # first member (no projection here)
        assert counts[3] == [3, 0], counts


def test_group_rejects_host_arrays(grids):
    import dgv0d3v_direct_collision_b200 as dgv
    (o, sol) = grids[0]
    f = np.zeros((1, sol.N))
    with pytest.raises(dgv.DGVError):
        dgv.collide_group([(sol, f, f.copy())])

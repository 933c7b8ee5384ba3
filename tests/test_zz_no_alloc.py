"""dgv_collide_f64_noalloc: the FP64 collision operator for callers that must
not allocate device memory after start-up (a driver whose pool allocator
already owns the free memory, or a process under a fixed memory budget).  The
call works in a static device array instead of allocating; these tests call
it through the C-ABI twice in a row and check each result against
dgv_collide_batched and against the oracle (the CPU restatement of
EvalCollisionPeriodicAPlus_DGV, collision_mod.f90:143-229) within the FP64
tolerance of the other parity tests, on grids of 27, 8 and 1 nodes per cell
(one and several slices of output cells), and at a batch so close to the
array's capacity that only one work chunk fits.

Kept in its own module, named so that pytest collects it last."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
LIMIT = 1 << 22  # doubles in the static work array


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b)), float(np.abs(a - b).max() / np.abs(b).max())


def _batch(s, nb, rng):
    u, v, w = s.nodes_u, s.nodes_v, s.nodes_w
    out = np.empty((nb, s.N))
    for b in range(nb):
        c = rng.uniform(-1.5, 1.5, 3)
        T = rng.uniform(0.6, 1.6)
        out[b] = np.exp(-((u - c[0]) ** 2 + (v - c[1]) ** 2 + (w - c[2]) ** 2) / T) / (np.pi * T) ** 1.5
    return out


def _call(L, s, f, q, nb):
    rc = L.dgv_collide_f64_noalloc(s._h, f.data_ptr(), q.data_ptr(), nb, None)
    assert rc == 0, L.dgv_last_error(s._h)


# (s, M, L): 27 nodes per cell in one slice of output cells; 8 nodes per cell
# over 512 cells (two slices); 1 node per cell over 1331 cells (four slices)
GRIDS = [(3, 5, 6.0), (2, 8, 6.0), (1, 11, 6.0)]


@pytest.mark.parametrize("grid", GRIDS, ids=["s3M5", "s2M8", "s1M11"])
def test_noalloc_matches_collide_and_oracle_on_two_calls(grid):
    torch = pytest.importorskip("torch")
    import dgv0d3v_direct_collision_b200 as dgv
    from dgv0d3v_direct_collision_b200 import _lib
    from oracle.oracle import Oracle

    L = _lib.load()
    s_, M_, L_ = grid
    s = dgv.DGVSolver(s_, M_, L_)
    s.generate_synthetic_A(seed=11, support=1)
    o = Oracle(s_, M_, L_)
    o.set_A(*o.synth_A(seed=11, support=1))
    rng = np.random.default_rng(5)
    for call in range(2):  # the second call reuses the array the first one left filled
        fb = _batch(s, 3, rng)
        f = torch.tensor(fb, dtype=torch.float64, device="cuda")
        q = torch.full_like(f, float("nan"))
        _call(L, s, f, q, 3)
        torch.cuda.synchronize()
        got = q.cpu().numpy()
        q_ref = s.EvalCollisionPeriodicAPlus_DGV(fb)
        norm_err, max_err = _rel(got, q_ref)
        assert norm_err < TOL64 and max_err < TOL64, (call, norm_err, max_err)
        norm_err, max_err = _rel(got[call], o.collide(fb[call]))
        assert norm_err < TOL64 and max_err < TOL64, ("oracle", call, norm_err, max_err)
    s.close()


def test_noalloc_at_capacity_and_refusals():
    """nb*N just below the array's capacity (one work chunk fits), the refusal
    above it, host arrays refused, and no change of the device's free memory
    across the first call on a new context (the array was loaded when the
    context was created)."""
    torch = pytest.importorskip("torch")
    import dgv0d3v_direct_collision_b200 as dgv
    from dgv0d3v_direct_collision_b200 import _lib

    L = _lib.load()
    s = dgv.DGVSolver(3, 5, 6.0)
    s.generate_synthetic_A(seed=11, support=1)
    nb = LIMIT // s.N  # 1242 VDFs of 3375 nodes
    rng = np.random.default_rng(9)
    fb = _batch(s, nb, rng)
    f = torch.tensor(fb, dtype=torch.float64, device="cuda")
    q = torch.full_like(f, float("nan"))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for call in range(2):
        _call(L, s, f, q, nb)
        torch.cuda.synchronize()
        if call == 0:
            assert torch.cuda.mem_get_info()[0] == free0
    got = q.cpu().numpy()
    ref = s.EvalCollisionPeriodicAPlus_DGV(fb)
    norm_err, max_err = _rel(got, ref)
    assert norm_err < TOL64 and max_err < TOL64, (norm_err, max_err)

    # sizes beyond the fixed array are refused with a message, nothing launched
    rc = L.dgv_collide_f64_noalloc(s._h, f.data_ptr(), q.data_ptr(), nb + 1, None)
    assert rc == _lib.DGV_EINVAL
    assert b"exceeds the fixed work array" in L.dgv_last_error(s._h)
    # host arrays are refused: staging them would need device memory
    fh = np.zeros(s.N)
    rc = L.dgv_collide_f64_noalloc(s._h, fh.ctypes.data, fh.ctypes.data, 1, None)
    assert rc == _lib.DGV_EINVAL
    s.close()

"""dgv_collide_f64_noalloc: the FP64 collision operator for callers that must
not allocate device memory after start-up (a driver whose pool allocator
already owns the free memory, or a process under a fixed memory budget).  The
call works in a static device array instead of allocating; this test calls it
through the C-ABI twice in a row and checks each result against
dgv_collide_batched within the FP64 tolerance of the other parity tests.

Kept in its own module, named so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b)), float(np.abs(a - b).max() / np.abs(b).max())


def test_noalloc_matches_collide_on_two_calls():
    torch = pytest.importorskip("torch")
    import dgv0d3v_direct_collision_b200 as dgv
    from dgv0d3v_direct_collision_b200 import _lib

    L = _lib.load()
    s = dgv.DGVSolver(3, 5, 6.0)
    s.generate_synthetic_A(seed=11, support=1)
    rng = np.random.default_rng(5)
    u, v, w = s.nodes_u, s.nodes_v, s.nodes_w

    def batch(nb):
        out = np.empty((nb, s.N))
        for b in range(nb):
            c = rng.uniform(-1.5, 1.5, 3)
            T = rng.uniform(0.6, 1.6)
            out[b] = np.exp(-((u - c[0]) ** 2 + (v - c[1]) ** 2 + (w - c[2]) ** 2) / T) / (np.pi * T) ** 1.5
        return out

    for call in range(2):  # the second call reuses the array the first one left filled
        fb = batch(3)
        f = torch.tensor(fb, dtype=torch.float64, device="cuda")
        q = torch.full_like(f, float("nan"))
        rc = L.dgv_collide_f64_noalloc(s._h, f.data_ptr(), q.data_ptr(), 3, None)
        assert rc == 0, L.dgv_last_error(s._h)
        torch.cuda.synchronize()
        q_ref = s.EvalCollisionPeriodicAPlus_DGV(fb)
        norm_err, max_err = _rel(q.cpu().numpy(), q_ref)
        assert norm_err < TOL64 and max_err < TOL64, (call, norm_err, max_err)

    # sizes beyond the fixed array are refused with a message, nothing launched
    big = torch.zeros((2, s.N), dtype=torch.float64, device="cuda")
    rc = L.dgv_collide_f64_noalloc(s._h, big.data_ptr(), big.data_ptr(), 2000, None)
    assert rc == _lib.DGV_EINVAL
    assert b"exceeds the fixed work array" in L.dgv_last_error(s._h)
    # host arrays are refused: staging them would need device memory
    fh = np.zeros(s.N)
    rc = L.dgv_collide_f64_noalloc(s._h, fh.ctypes.data, fh.ctypes.data, 1, None)
    assert rc == _lib.DGV_EINVAL

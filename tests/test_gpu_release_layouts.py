"""dgv_release_layouts: the FP32 rows and the tensor-core record sets can be
freed when a caller does not need them; each is rebuilt on its next use with
the same values, so results after a release equal those before, bit for bit
(FP32-compensated Q, block-form Q and adjoint, chunk-form Q), and the device's
free memory grows by about the layout's size.  Grid: 15^3 (s=3, M=5,
[-6,6]^3), seeded synthetic A-arrays."""
import numpy as np
import pytest

from helpers import mixture_vdf

pytestmark = pytest.mark.gpu


def test_release_and_rebuild_give_the_same_results():
    import torch

    import dgv0d3v_direct_collision_b200 as m
    from dgv0d3v_direct_collision_b200 import _lib
    s = m.DGVSolver(3, 5, 6.0)
    try:
        s.generate_synthetic_A(seed=11, support=1)
        s.set_nchunks(64)
        s.set_tc_tiles_per_cta(2)  # a fixed launch choice: no tuning between the calls
        s.set_tc_set_mb(48)
        rng = np.random.default_rng(5)
        fs = np.stack([mixture_vdf(s.nodes_u, s.nodes_v, s.nodes_w, rng, normalise_w=s.nodes_gwts) for _ in range(140)])
        vs = rng.standard_normal(fs.shape)
        q32 = s.EvalCollisionPeriodicAPlus_DGV(fs[:3], precision="f32c")
        qtc = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
        gtc = s.vjp(fs, vs, precision="tc")
        info = s.A_info()
        freed = s.release_layouts(f32=True, tc_block=True)
        # FP32 rows: pairs x 32 words (P = 27); block records: >= 40 % of the dense 96 KB per block
        assert freed >= 0.9 * (info["pairs"] * 32 * 4 + 0.4 * info["blocks"] * 96 * 1024)
        assert np.array_equal(s.EvalCollisionPeriodicAPlus_DGV(fs[:3], precision="f32c"), q32)
        assert np.array_equal(s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc"), qtc)
        assert np.array_equal(s.vjp(fs, vs, precision="tc"), gtc)
        # the adjoint's records alone
        assert s.release_layouts(tc_adjoint=True) > 0
        assert np.array_equal(s.vjp(fs, vs, precision="tc"), gtc)
        # the chunk form
        s.set_tc_form(1)
        qc = s.EvalCollisionPeriodicAPlus_DGV(fs[:40], precision="tc")
        assert s.release_layouts(tc_chunk=True) > 0
        assert np.array_equal(s.EvalCollisionPeriodicAPlus_DGV(fs[:40], precision="tc"), qc)
        s.set_tc_form(2)
        # unknown bits are refused
        L = _lib.load()
        assert L.dgv_release_layouts(s._h, 64, None) == _lib.DGV_EINVAL
        # an RK step after a release (its captured graph was released with the layouts)
        f = torch.tensor(fs[:2], device="cuda")
        s.TimeIntegratorORK_SH_DGV(f, 0.01, order=2, precision="tc")
        s.release_layouts(tc_block=True)
        g = torch.tensor(fs[:2], device="cuda")
        s.TimeIntegratorORK_SH_DGV(g, 0.01, order=2, precision="tc")
        assert torch.equal(f, g)
    finally:
        s.close()

"""One persistent launch of the block-form kernel (DGV_OPT_TCPERSIST = 1)
against one launch per block set: one CTA per SM walks (block set, row tile,
VDF-tile pair) units in set order, and per-warp flags make each unit's FP64
sums enter the accumulators after those of the same rows' previous set -- the
order of the per-set launches -- so forward and adjoint results are the same
bit for bit.  Cases: batches of 37 (one VDF tile of 64), 256 (two tiles of
128) and 300 (three tiles: with two per CTA the last pair holds one tile, so
the library uses one launch per set; with one per CTA it is persistent), 8 MB
of records per set (many sets, many flag waits), the adjoint, and a bounded
wait that runs out inside a persistent launch (the call returns
DGV_ETIMEOUT, the context stays usable).  Grid: 15^3 (s=3, M=5,
[-6,6]^3), seeded synthetic A-arrays."""
import time

import numpy as np
import pytest

from conftest import rel_err
from helpers import mixture_vdf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sol():
    import dgv0d3v_direct_collision_b200 as m
    s = m.DGVSolver(3, 5, 6.0)
    s.generate_synthetic_A(seed=11, support=1)
    yield s
    s.close()


def _fs(s, n, seed):
    rng = np.random.default_rng(seed)
    return np.stack([mixture_vdf(s.nodes_u, s.nodes_v, s.nodes_w, rng, normalise_w=s.nodes_gwts) for _ in range(n)])


@pytest.mark.parametrize("nb,tiles,mb", [(37, 2, 48), (256, 2, 48), (300, 2, 48), (300, 1, 48), (256, 2, 8)])
def test_persistent_equals_per_set_launches(sol, nb, tiles, mb):
    s = sol
    fs = _fs(s, nb, nb + tiles + mb)
    s.set_tc_tiles_per_cta(tiles)
    s.set_tc_set_mb(mb)
    s.set_tc_persistent(False)
    q_sets = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    n_sets = s.tc_plan(nb)["launches"]
    s.set_tc_persistent(True)
    q_pers = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    nbt = (nb + 127) // 128 if nb > 64 else 1
    uniform = nbt <= tiles or nbt % tiles == 0
    # a batch whose VDF-tile pairs hold different numbers of tiles (3 tiles, 2
    # per CTA) is served by one launch per set instead
    assert s.tc_plan(nb)["launches"] == (1 if uniform else n_sets) and n_sets >= 1
    assert np.array_equal(q_pers, q_sets)
    q64 = s.EvalCollisionPeriodicAPlus_DGV(fs[:4])
    assert rel_err(q_pers[:4], q64) < 1e-6


@pytest.mark.parametrize("nb", [40, 256])
def test_persistent_adjoint_equals_per_set_launches(sol, nb):
    s = sol
    fs = _fs(s, nb, 5 + nb)
    vs = np.random.default_rng(nb).standard_normal(fs.shape)
    s.set_tc_tiles_per_cta(2)
    s.set_tc_set_mb(48)
    s.set_tc_persistent(False)
    g_sets = s.vjp(fs, vs, precision="tc")
    s.set_tc_persistent(True)
    g_pers = s.vjp(fs, vs, precision="tc")
    assert np.array_equal(g_pers, g_sets)
    g64 = s.vjp(fs[0], vs[0])
    assert rel_err(g_pers[0], g64) < 1e-6


def test_persistent_wait_runs_out_and_context_stays_usable(sol):
    from dgv0d3v_direct_collision_b200 import _lib
    s = sol
    L = _lib.load()
    fs = _fs(s, 256, 77)
    s.set_tc_tiles_per_cta(2)
    s.set_tc_set_mb(8)
    s.set_tc_persistent(True)
    q_ref = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    assert L.dgv_set_option(s._h, _lib.DGV_OPT_WAIT_LIMIT_US, 20000) == 0  # 20 ms
    assert L.dgv_set_option(s._h, _lib.DGV_OPT_TEST_WITHHOLD, 1) == 0
    t = time.perf_counter()
    with pytest.raises(_lib.DGVError) as ei:
        s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    assert ei.value.code == _lib.DGV_ETIMEOUT
    assert time.perf_counter() - t < 10.0
    assert L.dgv_set_option(s._h, _lib.DGV_OPT_WAIT_LIMIT_US, 0) == 0
    assert np.array_equal(s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc"), q_ref)

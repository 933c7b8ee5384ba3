"""The bounded waits of the block-form tensor-core kernel.  Every mbarrier wait
gives up after a limit of device time (DGV_OPT_WAIT_LIMIT_US, default 4 s),
raises the context's host-mapped error flag, and every role of the kernel
drains what it issued, frees tensor memory and leaves; the call returns
DGV_ETIMEOUT.  The test makes one wait run out without a fault: with
DGV_OPT_TEST_WITHHOLD the first CTA arms no copy for one stage of its W ring,
so the MMA thread's wait on that stage (and then every wait behind it) runs
out.  Afterwards the same context computes normally: the flag is cleared and
no state is left behind."""
import time

import numpy as np
import pytest

from conftest import rel_err
from helpers import mixture_vdf

pytestmark = pytest.mark.gpu


def test_wait_runs_out_and_context_stays_usable():
    import dgv0d3v_direct_collision_b200 as m
    from dgv0d3v_direct_collision_b200 import _lib
    L = _lib.load()
    s = m.DGVSolver(3, 5, 6.0)
    s.generate_synthetic_A(seed=11, support=1)
    rng = np.random.default_rng(4)
    fs = np.stack([mixture_vdf(s.nodes_u, s.nodes_v, s.nodes_w, rng, normalise_w=s.nodes_gwts) for _ in range(40)])
    vs = rng.standard_normal(fs.shape)
    q_ref = s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
    g_ref = s.vjp(fs, vs, precision="tc")
    for which in ("collide", "vjp"):
        assert L.dgv_set_option(s._h, _lib.DGV_OPT_WAIT_LIMIT_US, 20000) == 0  # 20 ms
        assert L.dgv_set_option(s._h, _lib.DGV_OPT_TEST_WITHHOLD, 1) == 0
        t = time.perf_counter()
        with pytest.raises(_lib.DGVError) as ei:
            if which == "collide":
                s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc")
            else:
                s.vjp(fs, vs, precision="tc")
        elapsed = time.perf_counter() - t
        assert ei.value.code == _lib.DGV_ETIMEOUT, which
        assert elapsed < 10.0, (which, elapsed)
        assert L.dgv_set_option(s._h, _lib.DGV_OPT_WAIT_LIMIT_US, 0) == 0
        # the same context, the default limit: the results of before
        assert rel_err(s.EvalCollisionPeriodicAPlus_DGV(fs, precision="tc"), q_ref) < 1e-12, which
        assert rel_err(s.vjp(fs, vs, precision="tc"), g_ref) < 1e-12, which
    s.close()

"""RK4 relaxation in the FP32-compensated and FP64 paths side by side (the
21^3 RK4 case, here at 15^3 and 60 steps; `bench.py --trajectory` runs the
full 500 steps at 21^3): at every step Q of both paths on the FP64 state
agrees to 1e-6, the two trajectories' changes since the start agree to 1e-6,
and with the conservation projection on, the moments n, u, T of both drift by
round-off only (1e-12).  The FP64 RK steps themselves are pinned to the oracle
in test_gpu_parity.py.  Seeded synthetic A-arrays, seeded Maxwellian mixture."""
import numpy as np
import pytest

from conftest import rel_err
from helpers import mixture_vdf

pytestmark = pytest.mark.gpu


def test_rk4_f32c_vs_f64_trajectory():
    import torch

    import dgv0d3v_direct_collision_b200 as dgv
    kappa, dt, steps = 0.1, 0.005, 60
    s = dgv.DGVSolver(3, 5, 6.0, kappa=kappa)
    s.generate_synthetic_A(seed=11, support=1)
    s.set_projection(True)
    f0 = mixture_vdf(s.nodes_u, s.nodes_v, s.nodes_w, np.random.default_rng(21), normalise_w=s.nodes_gwts)
    f64 = torch.from_numpy(f0.copy()).cuda()
    f32 = f64.clone()
    r64, r32 = torch.zeros_like(f64), torch.zeros_like(f64)
    m0 = np.array(s.MassCheckRec(f0))
    for k in range(1, steps + 1):
        fh = f64.cpu().numpy()
        q64 = s.EvalCollisionPeriodicAPlus_DGV(fh, precision="f64")
        q32 = s.EvalCollisionPeriodicAPlus_DGV(fh, precision="f32c")
        assert rel_err(q32, q64) < 1e-6, k
        s.TimeIntegratorORK_SH_DGV(f64, dt, frhs1=r64, order=4, precision="f64")
        s.TimeIntegratorORK_SH_DGV(f32, dt, frhs1=r32, order=4, precision="f32c")
        a, b = f64.cpu().numpy(), f32.cpu().numpy()
        assert rel_err(b - f0, a - f0) < 1e-6, k
        for m in (np.array(s.MassCheckRec(a)), np.array(s.MassCheckRec(b))):
            assert np.all(np.abs(m - m0) <= 1e-12 * np.maximum(1.0, np.abs(m0))), (k, m - m0)
    assert rel_err(f64.cpu().numpy(), f0) > 1e-4  # the state did move

"""Batched RK steps (dgv_step_rk_batched): TimeIntegratorORK_SH_DGV
(time_integr_mod.f90:26-152) for many VDFs, each stage's Q evaluated for the
whole batch in one call, captured into a CUDA graph from the second call.

Against: the single-VDF steps (FP64, 1e-12), the oracle's trajectories in the
committed fixtures (tests/golden/make_rk_trajectory.py):
  C1 -- 15^3 (s=3, M=5, [-6,6]^3), two Maxwellians +/-1.5 u, RK2, dt = 0.01,
        100 steps: FP64 <= 1e-12 of f and <= 1e-10 of f - f0 at steps 1, 10,
        50, 100; tensor cores <= 1e-6 of f - f0;
  C2 -- 21^3 (s=3, M=7, [-6,6]^3), a seeded Maxwellian mixture, RK4 with
        dt = 0.005, 5 steps: FP64 <= 1e-12, FP32-compensated and tensor
        cores <= 1e-6 of f - f0 after steps 1 and 5.
Both with seeded synthetic A-arrays (generated the same way on both sides)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err
from helpers import mixture_vdf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1s():
    import dgv0d3v_direct_collision_b200 as m
    s = m.DGVSolver(3, 5, 6.0, kappa=1.0)
    s.generate_synthetic_A(seed=11, support=1)
    yield s
    s.close()


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5])
def test_batched_rk_equals_single_vdf_steps_f64(c1s, order):
    import torch
    s = c1s
    rng = np.random.default_rng(order)
    fs = np.stack([mixture_vdf(s.nodes_u, s.nodes_v, s.nodes_w, rng, normalise_w=s.nodes_gwts) for _ in range(5)])
    fb = torch.tensor(fs, device="cuda")
    rb = torch.zeros_like(fb)
    s.TimeIntegratorORK_SH_DGV(fb, 0.01, frhs1=rb, order=order, precision="f64")
    for k in range(5):
        f1 = torch.tensor(fs[k], device="cuda")
        r1 = torch.zeros_like(f1)
        s.TimeIntegratorORK_SH_DGV(f1, 0.01, frhs1=r1, order=order, precision="f64")
        assert rel_err(fb[k].cpu().numpy(), f1.cpu().numpy()) < 1e-13, k
        assert rel_err(fb[k].cpu().numpy() - fs[k], f1.cpu().numpy() - fs[k]) < 1e-12, k
        assert rel_err(rb[k].cpu().numpy(), r1.cpu().numpy()) < 1e-12, k


def test_batched_rk_tensor_cores_graph_replays(c1s):
    """130 VDFs (tiles of 128), RK4 on the tensor cores: the eager call, the
    captured call and two replays each match the FP64 batch step from the
    same state within 1e-6 of the increment."""
    import torch
    s = c1s
    rng = np.random.default_rng(42)
    fs = np.stack([mixture_vdf(s.nodes_u, s.nodes_v, s.nodes_w, rng, normalise_w=s.nodes_gwts) for _ in range(130)])
    ftc = torch.tensor(fs, device="cuda")
    r = torch.zeros_like(ftc)
    for call in range(4):
        f0 = ftc.clone()
        s.TimeIntegratorORK_SH_DGV(ftc, 0.01, frhs1=r, order=4, precision="tc")
        f64 = f0.clone()
        s.TimeIntegratorORK_SH_DGV(f64, 0.01, order=4, precision="f64")
        a, b, z = ftc.cpu().numpy(), f64.cpu().numpy(), f0.cpu().numpy()
        for k in (0, 1, 127, 128, 129):
            assert rel_err(a[k] - z[k], b[k] - z[k]) < 1e-6, (call, k)


def test_batched_rk_refused_with_run_modes(c1s):
    import torch
    from dgv0d3v_direct_collision_b200 import _lib
    s = c1s
    f = torch.tensor(np.stack([s.maxwelveldist(1.0, 0.1 * k, 0, 0, 1.0) for k in range(2)]), device="cuda")
    s.set_regime(0.1, 0.01)
    try:
        with pytest.raises(_lib.DGVError) as ei:
            s.TimeIntegratorORK_SH_DGV(f, 0.01, order=2)
        assert ei.value.code == _lib.DGV_EUNSUP
    finally:
        s.set_regime(0.0, 0.0)


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLDEN, "rk_c1.npz")), reason="fixture missing")
def test_c1_rk2_100_steps_vs_oracle_trajectory():
    import torch

    import dgv0d3v_direct_collision_b200 as m
    g = dict(np.load(os.path.join(GOLDEN, "rk_c1.npz")))
    s = m.DGVSolver(int(g["s"]), int(g["M"]), float(g["L"]), kappa=float(g["kappa"]))
    s.generate_synthetic_A(seed=int(g["seed_A"]), support=1)
    f0 = g["f0"]
    assert rel_err(s.EvalCollisionPeriodicAPlus_DGV(f0), g["q0"]) < 1e-12
    # FP64: one VDF (dgv_step_rk) and the same VDF twice in a batch
    f1 = torch.tensor(f0, device="cuda")
    fb = torch.tensor(np.stack([f0, f0]), device="cuda")
    ftc = torch.tensor(np.stack([f0, f0]), device="cuda")
    for k in range(1, 101):
        s.TimeIntegratorORK_SH_DGV(f1, float(g["dt"]), order=2, precision="f64")
        s.TimeIntegratorORK_SH_DGV(fb, float(g["dt"]), order=2, precision="f64")
        s.TimeIntegratorORK_SH_DGV(ftc, float(g["dt"]), order=2, precision="tc")
        if f"f{k}" in g:
            ref = g[f"f{k}"]
            for got in (f1.cpu().numpy(), fb[0].cpu().numpy(), fb[1].cpu().numpy()):
                assert rel_err(got, ref) < 1e-12, k
                assert rel_err(got - f0, ref - f0) < 1e-10, k
            assert rel_err(ftc[1].cpu().numpy() - f0, ref - f0) < 1e-6, k
    s.close()


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLDEN, "rk_c2.npz")), reason="fixture missing")
def test_c2_rk4_5_steps_21cubed_vs_oracle():
    import torch

    import dgv0d3v_direct_collision_b200 as m
    g = dict(np.load(os.path.join(GOLDEN, "rk_c2.npz")))
    s = m.DGVSolver(int(g["s"]), int(g["M"]), float(g["L"]), kappa=float(g["kappa"]))
    s.generate_synthetic_A(seed=int(g["seed_A"]), support=1)
    f0 = g["f0"]
    assert rel_err(s.EvalCollisionPeriodicAPlus_DGV(f0), g["q0"]) < 1e-12
    kept = [int(k) for k in g["steps_kept"]]
    for prec, tol in (("f64", 1e-12), ("f32c", 1e-6), ("tc", 1e-6)):
        f = torch.tensor(np.stack([f0, f0]) if prec == "tc" else f0, device="cuda")
        for k in range(1, max(kept) + 1):
            s.TimeIntegratorORK_SH_DGV(f, float(g["dt"]), order=4, precision=prec)
            if k in kept:
                ref = g[f"f{k}"]
                got = f.cpu().numpy()
                got = got[0] if got.ndim == 2 else got
                assert rel_err(got - f0, ref - f0) < tol, (prec, k)
                if prec == "f64":
                    assert rel_err(got, ref) < 1e-12, k
    s.close()

"""torch.autograd wrappers of the collision operator and of the RK steps.

``collision(f, solver)`` is Q(f,f) (``EvalCollisionPeriodicAPlus_DGV``,
collision_mod.f90:143-229) as a differentiable torch op: its backward is the
library's vector-Jacobian product (the adjoint of collision_mod.f90:213-216):
for a forward on the tensor cores the batched tensor-core VJP
(``dgv_vjp_batched``), otherwise the FP64 VJP.  ``rk_step`` is one step of ``TimeIntegratorORK_SH_DGV``
(time_integr_mod.f90:26-152) with the reference's stage coefficients; its
backward is the discrete adjoint of the step.  Only the step's input is kept
(a checkpoint); the backward recomputes the stages and walks them in reverse,
one VJP per stage.  ``rk_trajectory`` chains steps, so memory grows with the
number of steps by one state each.

The solver argument needs ``collide(f, out, precision=)``, ``vjp(f, v, out)``
(with ``precision=`` for the tensor-core backward) and ``kappa``; a ``DGVSolver`` (device tensors, used in place) is the
intended one.  The FP64 conservation projection has no adjoint here: the
wrappers refuse a solver with the projection switched on.
"""
from __future__ import annotations

import torch

# Explicit stage form of the reference's RK schemes: k_i = kappa*dt*Q(s_i),
# s_i = f + sum_j A[i][j] k_j, f_new = f + sum_i B[i] k_i.  Coefficients as in
# time_integr_mod.f90:55-57 (RK2), :76-82 (RK3), :97-104 (RK4), :124-146 (RK5);
# RK5's combined stage ft3 = -k2/5 + 546/625 k3 is expanded.
RK_TABLEAUX = {
    1: ([[]], [1.0]),
    2: ([[], [2.0 / 3.0]], [1.0 / 4.0, 3.0 / 4.0]),
    3: ([[], [1.0 / 2.0], [0.0, 3.0 / 4.0]], [2.0 / 9.0, 3.0 / 9.0, 4.0 / 9.0]),
    4: ([[], [1.0 / 2.0], [1.0 / 4.0, 1.0 / 4.0], [0.0, -1.0, 2.0]],
        [1.0 / 6.0, 0.0, 2.0 / 3.0, 1.0 / 6.0]),
    5: ([[], [1.0 / 2.0], [1.0 / 4.0, 1.0 / 4.0], [0.0, -1.0, 2.0],
         [7.0 / 27.0, 10.0 / 27.0, 0.0, 1.0 / 27.0],
         [28.0 / 625.0, -1.0 / 5.0, 546.0 / 625.0, 54.0 / 625.0, -378.0 / 625.0]],
        [1.0 / 24.0, 0.0, 0.0, 5.0 / 48.0, 27.0 / 56.0, 125.0 / 336.0]),
}


def _check_solver(solver):
    if getattr(solver, "projection", False):
        raise ValueError("autograd wrappers: switch the conservation projection off (it has no adjoint here)")


def _rows(x):
    return x.reshape(-1, x.shape[-1]) if x.dim() > 1 else x.reshape(1, -1)


def _sync(x):
    # the library works on its own stream and returns when its work is done;
    # torch's kernels producing x may still be running on torch's stream
    if x.is_cuda:
        torch.cuda.current_stream(x.device).synchronize()


def _q(solver, f, scale, precision):
    f = f.contiguous()
    q = torch.empty_like(f)
    _sync(f)
    solver.collide(f, q, precision=precision)
    return q * scale if scale != 1.0 else q


def _vjp(solver, f, v, scale, precision="f64"):
    """scale * J(f)^T v: the whole batch in one tensor-core call when the
    forward ran on the tensor cores (dgv_vjp_batched, DGV_PREC_TC), else the
    FP64 VJP row by row"""
    fr, vr = _rows(f.contiguous()), _rows(v.contiguous())
    g = torch.empty_like(fr)
    _sync(fr)
    _sync(vr)
    if precision == "tc":
        solver.vjp(fr, vr, g, precision="tc")
    else:
        for b in range(fr.shape[0]):
            solver.vjp(fr[b].contiguous(), vr[b].contiguous(), g[b])
    g = g.reshape(f.shape)
    return g * scale if scale != 1.0 else g


class _Collision(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f, solver, scale, precision):
        ctx.solver, ctx.scale, ctx.precision = solver, scale, precision
        ctx.save_for_backward(f)
        return _q(solver, f, scale, precision)

    @staticmethod
    def backward(ctx, gq):
        (f,) = ctx.saved_tensors
        return _vjp(ctx.solver, f, gq, ctx.scale, ctx.precision), None, None, None


def collision(f: torch.Tensor, solver, scale: float = 1.0, precision: str = "f64") -> torch.Tensor:
    """scale * Q(f,f) for f of shape (N,) or (B, N), float64; differentiable in f."""
    _check_solver(solver)
    if f.dtype != torch.float64:
        raise TypeError("collision: f must be float64")
    return _Collision.apply(f, solver, float(scale), precision)


def _stages(solver, f, dt, order, precision):
    A, _ = RK_TABLEAUX[order]
    h = solver.kappa * dt
    s_list, k_list = [], []
    for i in range(len(A)):
        s = f.clone()
        for j, a in enumerate(A[i]):
            if a != 0.0:
                s = s + a * k_list[j]
        s_list.append(s)
        k_list.append(_q(solver, s, h, precision))
    return s_list, k_list


class _RKStep(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f, solver, dt, order, precision):
        ctx.solver, ctx.dt, ctx.order, ctx.precision = solver, dt, order, precision
        ctx.save_for_backward(f)  # checkpoint: stages are recomputed in backward
        _, k_list = _stages(solver, f, dt, order, precision)
        _, B = RK_TABLEAUX[order]
        out = f.clone()
        for b, k in zip(B, k_list):
            if b != 0.0:
                out = out + b * k
        return out

    @staticmethod
    def backward(ctx, gout):
        (f,) = ctx.saved_tensors
        solver, dt, order = ctx.solver, ctx.dt, ctx.order
        A, B = RK_TABLEAUX[order]
        s_list, _ = _stages(solver, f, dt, order, ctx.precision)
        h = solver.kappa * dt
        ns = len(A)
        s_bar = [None] * ns
        gf = gout.clone()
        for i in reversed(range(ns)):
            k_bar = B[i] * gout
            for m in range(i + 1, ns):
                if i < len(A[m]) and A[m][i] != 0.0:
                    k_bar = k_bar + A[m][i] * s_bar[m]
            s_bar[i] = _vjp(solver, s_list[i], k_bar, h, ctx.precision)
            gf = gf + s_bar[i]
        return gf, None, None, None, None


def rk_step(f: torch.Tensor, solver, dt: float, order: int = 2, precision: str = "f64") -> torch.Tensor:
    """One RK step (orders 1-5, the reference's coefficients) of df/dt = kappa Q(f,f);
    differentiable, with the step input as the only saved state."""
    _check_solver(solver)
    if order not in RK_TABLEAUX:
        raise ValueError("rk_step: order must be 1..5")
    if f.dtype != torch.float64:
        raise TypeError("rk_step: f must be float64")
    return _RKStep.apply(f, solver, float(dt), int(order), precision)


def rk_trajectory(f: torch.Tensor, solver, dt: float, nsteps: int, order: int = 2,
                  precision: str = "f64") -> torch.Tensor:
    """nsteps RK steps; the backward recomputes each step from its saved input."""
    for _ in range(nsteps):
        f = rk_step(f, solver, dt, order, precision)
    return f

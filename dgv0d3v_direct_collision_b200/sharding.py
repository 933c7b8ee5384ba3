"""Multi-GPU partitioning of the collision workload (one process per GPU).

* Batches of VDFs are independent: `vdf_shard` gives each rank a contiguous,
  balanced slice and no collective touches the data path.
* A single large VDF is split by output cells, as the reference splits output
  nodes over MPI ranks (miscmpiset.f90:195-200, 1017-1098): every rank holds the
  full f and the full A-arrays, evaluates Q on its cells and one all-gather
  assembles Q -- the reference's bcast(f) + reduce(SUM) pair
  (spat_oper_mod.f90:118, 139) becomes a single gather of disjoint slices.
"""
from __future__ import annotations


def balanced_range(n: int, world: int, rank: int):
    """[start, stop) of rank's share of n items (sizes differ by at most 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    base, rem = divmod(n, world)
    start = rank * base + min(rank, rem)
    return start, start + base + (1 if rank < rem else 0)


def vdf_shard(nvdf: int, world: int, rank: int):
    return balanced_range(nvdf, world, rank)


def node_shard(Nc: int, P: int, world: int, rank: int):
    """Node range [start, stop) of rank's output cells (whole cells, so all P
    basis functions of a cell stay on one rank)."""
    c0, c1 = balanced_range(Nc, world, rank)
    return c0 * P, c1 * P


def gather_node_slices(q_local, Nc: int, P: int, group=None):
    """All-gather disjoint node slices of Q (torch tensors) into the full vector."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    sizes = [node_shard(Nc, P, world, r) for r in range(world)]
    width = max(b - a for a, b in sizes)
    buf = torch.zeros(width, dtype=q_local.dtype, device=q_local.device)
    buf[: q_local.numel()] = q_local
    out = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(out, buf, group=group)
    return torch.cat([o[: b - a] for o, (a, b) in zip(out, sizes)])


def sharded_collide(solver, f, group=None, precision: str = "f64"):
    """Q(f,f) of one VDF split over the ranks of `group` by output cells:
    every rank holds the full f and A, evaluates its balanced share of cells
    (dgv_collide_cells) and one all-gather assembles Q on every rank."""
    import torch
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    c0, c1 = balanced_range(solver.Nc, world, rank)
    if f.is_cuda:  # the library runs on its own stream; f may still be in flight on torch's
        torch.cuda.current_stream(f.device).synchronize()
    q_local = solver.collide_cells(f.contiguous(), c0, c1, precision=precision)
    return gather_node_slices(q_local, solver.Nc, solver.P, group)


def sharded_rk_step(solver, f, dt: float, order: int = 2, group=None, precision: str = "f64"):
    """One RK step (the reference's schemes, explicit stage form) of a single
    VDF sharded by output cells: one all-gather per stage, f replicated."""
    from .autograd import RK_TABLEAUX
    A, B = RK_TABLEAUX[order]
    h = solver.kappa * dt
    ks = []
    for i in range(len(A)):
        s = f
        for j, a in enumerate(A[i]):
            if a != 0.0:
                s = s + a * ks[j]
        ks.append(h * sharded_collide(solver, s, group, precision))
    out = f
    for b, k in zip(B, ks):
        if b != 0.0:
            out = out + b * k
    return out

"""Benchmark: Q(f,f) evaluations per second at 27^3 nodes, batch 256.

Workload (one step): one batched evaluation of the collision operator for 256
velocity distributions on the grid s=3 nodes x M=9 cells per axis on
[-7,7]^3 (N = 19683 nodes), A-arrays = seeded synthetic records with the
reference's index structure (generated on the device), VDFs = seeded mixtures
of 1-4 Maxwellians (weights ~ Dirichlet(1), bulk velocities ~ U[-2,2]^3,
temperatures ~ U[0.5,2], density 1).  The headline arm is the batched
tensor-core path (split-fp16 operands, compensated accumulation) with the FP64
conservation projection; the plain FP64 path is timed beside it on the first
32 VDFs of the same batch, and the error of the tensor-core path against it
is stated.

Multi-GPU: one process per GPU (torchrun); each rank evaluates its own 256
VDFs (weak scaling, no data-path collective); time = max over ranks.

`--impl reference` times the CPU restatement of the reference's collision loop
(oracle/, EvalCollisionPeriodicAPlus_DGV collision_mod.f90:143-229) on the
host cores, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

S, M, L = 3, 9, 7.0
BATCH = 256
SEED_A = 20260101
METRIC = "Q(f,f) evals/s at 27^3 batch 256: batched FP32 vs plain FP64 GPU, err<=1e-6"
WORKLOAD = "27^3 nodes (s=3, M=9, [-7,7]^3) x 256 VDFs, one batched Q(f,f) evaluation per step"


def mixture_batch(u, v, w, gwts, n, seed):
    rng = np.random.default_rng(seed)
    out = np.empty((n, len(u)))
    for b in range(n):
        k = int(rng.integers(1, 5))
        wts = rng.dirichlet(np.ones(k))
        f = np.zeros(len(u))
        for j in range(k):
            c = rng.uniform(-2, 2, 3)
            T = rng.uniform(0.5, 2.0)
            f += wts[j] * np.exp(-((u - c[0]) ** 2 + (v - c[1]) ** 2 + (w - c[2]) ** 2) / T) / (np.pi * T) ** 1.5
        out[b] = f / float(np.sum(f * gwts))
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def balanced_cells(Mc: int):
    """The M^2 cells (u, v, w) of an M^3 grid with (u + 2v + 4w) mod M == 0
    (M odd): every (u, v) once, every w value M times, so boundary and
    interior cells (whose per-node cost differs by the number of valid
    shifts) appear in their grid proportions; in a seeded random order."""
    cells = [(u * Mc + v) * Mc + w for u in range(Mc) for v in range(Mc) for w in range(Mc)
             if (u + 2 * v + 4 * w) % Mc == 0]
    return np.random.default_rng(0).permutation(np.array(cells))


def synth_A_some(o, ps):
    """The oracle's synthetic records of the basis functions ps only (the
    records of one basis function are only read by the nodes of that basis
    function, collision_mod.f90:186-188), in the reference layout."""
    parts = {p: o.synth_A(seed=SEED_A, support=1, p_only=p) for p in ps}
    cap = np.sum([q[0] for q in parts.values()], axis=0).astype(np.int32)
    ordered = [parts[p] for p in sorted(ps)]  # records in node order
    A = np.concatenate([q[1] for q in ordered])
    xi = np.concatenate([q[2] for q in ordered])
    xi1 = np.concatenate([q[3] for q in ordered])
    return cap, A, xi, xi1


class CpuBaseline:
    """Oracle (CPU restatement of EvalCollisionPeriodicAPlus_DGV) on a sample
    of output nodes of the same workload.  All nodes of one basis function
    scan the same record list, so time per node x N gives the time of one
    full evaluation.  The sample: the balanced cells of the grid at three
    basis functions (243 nodes at 27^3, ~15 rounds of 16 threads, so the
    threads idle at the end of the last round matter little).  Set up once
    (grid, synthetic A of those basis functions, f), then timed as often as
    asked."""
    P_SAMPLE = (4, 13, 22)

    def __init__(self, nthreads: int = 0):
        from oracle.oracle import Oracle
        self.o = Oracle(S, M, L)
        self.o.set_A(*synth_A_some(self.o, self.P_SAMPLE))
        self.f = mixture_batch(self.o.u, self.o.v, self.o.w, self.o.gwts, 1, 7)[0]
        self.cores = nthreads or os.cpu_count()
        self.nodes_all = np.array([c * self.o.P + p for c in balanced_cells(M) for p in self.P_SAMPLE])
        self.n = None

    def sample(self, seconds_target: float = 15.0):
        o = self.o
        nall = len(self.nodes_all)
        if self.n is None:  # size the sample from a short probe: whole rounds of the threads
            n0 = min(nall, max(self.cores, 8))
            t = time.perf_counter()
            o.collide(self.f, nodes=self.nodes_all[:n0], nthreads=self.cores)
            dt0 = time.perf_counter() - t
            n = int(min(nall, max(n0, seconds_target / max(dt0 / n0, 1e-9))))
            # whole rounds of the threads: a partial last round would leave
            # threads idle and overstate the time per node
            self.n = max(min(nall, self.cores), n // self.cores * self.cores)
        t = time.perf_counter()
        o.collide(self.f, nodes=self.nodes_all[:self.n], nthreads=self.cores)
        dt1 = time.perf_counter() - t
        eval_s = dt1 / self.n * o.N
        return {"value": 1.0 / eval_s, "unit": "evals/s", "cores": self.cores, "kind": "port",
                "sample": f"{self.n} of {o.N} output nodes of one 27^3 VDF (basis functions "
                          f"{list(self.P_SAMPLE)} at the {len(balanced_cells(M))} balanced cells), {dt1:.1f} s; "
                          f"full evaluation = time per node x N"}, dt1


def calibrate_sampling(nthreads: int = 0):
    """Checks the node-sample estimate against a full evaluation where one is
    cheap: the 15^3 grid (s=3, M=5, [-6,6]^3, all 27 basis functions' synthetic
    records), one seeded mixture VDF.  The full oracle evaluation is timed once,
    and the estimate the 27^3 baseline uses (balanced cells, whole rounds of
    the threads, time per node x N) beside it."""
    from oracle.oracle import Oracle
    cores = nthreads or os.cpu_count()
    o = Oracle(3, 5, 6.0)
    f = mixture_batch(o.u, o.v, o.w, o.gwts, 1, 7)[0]
    o.set_A(*o.synth_A(seed=SEED_A, support=1))
    t = time.perf_counter()
    o.collide(f, nthreads=cores)
    full = time.perf_counter() - t
    # the estimator of the 27^3 baseline: balanced cells, whole rounds of the
    # threads, time per node x N (nine basis functions here: 225 nodes, about
    # as many rounds as the 27^3 sample)
    cand = np.array([c * o.P + p for c in balanced_cells(5) for p in range(0, o.P, 3)])
    nodes = cand[:max(cores, len(cand) // cores * cores)]
    t = time.perf_counter()
    o.collide(f, nodes=nodes, nthreads=cores)
    est = (time.perf_counter() - t) / len(nodes) * o.N
    return {"grid": "15^3 (s=3, M=5, [-6,6]^3), one VDF", "full_s": full, "estimated_s": est,
            "estimate_over_full": est / full, "sample_nodes": int(len(nodes)), "cores": cores}


def cpu_baseline(seconds_target: float = 15.0, nthreads: int = 0):
    res, dt = CpuBaseline(nthreads).sample(seconds_target)
    res["calibration"] = calibrate_sampling(nthreads)
    return res, dt


def run_reference(args, world, rank):
    if rank != 0:
        return
    cb = CpuBaseline()
    res = None
    times = []
    for k in range(args.warmup + args.steps):
        r, _ = cb.sample(seconds_target=args.ref_seconds)
        if k >= args.warmup:
            times.append(1.0 / r["value"])
            res = r
    val = 1.0 / statistics.mean(times)
    res["value"] = val
    res["calibration"] = calibrate_sampling()
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "evals/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / val,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "grid": "s=3,M=9,L=7", "batch": BATCH,
                                              "A": "seeded synthetic records, reference index structure",
                                              "each_step": "the same bounded node sample, scaled to one evaluation"},
            "cpu_baseline": res,
            "e2e": {"value": val, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def load_profile_traffic(form: int, set_mb: int = 0, persistent: int = 0):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/k_collide_tc2_27cubed_b256.json for the block form, per
    MB of block records per set, "<MB>p" for one persistent launch per
    evaluation; k_collide_tc_27cubed_b256.json for the chunk form), or None."""
    name = "k_collide_tc2_27cubed_b256.json" if form == 2 else "k_collide_tc_27cubed_b256.json"
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", name)))
        if "dram_bytes_per_launch_by_set_mb" in d:
            v = d["dram_bytes_per_launch_by_set_mb"].get(str(set_mb) + ("p" if persistent else ""))
            return (float(v) if v is not None else None), d.get("note", "")
        return float(d["dram_bytes_per_launch"]), d.get("note", "")
    except Exception:
        return None, ""


def run_ours(args, world, rank, local):
    import torch

    import dgv0d3v_direct_collision_b200 as dgv
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    solver = dgv.DGVSolver(S, M, L, device=local)
    solver.set_stream(stream.cuda_stream)
    if args.tc_form:
        solver.set_tc_form(args.tc_form)
    if args.tc_tiles:
        solver.set_tc_tiles_per_cta(args.tc_tiles)
    if args.tc_set_mb:
        solver.set_tc_set_mb(args.tc_set_mb)
    if args.tc_persistent >= 0:
        solver.set_tc_persistent(bool(args.tc_persistent))
    t = time.perf_counter()
    solver.generate_synthetic_A(seed=SEED_A, support=1)
    t_gen = time.perf_counter() - t
    info = solver.A_info()
    N = solver.N
    fb = mixture_batch(solver.nodes_u, solver.nodes_v, solver.nodes_w, solver.nodes_gwts, BATCH, 1000 + rank)
    f_dev = torch.tensor(fb, dtype=torch.float64, device=f"cuda:{local}")
    qtc = torch.empty_like(f_dev)
    solver.set_projection(True)

    def step():
        solver.EvalCollisionPeriodicAPlus_DGV(f_dev, qtc, precision="tc")

    t = time.perf_counter()
    with torch.cuda.stream(stream):
        step()  # first call builds the tensor-core layout and work lists
        torch.cuda.synchronize()
    t_prep = time.perf_counter() - t
    plan = solver.tc_plan(BATCH)  # the records and lists exist now
    from dgv0d3v_direct_collision_b200._lib import DGV_OPT_TCPERSIST, DGV_OPT_TCSETMB, DGV_OPT_TCTILES
    tc_launch = {"tiles_per_cta": solver.get_option(DGV_OPT_TCTILES),
                 "set_mb": solver.get_option(DGV_OPT_TCSETMB),
                 "persistent": solver.get_option(DGV_OPT_TCPERSIST),
                 "chosen_by": ("the library's autotuner" if not (args.tc_tiles or args.tc_set_mb or args.tc_persistent >= 0)
                               else "options")}
    solver.set_kernel_timing(True)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup - 1):
            step()
        torch.cuda.synchronize()
        solver.kernel_stats(reset=True)
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            e0.record(stream)
            for _ in range(args.steps):
                step()
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        barrier(world)
        torch.cuda.synchronize()
    kst = solver.kernel_stats(reset=True)
    solver.set_kernel_timing(False)
    ms_max = max_over_ranks(ms, world)
    value = world * BATCH * args.steps / (ms_max / 1000.0)

    # plain FP64 path on the first NB64 VDFs of the batch (its throughput per
    # VDF does not depend on the batch size) and the error of the
    # tensor-core path against it; both with the FP64 conservation projection
    NB64 = min(BATCH, args.f64_vdfs)
    f64_in = f_dev[:NB64].contiguous()
    q64 = torch.empty_like(f64_in)
    with torch.cuda.stream(stream):
        solver.EvalCollisionPeriodicAPlus_DGV(f64_in, q64, precision="f64")  # warm-up (chunk choice, buffers)
        torch.cuda.synchronize()
        e0.record(stream)
        solver.EvalCollisionPeriodicAPlus_DGV(f64_in, q64, precision="f64")
        e1.record(stream)
        torch.cuda.synchronize()
    ms64 = max_over_ranks(e0.elapsed_time(e1), world)
    value64 = world * NB64 / (ms64 / 1000.0)
    qtch, q64h = qtc[:NB64].cpu().numpy(), q64.cpu().numpy()
    errs = np.linalg.norm(qtch - q64h, axis=1) / np.linalg.norm(q64h, axis=1)
    merrs = np.abs(qtch - q64h).max(axis=1) / np.abs(q64h).max(axis=1)
    psi = [np.ones(N), solver.nodes_u, solver.nodes_v, solver.nodes_w,
           solver.nodes_u ** 2 + solver.nodes_v ** 2 + solver.nodes_w ** 2]
    qall = qtc.cpu().numpy()
    cons = max(abs(np.sum(solver.nodes_gwts * p_ * q)) / np.sum(np.abs(solver.nodes_gwts * p_ * q))
               for q in qall for p_ in psi)

    # end to end through the C-ABI with host buffers (pinned): H2D + compute + D2H per step
    f_host = torch.tensor(fb, dtype=torch.float64).pin_memory()
    q_host = torch.empty_like(f_host).pin_memory()
    fh, qh = f_host.numpy(), q_host.numpy()
    solver.EvalCollisionPeriodicAPlus_DGV(fh, qh, precision="tc")
    barrier(world)
    with torch.cuda.stream(stream):
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            solver.EvalCollisionPeriodicAPlus_DGV(fh, qh, precision="tc")
        e1.record(stream)
        torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1), world)
    e2e = world * BATCH * args.steps / (ms_e2e / 1000.0)

    # adjoint (vector-Jacobian product) of the same batch on the tensor cores,
    # cotangents v ~ N(0,1) per node; its time per batch against the forward's
    # (one batched evaluation with the projection, timed above); error against
    # the FP64 device VJP on two VDFs
    adjoint = None
    if args.adjoint_steps > 0:
        v_dev = torch.tensor(np.random.default_rng(2000 + rank).standard_normal(fb.shape), device=f_dev.device)
        g_dev = torch.empty_like(f_dev)
        with torch.cuda.stream(stream):
            t = time.perf_counter()
            solver.vjp(f_dev, v_dev, g_dev, precision="tc")  # builds the adjoint's block records and lists
            torch.cuda.synchronize()
            t_adj = time.perf_counter() - t
            solver.vjp(f_dev, v_dev, g_dev, precision="tc")
            torch.cuda.synchronize()
            barrier(world)
            e0.record(stream)
            for _ in range(args.adjoint_steps):
                solver.vjp(f_dev, v_dev, g_dev, precision="tc")
            e1.record(stream)
            torch.cuda.synchronize()
        ms_adj = max_over_ranks(e0.elapsed_time(e1), world) / args.adjoint_steps
        g64 = solver.vjp(f_dev[:2].contiguous(), v_dev[:2].contiguous(), precision="f64").cpu().numpy()
        gtc = g_dev[:2].cpu().numpy()
        aerr = float(max(np.linalg.norm(gtc[k] - g64[k]) / np.linalg.norm(g64[k]) for k in range(2)))
        adjoint = {"ms_per_batch": ms_adj, "evals_per_s": world * BATCH / (ms_adj / 1000.0),
                   "adjoint_over_forward": ms_adj / (ms_max / args.steps), "steps": args.adjoint_steps,
                   "err_tc_vs_f64_vjp_norm_max": aerr, "setup_s": t_adj,
                   "form": "block form: G = f(c2) W1 and f(c1) W2 per cell-pair block on the tensor cores, "
                           "contracted with c = 2v/w; target-cell ownership"}

    if rank != 0:
        return
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        tc_peak, peak_src = float(peaks["bf16_tflops_sustained"]), "measured (bf16 sustained)"
    except Exception:
        tc_peak, peak_src = 1400.0, "fallback (bf16 sustained)"
    # algorithmic work: one record-shift = A * f(a) * f(b) accumulated = 3 FLOPs
    alg_flop_eval = 3.0 * info["record_shifts"]
    k_ms_launch = kst["ms"] / max(kst["launches"], 1)
    alg_flop_launch = alg_flop_eval * BATCH * args.steps / max(kst["launches"], 1)
    achieved = alg_flop_launch / (k_ms_launch / 1000.0) / 1e12
    # FLOPs the MMAs issue per launch (dense tiles, three split products) over the same time
    issued = plan["tensor_flop"] / max(plan["launches"], 1) / (k_ms_launch / 1000.0) / 1e12
    form = solver.tc_form
    traffic, tnote = load_profile_traffic(form, tc_launch["set_mb"], tc_launch["persistent"])
    kname = "k_collide_tc2<128,27>" if form == 2 else "k_collide_tc<128>"
    knote = ("algorithmic FLOPs = 3 per record-shift (A*f*f + add) x VDFs; the block form computes "
             "G = f(c2) W per cell-pair block on the tensor core (dense W: 27 x 729 per block, 3 fp16 "
             "products hi*hi, hi*lo, lo*hi, M=128 x N=256 tiles) and contracts G with f(c1) on the CUDA cores. "
             if form == 2 else
             "algorithmic FLOPs = 3 per record-shift (A*f*f + add) x VDFs; the kernel issues "
             "3 fp16 products per term (hi*hi, hi*lo, lo*hi) on M=128 x N<=64 tiles. ")
    line = {
        "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f16 hi+lo split products, f32 accumulate, f64 sums",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": "s=3,M=9,L=7", "batch_per_gpu": BATCH, "global_batch": BATCH * world,
                   "precision": "tensor cores (tcgen05): split-fp16 operands, compensated FP32/FP64 accumulation, "
                                "FP64 conservation projection",
                   "tc_form": "block (dense cell-pair W, DGV_OPT_TCFORM=2)" if form == 2 else "chunk (pairs, DGV_OPT_TCFORM=1)",
                   "A": f"seeded synthetic records, reference index structure: {info['records']} records, "
                        f"{info['pairs']} pairs, {info['blocks']} cell-pair blocks",
                   "record_shifts_per_eval": info["record_shifts"],
                   "l2": "inputs larger than L2: the A records (~14.6 GB block form / ~8 GB chunk form) "
                         "are streamed from HBM every step",
                   "parallelism": f"replicas over VDFs, dp{world}",
                   "tc_launch": tc_launch},
        "f64_plain_evals_per_s": value64, "f64_timed_vdfs": NB64, "tc_over_f64": value / value64,
        "err_tc_vs_f64_norm_max": float(errs.max()), "err_tc_vs_f64_maxabs_rel_max": float(merrs.max()),
        "conservation_rel_max": float(cons),
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": tc_peak, "unit": "TFLOP/s",
                     "frac": achieved / tc_peak, "traffic": traffic, "peak_source": peak_src,
                     "kernel": kname, "launches_per_step": kst["launches"] / args.steps,
                     "issued_tensor_tflops": issued, "issued_frac": issued / tc_peak,
                     "issued_over_algorithmic": plan["tensor_flop"] / (alg_flop_eval * BATCH),
                     "kernel_ms_per_launch": k_ms_launch,
                     "alg_flop_per_launch": alg_flop_launch,
                     "note": knote + "traffic = ncu dram read+write bytes per launch. " + tnote},
        "cpu_baseline": None,
        "e2e": {"value": e2e, "unit": "evals/s", "h2d_bytes_per_step": int(BATCH * N * 8),
                "d2h_bytes_per_step": int(BATCH * N * 8)},
        "adjoint": adjoint,
        "gpu_launches": int(kst["all_launches"]),
        "clocks": clk.summary(),
        "setup_s": {"synthetic_A": t_gen, "tensor_core_layout_and_lists": t_prep},
    }
    if world == 1 and not args.no_cpu_baseline:
        cb, _ = cpu_baseline(seconds_target=args.ref_seconds)
        line["cpu_baseline"] = cb
    print(json.dumps(line))


def run_mixed(args):
    """Mixed-grid batch: 768 VDFs on the 21^3 grid (s=3, M=7, [-6,6]^3) and
    256 on the 15^3 grid (s=3, M=5, [-6,6]^3), seeded Maxwellian mixtures times
    (1 + 0.1 N(0,1)) per node clipped at 0, tensor-core path, evaluated per
    step by one dgv_collide_group call (one CUDA graph over both contexts'
    streams).  Timed beside it: the same work as two separate batched calls.
    Prints its own JSON line (not the headline)."""
    import torch

    import dgv0d3v_direct_collision_b200 as dgv
    parts = [(3, 7, 6.0, 768), (3, 5, 6.0, 256)]
    members = []
    for i, (s_, m_, l_, nb) in enumerate(parts):
        sol = dgv.DGVSolver(s_, m_, l_)
        sol.generate_synthetic_A(seed=SEED_A + i, support=1)
        fb = mixture_batch(sol.nodes_u, sol.nodes_v, sol.nodes_w, sol.nodes_gwts, nb, 77 + i)
        # multiplicative perturbation per node, clipped at 0
        fb *= np.clip(1.0 + 0.1 * np.random.default_rng(99 + i).standard_normal(fb.shape), 0.0, None)
        f = torch.tensor(fb, dtype=torch.float64, device="cuda")
        members.append((sol, f, torch.empty_like(f)))
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        for sol, _, _ in members:  # launches of the timed steps only
            sol.kernel_stats(reset=True)
        with ClockSampler(0) as clk:
            e0.record(stream)
            for _ in range(args.steps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps, clk.summary()

    def group():
        dgv.collide_group(members, precision="tc", stream_ptr=stream.cuda_stream)

    def separate():
        for sol, f, q in members:
            sol.set_stream(stream.cuda_stream)
            sol.EvalCollisionPeriodicAPlus_DGV(f, q, precision="tc")

    for sol, _, _ in members:
        sol.set_kernel_timing(True)
    ms_g, clk = timed(group)
    launches = sum(m[0].kernel_stats(reset=True)["all_launches"] for m in members) / args.steps
    q_group = [m[2].clone() for m in members]
    ms_s, _ = timed(separate)
    same = all(torch.equal(a, m[2]) for a, m in zip(q_group, members))
    nvdf = sum(p[3] for p in parts)
    print(json.dumps({
        "metric": "mixed-grid batch Q(f,f) evals/s (768 x 21^3 + 256 x 15^3, one graph launch per step)",
        "value": nvdf / (ms_g / 1000.0), "unit": "evals/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_g, "higher_is_better": True, "dtype": "f16 hi+lo split products, f32 accumulate, f64 sums",
        "data": "synthetic",
        "config": {"workload": "768 VDFs on s=3,M=7,[-6,6]^3 + 256 VDFs on s=3,M=5,[-6,6]^3, tensor-core path",
                   "A": [m[0].A_info() for m in members],
                   "l2": "inputs larger than L2: the block records of both grids (~4 GB) are streamed every step"},
        "separate_calls_ms_per_step": ms_s, "group_over_separate": ms_s / ms_g,
        "group_equals_separate": bool(same), "gpu_launches": int(round(launches)),
        "gpu_launches_note": "kernel launches per step inside the one graph launch (preparation and final "
                             "kernels per grid, one persistent collision kernel for both grids)",
        "clocks": clk}))


def run_trajectory(args):
    """RK4 relaxation on the 21^3 grid (s=3, M=7, [-6,6]^3): a seeded
    Maxwellian mixture (1-4 components, density 1) advanced 500 steps with
    dt = 0.005 by the FP32-compensated and the FP64 paths side by side, with
    the conservation projection.  At every step: the error of the FP32 Q
    against the FP64 Q on the FP64 state, the distance between the two
    trajectories, and the drift of the moments of both.  Prints a JSON
    summary (not the headline)."""
    import torch

    import dgv0d3v_direct_collision_b200 as dgv
    kappa, dt, steps = 0.1, 0.005, args.trajectory_steps
    s = dgv.DGVSolver(3, 7, 6.0, kappa=kappa)
    s.generate_synthetic_A(seed=SEED_A, support=1)
    s.set_projection(True)
    f0 = mixture_batch(s.nodes_u, s.nodes_v, s.nodes_w, s.nodes_gwts, 1, 5)[0]
    f64 = torch.tensor(f0, device="cuda")
    f32 = f64.clone()
    r64, r32 = torch.zeros_like(f64), torch.zeros_like(f64)
    q64, q32 = torch.zeros_like(f64), torch.zeros_like(f64)
    m0 = np.array(s.MassCheckRec(f0))

    def rel(x, y):
        return float(torch.linalg.norm(x - y) / torch.linalg.norm(y))

    qerr, traj, drift = [], [], []
    t0 = time.perf_counter()
    for _ in range(steps):
        s.EvalCollisionPeriodicAPlus_DGV(f64, q64, precision="f64")
        s.EvalCollisionPeriodicAPlus_DGV(f64, q32, precision="f32c")
        qerr.append(rel(q32, q64))
        s.TimeIntegratorORK_SH_DGV(f64, dt, frhs1=r64, order=4, precision="f64")
        s.TimeIntegratorORK_SH_DGV(f32, dt, frhs1=r32, order=4, precision="f32c")
        traj.append(rel(f32, f64))
        m64, m32 = np.array(s.MassCheckRec(f64)), np.array(s.MassCheckRec(f32))
        drift.append(float(max(np.max(np.abs(m64 - m0) / np.maximum(1.0, np.abs(m0))),
                               np.max(np.abs(m32 - m0) / np.maximum(1.0, np.abs(m0))))))
    wall = time.perf_counter() - t0
    print(json.dumps({
        "case": "RK4 relaxation, 21^3 (s=3, M=7, [-6,6]^3), FP32-compensated vs FP64, projection on",
        "steps": steps, "dt": dt, "kappa": kappa, "A": s.A_info(),
        "q_err_f32c_vs_f64": {"max": max(qerr), "median": float(np.median(qerr)), "last": qerr[-1]},
        "trajectory_distance": {"max": max(traj), "last": traj[-1]},
        "moment_drift_max": max(drift),
        "state_change": float(torch.linalg.norm(f64 - torch.tensor(f0, device="cuda")) / np.linalg.norm(f0)),
        "wall_s": wall}))


def run_profile_case(case: str, args=None):
    """Cases for profiler captures.  "<prec>_21": the 21^3 grid (s=3, M=7,
    [-6,6]^3; A rows ~5.6 GB in total) -- one VDF with a fixed chunk count (no
    tuning launches) for the CUDA-core kernels, a batch of 256 VDFs for the
    tensor-core kernels (one launch per block set; "tc" the chunk form, "tc2"
    the block form).  "<prec>_15": the 15^3 grid (s=3, M=5, [-6,6]^3; rows
    ~0.6 GB), 256 VDFs ("vjptc": the tensor-core adjoint with v = f; "f64":
    one VDF).  "<prec>_27": the benchmark workload itself (27^3 x
    256 VDFs), for single-pass counters only.  Two evaluations each: a
    warm-up, then the one to capture."""
    import torch

    import dgv0d3v_direct_collision_b200 as dgv
    prec, grid = case.split("_")
    s = {"27": lambda: dgv.DGVSolver(S, M, L), "21": lambda: dgv.DGVSolver(3, 7, 6.0),
         "15": lambda: dgv.DGVSolver(3, 5, 6.0)}[grid]()
    s.generate_synthetic_A(seed=SEED_A, support=1)
    if prec == "tc2":
        s.set_tc_form(2)
        prec = "tc"
    if args is not None and args.tc_set_mb:
        s.set_tc_set_mb(args.tc_set_mb)
    if args is not None and args.tc_tiles:
        s.set_tc_tiles_per_cta(args.tc_tiles)
    if args is not None and args.tc_persistent >= 0:
        s.set_tc_persistent(bool(args.tc_persistent))
    if prec not in ("tc", "vjptc"):
        s.set_nchunks(296)
    nb = BATCH if prec in ("tc", "vjptc") else 1
    fb = mixture_batch(s.nodes_u, s.nodes_v, s.nodes_w, s.nodes_gwts, nb, 3)
    f = torch.tensor(fb if nb > 1 else fb[0], dtype=torch.float64, device="cuda")
    q = torch.empty_like(f)
    times = []
    for _ in range(2):
        t = time.perf_counter()
        if prec == "vjp":
            s.vjp(f, f, q)
        elif prec == "vjptc":
            s.vjp(f, f, q, precision="tc")
        else:
            s.EvalCollisionPeriodicAPlus_DGV(f, q, precision=prec)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t)
    print(json.dumps({"profile_case": case, "wall_s": times, "A": s.A_info()}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--profile-case", choices=["f64_21", "f32c_21", "vjp_21", "tc_21", "tc_27", "tc2_21", "tc2_27",
                                               "tc_15", "tc2_15", "vjptc_15", "vjptc_27", "f64_15"],
                    default=None,
                    help="small single-VDF case for profiler captures (no JSON bench line)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--f64-vdfs", type=int, default=32,
                    help="VDFs of the batch the plain FP64 arm is timed on")
    ap.add_argument("--mixed", action="store_true",
                    help="time the mixed-grid batch (768 x 21^3 + 256 x 15^3) instead of the headline")
    ap.add_argument("--trajectory", action="store_true",
                    help="RK4 relaxation at 21^3, FP32-compensated vs FP64 per step (report, not the headline)")
    ap.add_argument("--trajectory-steps", type=int, default=500)
    ap.add_argument("--tc-form", type=int, default=0, choices=[0, 1, 2],
                    help="tensor-core form of the headline arm (0 = the library default)")
    ap.add_argument("--tc-tiles", type=int, default=0, choices=[0, 1, 2],
                    help="block form: VDF tiles per CTA (0 = the library default)")
    ap.add_argument("--adjoint-steps", type=int, default=3,
                    help="timed tensor-core VJP evaluations of the batch (0 = skip the adjoint)")
    ap.add_argument("--tc-set-mb", type=int, default=0,
                    help="block form: MB of block records per launch (0 = the library default)")
    ap.add_argument("--tc-persistent", type=int, default=-1, choices=[-1, 0, 1],
                    help="block form: 1 = one persistent launch per evaluation, 0 = one launch per set "
                         "(-1 = the library's choice)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.profile_case:
        run_profile_case(args.profile_case, args)
        return
    if args.mixed:
        run_mixed(args)
        return
    if args.trajectory:
        run_trajectory(args)
        return
    if args.impl == "reference":
        # the CPU reference runs on rank 0 only; other ranks exit without work
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, world, rank)
        return
    world, rank, local = dist_setup()
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

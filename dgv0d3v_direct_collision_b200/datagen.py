"""Training-data writer: (f, Q(f)) pairs for data-driven collision models.

The reference states this as the code's purpose going forward (README.md:28-30:
compute the collision operator for a bunch of VDFs and save the VDFs and the
outputs on disk).  `TrainingDataWriter` does it in shards:

- each shard holds `vdfs_per_shard` VDFs drawn by a seeded sampler, the
  stream of shard i being `numpy.random.default_rng([seed, i])`, so any shard
  can be regenerated alone and a run can be resumed or split over processes;
- Q of a shard is one batched call of the library (`dgv_collide_batched`);
  the host work around it (drawing the next shard, writing the previous one)
  runs in two threads, so the GPU call overlaps it;
- shards are `shard_%06d.npz` files (arrays `f`, `q` of shape [B, N] in node
  order, `params`, the sampler's parameters per VDF), each written to a
  temporary name and renamed; `manifest.json` records the grid, the operator,
  the sampler and the shards finished, and a writer started on the same
  directory with the same settings skips those shards.

Samplers (seeded synthetic inputs of the shapes the collision benchmarks
use): "mixture" -- K ~ U{1..kmax} Maxwellians, weights ~ Dirichlet(1), bulk
velocities ~ U[-2,2]^3, temperatures ~ U[0.5,2], normalised to density 1;
"bimodal" -- two Maxwellians of equal weight at +-U[1,2] along a random unit
direction, temperatures ~ U[0.5,1.5], normalised to density 1.  The
Maxwellian is maxwelveldist's (distributions_mod.f90:83-95):
n exp(-|v-u0|^2/T) / (pi T)^{3/2}.
"""
from __future__ import annotations

import json
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

SAMPLERS = ("mixture", "bimodal")
PARAMS_PER_COMPONENT = 5  # weight, u0, v0, w0, T


def _maxwellian(u, v, w, n, u0, T):
    r2 = (u - u0[0]) ** 2 + (v - u0[1]) ** 2 + (w - u0[2]) ** 2
    return n * np.exp(-r2 / T) / (np.pi * T) ** 1.5


def sample_vdfs(nodes_u, nodes_v, nodes_w, gwts, rng, count: int, kind: str = "mixture", kmax: int = 4):
    """count VDFs [count, N] and their parameters [count, kmax, 5] (weight,
    bulk velocity, temperature per component; unused components zero)."""
    if kind not in SAMPLERS:
        raise ValueError(f"kind must be one of {SAMPLERS}")
    ncomp = kmax if kind == "mixture" else 2
    f = np.zeros((count, len(nodes_u)))
    params = np.zeros((count, ncomp, PARAMS_PER_COMPONENT))
    for b in range(count):
        if kind == "mixture":
            k = int(rng.integers(1, kmax + 1))
            wts = rng.dirichlet(np.ones(k))
            comps = [(wts[j], rng.uniform(-2, 2, 3), rng.uniform(0.5, 2.0)) for j in range(k)]
        else:
            d = rng.standard_normal(3)
            d /= np.linalg.norm(d)
            s = rng.uniform(1.0, 2.0)
            comps = [(0.5, s * d, rng.uniform(0.5, 1.5)), (0.5, -s * d, rng.uniform(0.5, 1.5))]
        for j, (wt, u0, T) in enumerate(comps):
            f[b] += _maxwellian(nodes_u, nodes_v, nodes_w, wt, u0, T)
            params[b, j] = (wt, u0[0], u0[1], u0[2], T)
        dens = float(np.sum(f[b] * gwts))
        f[b] /= dens
        params[b, :len(comps), 0] /= dens
    return f, params


def _grid_of(solver) -> dict:
    d = solver.desc
    return {name: getattr(d, name) for name, _ in d._fields_}


class TrainingDataWriter:
    """Writes shards of (f, Q(f)) pairs computed by `solver` into `out_dir`."""

    def __init__(self, solver, out_dir: str, vdfs_per_shard: int = 256, *, kind: str = "mixture",
                 kmax: int = 4, seed: int = 0, precision: str | None = None, dtype: str = "f8",
                 operator: str = ""):
        if kind not in SAMPLERS:
            raise ValueError(f"kind must be one of {SAMPLERS}")
        if dtype not in ("f8", "f4"):
            raise ValueError("dtype must be 'f8' or 'f4'")
        if vdfs_per_shard < 1:
            raise ValueError("vdfs_per_shard must be positive")
        self.solver = solver
        self.out_dir = out_dir
        self.config = {
            "format": "dgv-training-shards/1",
            "grid": _grid_of(solver),
            "N": int(solver.N),
            "operator": {"tag": operator, **{k: int(v) for k, v in solver.A_info().items() if k != "record_shifts"}},
            "precision": precision or solver.precision,
            "projection": bool(getattr(solver, "projection", False)),
            "sampler": {"kind": kind, "kmax": kmax, "seed": seed},
            "vdfs_per_shard": vdfs_per_shard,
            "dtype": dtype,
            "layout": "f, q: [vdfs_per_shard, N] in node order; params: [vdfs_per_shard, components, 5]",
        }
        os.makedirs(out_dir, exist_ok=True)
        self.done = set()
        man = self.manifest_path
        if os.path.exists(man):
            with open(man) as fh:
                old = json.load(fh)
            if old.get("config") != json.loads(json.dumps(self.config)):
                raise ValueError(f"{man} was written with other settings; use another directory")
            self.done = {int(i) for i in old.get("shards", [])}

    @property
    def manifest_path(self) -> str:
        return os.path.join(self.out_dir, "manifest.json")

    def shard_path(self, i: int) -> str:
        return os.path.join(self.out_dir, "shard_%06d.npz" % i)

    def sample(self, i: int):
        """VDFs and parameters of shard i (regenerable from the seed alone)."""
        s = self.solver
        sp = self.config["sampler"]
        rng = np.random.default_rng([sp["seed"], i])
        return sample_vdfs(s.nodes_u, s.nodes_v, s.nodes_w, s.nodes_gwts, rng, self.config["vdfs_per_shard"],
                           sp["kind"], sp["kmax"])

    def _save(self, i: int, f, q, params):
        dt = np.float64 if self.config["dtype"] == "f8" else np.float32
        tmp = self.shard_path(i) + ".tmp.npz"
        np.savez(tmp, f=f.astype(dt, copy=False), q=q.astype(dt, copy=False), params=params)
        os.replace(tmp, self.shard_path(i))
        return i

    def _write_manifest(self):
        tmp = self.manifest_path + ".tmp"
        with open(tmp, "w") as fh:
            json.dump({"config": self.config, "shards": sorted(self.done)}, fh, indent=1)
        os.replace(tmp, self.manifest_path)

    def write(self, n_shards: int, start: int = 0) -> list:
        """Compute and write shards start .. start+n_shards-1, skipping those
        already finished; returns the indices written by this call."""
        todo = [i for i in range(start, start + n_shards) if i not in self.done]
        written = []
        if not todo:
            return written
        prec = self.config["precision"]
        def finish(fut):
            i = fut.result()
            self.done.add(i)
            written.append(i)
            self._write_manifest()

        with ThreadPoolExecutor(max_workers=2) as pool:
            gen = pool.submit(self.sample, todo[0])
            pending = None
            for k, i in enumerate(todo):
                f, params = gen.result()
                if k + 1 < len(todo):
                    gen = pool.submit(self.sample, todo[k + 1])
                q = self.solver.collide(f, precision=prec)  # GPU; the GIL is released in the call
                if pending is not None:
                    finish(pending)
                pending = pool.submit(self._save, i, f, q, params)
            finish(pending)
        return written


def read_shard(path: str) -> dict:
    """Arrays of one shard file."""
    with np.load(path) as z:
        return {k: z[k] for k in z.files}

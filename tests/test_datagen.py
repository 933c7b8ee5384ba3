"""Training-data writer (the reference's stated purpose, README.md:28-30) on
the CPU with a stand-in solver whose Q is a known map: shard contents and
layout, seeded regeneration of any shard, the samplers' distributions and
normalisation, resume after an interrupted run, and refusal to mix settings
in one directory."""
import json
import os

import numpy as np
import pytest

from dgv0d3v_direct_collision_b200._lib import GridDesc
from dgv0d3v_direct_collision_b200.datagen import TrainingDataWriter, read_shard, sample_vdfs


class FakeSolver:
    """Grid of the real layout (s=2, M=3, [-3,3]^3 nodes by tensor product);
    Q(f) = 2 f + 1 so that the written q can be checked exactly."""

    def __init__(self):
        x, w = np.polynomial.legendre.leggauss(2)
        edges = np.linspace(-3, 3, 4)
        pts, wts = [], []
        for c in range(3):
            a, b = edges[c], edges[c + 1]
            pts += list((a + b) / 2 + (b - a) / 2 * x)
            wts += list((b - a) / 2 * w)
        pts, wts = np.array(pts), np.array(wts)
        U, V, W = np.meshgrid(pts, pts, pts, indexing="ij")
        WU, WV, WW = np.meshgrid(wts, wts, wts, indexing="ij")
        self.nodes_u, self.nodes_v, self.nodes_w = U.ravel(), V.ravel(), W.ravel()
        self.nodes_gwts = (WU * WV * WW).ravel()
        self.N = self.nodes_u.size
        self.desc = GridDesc(2, 2, 2, 3, 3, 3, -3, 3, -3, 3, -3, 3, 1.0)
        self.precision = "f64"
        self.calls = 0

    def A_info(self):
        return {"records": 10, "pairs": 5, "blocks": 2, "record_shifts": 1.5}

    def collide(self, f, precision=None):
        self.calls += 1
        return 2.0 * f + 1.0


@pytest.mark.parametrize("kind", ["mixture", "bimodal"])
def test_samplers(kind):
    s = FakeSolver()
    rng = np.random.default_rng(5)
    f, params = sample_vdfs(s.nodes_u, s.nodes_v, s.nodes_w, s.nodes_gwts, rng, 40, kind)
    assert f.shape == (40, s.N) and np.all(f >= 0)
    np.testing.assert_allclose(f @ s.nodes_gwts, 1.0, rtol=1e-13)
    T = params[..., 4]
    used = params[..., 0] > 0
    if kind == "mixture":
        assert np.all((T[used] >= 0.5) & (T[used] <= 2.0))
        assert np.all(np.abs(params[..., 1:4][used]) <= 2.0)
        assert set(used.sum(axis=1)) <= {1, 2, 3, 4}
    else:
        assert np.all(used) and np.all((T >= 0.5) & (T <= 1.5))
        u = params[..., 1:4]
        np.testing.assert_allclose(u[:, 0], -u[:, 1], atol=1e-15)
        sp = np.linalg.norm(u[:, 0], axis=1)
        assert np.all((sp >= 1.0) & (sp <= 2.0))
    # the parameters rebuild the VDF (maxwelveldist, weights already normalised)
    b = 3
    g = np.zeros(s.N)
    for wt, u0, v0, w0, t in params[b]:
        if wt > 0:
            r2 = (s.nodes_u - u0) ** 2 + (s.nodes_v - v0) ** 2 + (s.nodes_w - w0) ** 2
            g += wt * np.exp(-r2 / t) / (np.pi * t) ** 1.5
    np.testing.assert_allclose(g, f[b], rtol=1e-12)


def test_shards_resume_and_regeneration(tmp_path):
    s = FakeSolver()
    out = str(tmp_path / "data")
    w = TrainingDataWriter(s, out, vdfs_per_shard=6, seed=7)
    assert w.write(3) == [0, 1, 2]
    assert s.calls == 3
    man = json.load(open(os.path.join(out, "manifest.json")))
    assert man["shards"] == [0, 1, 2] and man["config"]["N"] == s.N
    for i in range(3):
        d = read_shard(w.shard_path(i))
        assert d["f"].shape == (6, s.N) and d["f"].dtype == np.float64
        np.testing.assert_array_equal(d["q"], 2.0 * d["f"] + 1.0)
        f2, p2 = w.sample(i)  # regenerable from (seed, shard) alone
        np.testing.assert_array_equal(d["f"], f2)
        np.testing.assert_array_equal(d["params"], p2)
    assert not np.array_equal(read_shard(w.shard_path(0))["f"], read_shard(w.shard_path(1))["f"])

    # an interrupted run: shard 3 never finished; a new writer redoes only 3 and 4
    w2 = TrainingDataWriter(s, out, vdfs_per_shard=6, seed=7)
    assert w2.write(5) == [3, 4]
    assert s.calls == 5
    assert json.load(open(os.path.join(out, "manifest.json")))["shards"] == [0, 1, 2, 3, 4]
    assert not [p for p in os.listdir(out) if ".tmp" in p]

    # other settings in the same directory are refused
    with pytest.raises(ValueError):
        TrainingDataWriter(s, out, vdfs_per_shard=6, seed=8)
    with pytest.raises(ValueError):
        TrainingDataWriter(s, out, vdfs_per_shard=6, seed=7, kind="bimodal")


def test_float32_storage_and_split_ranges(tmp_path):
    s = FakeSolver()
    a = TrainingDataWriter(s, str(tmp_path / "a"), vdfs_per_shard=4, seed=1, dtype="f4")
    b = TrainingDataWriter(s, str(tmp_path / "b"), vdfs_per_shard=4, seed=1, dtype="f4")
    a.write(2, start=0)
    b.write(2, start=2)  # a second process can take another range of the same stream
    full = TrainingDataWriter(s, str(tmp_path / "c"), vdfs_per_shard=4, seed=1, dtype="f4")
    full.write(4)
    for i, w in [(0, a), (1, a), (2, b), (3, b)]:
        d, e = read_shard(w.shard_path(i)), read_shard(full.shard_path(i))
        assert d["f"].dtype == np.float32
        np.testing.assert_array_equal(d["f"], e["f"])
        np.testing.assert_array_equal(d["q"], e["q"])

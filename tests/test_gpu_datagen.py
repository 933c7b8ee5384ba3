"""Training-data writer on the device: the shards written with the FP64 path
and with the tensor-core path hold Q(f) of the oracle for the written f
(tolerances 1e-12 and 1e-6 norm-wise per VDF).  15^3 grid (s=3, M=5,
[-6,6]^3) with seeded synthetic A-arrays on both sides."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sides():
    import dgv0d3v_direct_collision_b200 as dgv
    from oracle.oracle import Oracle
    o = Oracle(3, 5, 6.0)
    cap, A, xi, xi1 = o.synth_A(seed=11, support=1)
    o.set_A(cap, A, xi, xi1)
    s = dgv.DGVSolver(3, 5, 6.0)
    s.generate_synthetic_A(seed=11, support=1)
    return o, s


@pytest.mark.parametrize("precision,tol,kind", [("f64", 1e-12, "mixture"), ("tc", 1e-6, "bimodal")])
def test_shards_hold_oracle_q(sides, tmp_path, precision, tol, kind):
    from dgv0d3v_direct_collision_b200.datagen import TrainingDataWriter, read_shard
    o, s = sides
    w = TrainingDataWriter(s, str(tmp_path / precision), vdfs_per_shard=3, kind=kind, seed=4,
                           precision=precision, operator="synthetic seed 11")
    assert w.write(2) == [0, 1]
    for i in range(2):
        d = read_shard(w.shard_path(i))
        for b in range(3):
            ref = o.collide(d["f"][b])
            assert rel_err(d["q"][b], ref) < tol, (i, b)

"""GPU tests of the sharded driver over the device library: ranks emulated
as separate handles on one GPU (each phase runs on every handle before the
next; no kernel waits on another), compared bit for bit with pt_step, and the
per-bucket work against the pass counters."""
import numpy as np
import pytest

from paratreet_b200 import ics
from paratreet_b200.sharding import DeviceEngine, ShardedGravity, run_emulated

pytestmark = pytest.mark.gpu


def sim(**kw):
    from paratreet_b200.gravity import GravitySimulation
    return GravitySimulation(**kw)


@pytest.mark.parametrize("precision,world", [("fp64", 1), ("fp64", 2), ("fp64", 3), ("mixed", 2)])
def test_emulated_ranks_match_pt_step(precision, world):
    p = ics.mixture(60000, seed=7, soft=1e-3)
    kw = dict(max_particles_per_leaf=16, theta=0.7, max_timestep=1e-3, precision=precision)
    with sim(**kw) as ref:
        ref.set_particles(p)
        ref.run(3)
        want = ref.state()
    handles = [sim(**kw) for _ in range(world)]
    try:
        for h in handles:
            h.set_particles(p)
        shards = [ShardedGravity(DeviceEngine(h), world, r) for r, h in enumerate(handles)]
        run_emulated(shards, 3)
        for h in handles:
            got = h.state()
            for k in want:
                assert np.array_equal(got[k], want[k]), k
        if world > 1:  # later passes were split by measured work
            nb = handles[0].counters()["n_buckets"]
            assert shards[0].cuts[-1] == nb and len(set(shards[0].cuts)) == world + 1
    finally:
        for h in handles:
            h.close()


def test_bucket_work_matches_counters():
    p = ics.plummer(50000, seed=3, soft=0.01)
    with sim(max_particles_per_leaf=32, precision="mixed") as s:
        s.set_particles(p)
        s.start_down()
        w = s.bucket_work()
        c = s.counters()
        assert w.size == c["n_buckets"] and int(w.sum()) == c["n_pp"] + c["n_pc"]
        nb = w.size
        s.start_down(buckets=(nb // 4, nb // 2))
        w2 = s.bucket_work()
        assert np.all(w2[: nb // 4] == 0) and np.all(w2[nb // 2:] == 0)
        assert np.array_equal(w2[nb // 4: nb // 2], w[nb // 4: nb // 2])

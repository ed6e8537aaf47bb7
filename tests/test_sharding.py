"""CPU tests of the multi-rank host logic (paratreet_b200/sharding.py): the
work-balanced bucket cuts, and whole sharded runs over 2 and 3 gloo ranks
(one process each, 127.0.0.1) driving a small numpy engine with the same
interface as the device library -- re-sort by key every pass, buckets of
consecutive particles, zero outside the traversed range, per-bucket work, a
KKD advance -- compared bit for bit with a single-rank run."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch

from paratreet_b200 import ics
from paratreet_b200.sharding import BIG, ShardedGravity, balanced_cuts, rescale_cuts, run_emulated


class NumpyEngine:
    """Direct-sum stand-in for the device engine (Plummer softening)."""

    def __init__(self, p, bucket=16, dt_max=0.01):
        self.f = {k: np.array(p[k], dtype=np.float64) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "soft")}
        self.n = self.f["x"].size
        self.bucket, self.dt_max = bucket, dt_max
        self.nb = 0
        self.acc = [torch.zeros(self.n, dtype=torch.float64) for _ in range(5)]
        self.work = torch.zeros(0, dtype=torch.int64)

    def n_buckets(self):
        return self.nb

    def _sort(self):
        q = [np.floor((self.f[a] - self.f[a].min()) / (np.ptp(self.f[a]) + 1e-300) * 1023).astype(np.int64)
             for a in "xyz"]
        key = np.zeros(self.n, np.int64)
        for bit in range(10):  # interleave 10 bits per dimension, x most significant
            for d in range(3):
                key |= ((q[d] >> bit) & 1) << (3 * bit + 2 - d)
        o = np.argsort(key, kind="stable")
        for k in self.f:
            self.f[k] = self.f[k][o]

    def compute_range(self, b0, b1):
        self._sort()
        self.nb = (self.n + self.bucket - 1) // self.bucket
        for t in self.acc:
            t.zero_()
        self.work = torch.zeros(self.nb, dtype=torch.int64)
        X = np.stack([self.f["x"], self.f["y"], self.f["z"]], 1)
        for b in range(max(0, b0), min(b1, self.nb)):
            i0, i1 = b * self.bucket, min(self.n, (b + 1) * self.bucket)
            d = X[None, :, :] - X[i0:i1, None, :]
            r2 = (d * d).sum(-1) + self.f["soft"][None, :] ** 2
            r2[np.arange(i1 - i0), np.arange(i0, i1)] = np.inf  # no self term
            inv = 1.0 / np.sqrt(r2)
            w = self.f["m"][None, :] * inv ** 3
            a = (d * w[..., None]).sum(1)
            for k in range(3):
                self.acc[k][i0:i1] = torch.from_numpy(a[:, k])
            pot = -(self.f["m"][None, :] * inv).sum(1)
            self.acc[3][i0:i1] = torch.from_numpy(pot)
            self.acc[4][i0:i1] = torch.from_numpy(pot)
            self.work[b] = (i1 - i0) * self.n

    def tensors(self):
        return self.acc

    def bucket_work(self):
        return self.work

    def advance(self):
        v2 = max(float((self.f["vx"] ** 2 + self.f["vy"] ** 2 + self.f["vz"] ** 2).max()), 1e-300)
        L = max(np.ptp(self.f[a]) for a in "xyz")
        dt = min(L / np.sqrt(v2) / np.cbrt(self.n), self.dt_max)
        for k, a in zip(("vx", "vy", "vz"), self.acc[:3]):
            self.f[k] += 0.5 * dt * a.numpy()
            self.f[k] += 0.5 * dt * a.numpy()
        for k in "xyz":
            self.f[k] += dt * self.f["v" + k]
        return dt

    def state(self):
        o = np.lexsort((self.f["z"], self.f["y"], self.f["x"]))  # a canonical order to compare
        return {k: v[o] for k, v in self.f.items()}


def particles(n=400, seed=5):
    return ics.plummer(n, seed=seed, soft=0.05)


def test_balanced_cuts():
    rng = np.random.default_rng(1)
    w = rng.integers(1, 1000, 997)
    for world in (1, 2, 3, 7, 16):
        c = balanced_cuts(w, world)
        assert c[0] == 0 and c[-1] == w.size and len(c) == world + 1
        assert all(a <= b for a, b in zip(c, c[1:]))
        loads = [w[a:b].sum() for a, b in zip(c, c[1:])]
        assert max(loads) <= w.sum() / world + w.max()  # within one bucket of the ideal
    # equal weights -> equal counts; zero weights -> equal counts
    assert balanced_cuts(np.ones(12), 4) == [0, 3, 6, 9, 12]
    assert balanced_cuts(np.zeros(12), 4) == [0, 3, 6, 9, 12]
    assert balanced_cuts([], 3) == [0, 0, 0, 0]
    # one heavy bucket: it gets a range of its own
    c = balanced_cuts([1, 1, 1, 100, 1, 1], 2)
    loads = [sum([1, 1, 1, 100, 1, 1][a:b]) for a, b in zip(c, c[1:])]
    assert max(loads) <= 103
    r = rescale_cuts([0, 5, 10, 20], 20, 40)
    assert r == [0, 10, 20, BIG]


def test_emulated_ranks_match_one_rank():
    p = particles()
    ref = ShardedGravity(NumpyEngine(p), 1, 0)
    for _ in range(4):
        ref.step()
    shards = [ShardedGravity(NumpyEngine(p), 3, r) for r in range(3)]
    run_emulated(shards, 4)
    want = ref.engine.state()
    for s in shards:
        got = s.engine.state()
        for k in want:
            assert np.array_equal(got[k], want[k]), k
    # after the first pass the cuts follow the measured work
    assert shards[0].cuts is not None and shards[0].cuts[-1] == shards[0].engine.n_buckets()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out, nsteps):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", world_size=world, rank=rank,
                            timeout=datetime.timedelta(seconds=60))
    try:
        g = ShardedGravity(NumpyEngine(particles()), world, rank)
        dts = [g.step() for _ in range(nsteps)]
        st = g.engine.state()
        np.savez(os.path.join(out, f"rank{rank}.npz"), dts=np.array(dts), cuts=np.array(g.cuts), **st)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_match_one_rank(tmp_path, world):
    import torch.multiprocessing as mp
    nsteps = 3
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path), nsteps), nprocs=world,
                       join=True, start_method="spawn")
    ref = ShardedGravity(NumpyEngine(particles()), 1, 0)
    dts = [ref.step() for _ in range(nsteps)]
    want = ref.engine.state()
    cuts = None
    for r in range(world):
        got = np.load(os.path.join(str(tmp_path), f"rank{r}.npz"))
        assert np.array_equal(got["dts"], np.array(dts))
        for k in want:
            assert np.array_equal(got[k], want[k]), (r, k)
        cuts = got["cuts"] if cuts is None else cuts
        assert np.array_equal(got["cuts"], cuts)  # every rank agrees on the next cut


def test_cuts_properties():
    """Any weights and rank count: the cuts are monotone, start at 0 and end at
    the bucket count, every range is within one bucket of the ideal load, and
    the cuts carried over to a tree of another size still cover every bucket
    once (the last range stays open)."""
    from hypothesis import given, settings, strategies as st

    @settings(max_examples=200, deadline=None)
    @given(st.lists(st.integers(0, 10 ** 6), min_size=0, max_size=300), st.integers(1, 12),
           st.integers(0, 600))
    def check(w, world, nb_new):
        w = np.asarray(w, dtype=np.int64)
        c = balanced_cuts(w, world)
        assert len(c) == world + 1 and c[0] == 0 and c[-1] == w.size
        assert all(a <= b for a, b in zip(c, c[1:]))
        if w.size and w.sum() > 0:
            loads = [int(w[a:b].sum()) for a, b in zip(c, c[1:])]
            assert max(loads) <= w.sum() / world + w.max()
        r = rescale_cuts(c, w.size, nb_new)
        assert r[0] == 0 and r[-1] == BIG and all(a <= b for a, b in zip(r, r[1:]))
        covered = sum(min(b, nb_new) - min(a, nb_new) for a, b in zip(r, r[1:]))
        assert covered == nb_new

    check()

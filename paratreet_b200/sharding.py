"""One N-body system over several ranks (one process per GPU).

Every rank holds all particles and builds the whole tree (cheap next to the
traversal); the DFS-ordered bucket list is cut into contiguous ranges, one
per rank, each traversed by its rank only (``pt_compute_forces_range``).  The
buckets play the role of the reference's Partitions and the ranges that of
its SFC / Oct decompositions (src/Decomposition.C:119-194, :356-453), which
split the key-ordered particles into contiguous pieces; here the cut is
balanced by the measured interactions per bucket of the previous force pass
(``pt_get_bucket_work``) instead of by particle counts.

Exchange, once per step: all ranks built identical trees, so their sorted
particle order is the same, and outside its range every rank's acceleration
and potential arrays are zero.  One sum all-reduce of those five arrays (and
of the per-bucket work) therefore gives every rank the full result, bit for
bit (x + 0 = x), after which every rank advances all particles
(``pt_advance``: the reference's kick + perturb) and stays identical to the
others.  No kernel waits on another rank.

The driver is written against a small engine interface so that the same code
runs the device library (``DeviceEngine``) and, in the CPU tests, a numpy
stand-in under ``gloo``:

    engine.n_buckets() -> int            buckets of the last tree (0 before any)
    engine.compute_range(b0, b1)         tree build + traversal of [b0, b1)
    engine.tensors() -> list[Tensor]     ax, ay, az, pot, pot_full (summed in place)
    engine.bucket_work() -> Tensor       int64 per bucket of the last pass
    engine.advance() -> float            kick + drift with the summed result; dt
"""
from __future__ import annotations

import ctypes as C

import numpy as np

BIG = (1 << 62)  # end of the last range: the library clamps to its bucket count


def balanced_cuts(weights, world: int) -> list[int]:
    """world + 1 cut indices 0 = c_0 <= ... <= c_world = len(weights) so that
    the contiguous ranges [c_r, c_{r+1}) carry as equal a share of the summed
    weights as whole buckets allow (each cut is the bucket boundary nearest to
    its quantile of the prefix sum)."""
    w = np.asarray(weights, dtype=np.float64)
    nb = int(w.size)
    if world < 1:
        raise ValueError("world must be >= 1")
    total = float(w.sum()) if nb else 0.0
    if nb == 0 or total <= 0.0:
        return [r * nb // world for r in range(world)] + [nb]
    pref = np.concatenate([[0.0], np.cumsum(w)])  # pref[k] = work of buckets [0, k)
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        k = int(np.searchsorted(pref, target, side="left"))
        k = min(max(k, 1), nb)
        if k > 1 and abs(pref[k - 1] - target) <= abs(pref[k] - target):
            k -= 1
        cuts.append(max(k, cuts[-1]))
    cuts.append(nb)
    return cuts


def rescale_cuts(cuts: list[int], nb_old: int, nb_new: int) -> list[int]:
    """Carry cut positions over to a rebuilt tree with nb_new buckets (the
    same fractions of the key-ordered list); the last range stays open."""
    world = len(cuts) - 1
    if nb_old <= 0:  # nothing measured (an empty tree): equal bucket counts
        return [r * nb_new // world for r in range(world)] + [BIG]
    out = [0] + [min(nb_new, int(round(c * nb_new / nb_old))) for c in cuts[1:-1]] + [BIG]
    for i in range(1, len(out)):
        out[i] = max(out[i], out[i - 1])
    return out


class ShardedGravity:
    """Bucket-sharded force passes and steps of one system.  ``reduce`` sums a
    list of tensors over the ranks in place (default: torch.distributed
    all_reduce); with ``reduce=None`` and world 1 it is a no-op."""

    def __init__(self, engine, world: int, rank: int, reduce=None):
        if not 0 <= rank < world:
            raise ValueError("rank out of range")
        self.engine, self.world, self.rank = engine, world, rank
        self._reduce = reduce
        self.cuts = None       # world + 1 bucket indices of the coming pass
        self.nb_cuts = 0       # bucket count the cuts refer to
        self.last_work = None  # summed per-bucket work of the last pass

    # one step in three phases, so that ranks emulated in one process can be
    # interleaved (compute on all, exchange, finish on all)
    def compute(self):
        nb = self.engine.n_buckets()
        if self.cuts is None:
            # no measurement yet: equal bucket counts (the tree is built by the pass)
            cuts = [0] + [BIG] * self.world if nb == 0 else \
                [r * nb // self.world for r in range(self.world)] + [BIG]
        else:
            cuts = rescale_cuts(self.cuts, self.nb_cuts, nb) if nb != self.nb_cuts else \
                self.cuts[:-1] + [BIG]
        self._range = (cuts[self.rank], cuts[self.rank + 1])
        if self.world == 1:
            self._range = (0, BIG)
        self.engine.compute_range(*self._range)

    def tensors(self):
        """The tensors a step sums over the ranks: accelerations, potentials
        and the per-bucket work."""
        return self.engine.tensors() + [self.engine.bucket_work()]

    def exchange(self):
        ts = self.tensors()
        if self.world > 1:
            if self._reduce is None:
                import torch.distributed as dist
                for t in ts:
                    dist.all_reduce(t, op=dist.ReduceOp.SUM)
            else:
                self._reduce(ts)
        _synchronize(self.engine)
        self._after_exchange(ts[-1])

    def _after_exchange(self, work):
        self.balance(work)

    def balance(self, work):
        """Cut the next pass's buckets by this per-bucket work (the same on
        every rank: summed over the ranks, or from a full pass)."""
        w = work.cpu().numpy() if hasattr(work, "cpu") else np.asarray(work)
        self.last_work = w
        self.nb_cuts = int(w.size)
        self.cuts = balanced_cuts(w, self.world)

    def finish(self) -> float:
        return self.engine.advance()

    def forces(self):
        """One sharded force pass; every rank ends with the full result."""
        self.compute()
        self.exchange()

    def step(self) -> float:
        """One Driver::run iteration (KKD) over the ranks; returns dt."""
        self.forces()
        return self.finish()


def run_emulated(shards: list[ShardedGravity], nsteps: int) -> list[float]:
    """Steps of several ranks emulated in one process (one device or the CPU):
    every phase runs on all shards before the next; the exchange sums the
    shards' tensors on the host side of the caller and writes them back."""
    dts = []
    for _ in range(nsteps):
        for s in shards:
            s.compute()
        lists = [s.tensors() for s in shards]
        for k in range(len(lists[0])):
            total = lists[0][k].clone()
            for other in lists[1:]:
                total += other[k]
            for ts in lists:
                ts[k].copy_(total)
        for s in shards:
            _synchronize(s.engine)
        for s, ts in zip(shards, lists):
            s._after_exchange(ts[-1])
        dts.append([s.finish() for s in shards][0])
    return dts


def _synchronize(engine):
    """Order the summed tensors before the engine's next launches (the
    library may run on a stream of its own)."""
    sync = getattr(engine, "synchronize", None)
    if sync is not None:
        sync()


class DeviceEngine:
    """The engine interface over a GravitySimulation (device library): the
    five result arrays are wrapped in place as CUDA tensors."""

    def __init__(self, sim):
        import torch
        self.sim, self.torch = sim, torch
        self.device = torch.device("cuda", sim.conf.device)
        self._work = None

    def n_buckets(self) -> int:
        try:
            return int(self.sim.counters()["n_buckets"])
        except Exception:
            return 0

    def compute_range(self, b0: int, b1: int):
        self.sim.start_down(buckets=(b0, b1))

    def tensors(self):
        ptrs = [C.c_void_p() for _ in range(5)]
        order = C.c_void_p()
        self.sim._check(self.sim._lib.pt_device_accel(self.sim._h, *[C.byref(p) for p in ptrs], C.byref(order)))
        return [_wrap_device(int(p.value), self.sim.n, self.device) for p in ptrs]

    def bucket_work(self):
        w = self.sim.bucket_work().astype(np.int64)
        return self.torch.from_numpy(w).to(self.device)

    def advance(self) -> float:
        return self.sim.advance()

    def synchronize(self):
        self.torch.cuda.synchronize(self.device)


class _CudaArray:
    """A device FP64 array exposed through __cuda_array_interface__ (version 3)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None, "stream": None}


def _wrap_device(ptr: int, n: int, device):
    import torch
    with torch.cuda.device(device):
        return torch.as_tensor(_CudaArray(ptr, n), device=device)

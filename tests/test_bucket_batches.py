"""The per-SM bucket batches of the list kernels (grab_bucket in
paratreet_b200/csrc/k_mixed2.cu), restated step by step on the host.

Each warp's grab is a short sequence of atomic operations on its SM's queue
word and on the global counter.  The model interleaves the steps of many
warps at random and checks what the kernels rely on: every bucket index below
the total is handed out exactly once, whatever the interleaving, and every
warp eventually draws an index past the end and leaves.  The CUDA code is
covered by the GPU parity tests (bit-equal lists and results); this covers
the protocol's corner cases (several warps drawing past a batch while its
refill is in flight, the first draw of an empty queue, batches that run past
the end) with far more interleavings than a GPU run shows.
"""
import random

import pytest

MASK32 = (1 << 32) - 1


def grab_steps(state, sm, batch):
    """One warp's grab as a generator of atomic steps; returns the index."""
    old = state["q"][sm]
    state["q"][sm] = (old + 1) & ((1 << 64) - 1)  # atomicAdd(q, 1)
    yield
    hi, idx = old >> 32, old & MASK32
    if hi != 0 and idx < batch:
        return hi - 1 + idx
    if (idx == 0) if hi == 0 else (idx == batch):
        bi = state["work"]
        state["work"] = (bi + batch) & MASK32  # atomicAdd(work, batch)
        yield
        state["q"][sm] = ((bi + 1) << 32) | 1  # atomicExch(q, ...)
        yield
        return bi
    bi = state["work"]
    state["work"] = (bi + 1) & MASK32  # atomicAdd(work, 1)
    yield
    return bi


def warp(state, sm, batch, total, got):
    while True:
        bi = yield from grab_steps(state, sm, batch)
        if bi >= total:
            return
        got.append(bi)
        yield  # the bucket's work: other warps run meanwhile


def run(total, n_sm, warps_per_sm, batch, seed):
    rng = random.Random(seed)
    state = {"q": [0] * n_sm, "work": 0}
    got = []
    live = [warp(state, s, batch, total, got) for s in range(n_sm) for _ in range(warps_per_sm)]
    while live:
        k = rng.randrange(len(live))
        try:
            next(live[k])
        except StopIteration:
            live.pop(k)
    return got


@pytest.mark.parametrize("total,n_sm,warps_per_sm,batch", [
    (1, 1, 1, 32), (31, 2, 3, 32), (32, 1, 28, 32), (33, 1, 28, 32), (1000, 4, 28, 32),
    (5000, 8, 7, 32), (777, 3, 5, 4), (64, 2, 40, 1), (2049, 6, 28, 64),
])
def test_every_bucket_once(total, n_sm, warps_per_sm, batch):
    for seed in range(6):
        got = run(total, n_sm, warps_per_sm, batch, seed)
        assert sorted(got) == list(range(total)), (seed, len(got))


def test_neighbouring_buckets_share_an_sm():
    """With few warps per SM, almost every bucket comes out of a batch: the
    SM's warps work on consecutive buckets."""
    total, batch = 4096, 32
    rng = random.Random(7)
    state = {"q": [0] * 4, "work": 0}
    owner = {}
    live = []
    for s in range(4):
        for _ in range(4):
            got = []
            live.append((s, got, warp(state, s, batch, total, got)))
    while live:
        k = rng.randrange(len(live))
        s, got, g = live[k]
        try:
            next(g)
            for b in got:
                owner[b] = s
        except StopIteration:
            live.pop(k)
    same = sum(owner[b] == owner[b + 1] for b in range(total - 1))
    assert sorted(owner) == list(range(total))
    assert same > 0.9 * (total - 1)

"""Tipsy reader/writer and the .acc output (CPU).  Round trips on seeded
particles in both precisions and byte orders, type ordering, and, where the
reference tree is mounted, its own fixture tests/gravity/lambs.00200_subsamp_30K
and direct.acc against the committed known-answer arrays."""
import os

import numpy as np
import pytest

from paratreet_b200 import ics, tipsy

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# the reference checkout: $PT_REFERENCE, else a sibling of this repository
REF_ROOT = os.environ.get("PT_REFERENCE",
                          os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))),
                                       "reference"))
REF_GRAVITY = os.path.join(REF_ROOT, "tests", "gravity")


def mixed_types(n=300, seed=1):
    p = ics.plummer(n, seed=seed, soft=0.02)
    rng = np.random.default_rng(seed)
    p["type"] = rng.integers(0, 3, n).astype(np.int8)
    return p


@pytest.mark.parametrize("double", [True, False])
def test_round_trip(tmp_path, double):
    p = mixed_types()
    f = str(tmp_path / "a.tipsy")
    tipsy.write_tipsy(f, p, time=0.25, double=double, softening=True)
    q, h = tipsy.read_tipsy(f)
    assert (h.time, h.nbodies, h.ndim) == (0.25, p["x"].size, 3)
    assert (h.nsph, h.ndark, h.nstar) == tuple(int(np.sum(p["type"] == t)) for t in (0, 1, 2))
    # the file holds gas, dark, star in that order; map back through the types
    o = np.concatenate([np.flatnonzero(p["type"] == t) for t in (0, 1, 2)])
    cast = (lambda a: a) if double else (lambda a: a.astype(np.float32).astype(np.float64))
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(q[k], cast(p[k][o])), k
    assert np.array_equal(q["m"], p["m"][o].astype(np.float32).astype(np.float64))
    soft = np.where(p["type"][o] == 2, 0.0, p["soft"][o].astype(np.float32))  # stars: no softening read
    assert np.array_equal(q["soft"], soft)
    assert np.array_equal(q["type"], p["type"][o])


def test_writer_fills_only_mass_position_velocity(tmp_path):
    p = ics.plummer(50, seed=3, soft=0.1)
    f = str(tmp_path / "b.tipsy")
    tipsy.write_tipsy(f, p)
    q, h = tipsy.read_tipsy(f)
    assert h.ndark == 50 and np.all(q["soft"] == 0.0)
    q2, _ = tipsy.read_tipsy(f, soft=0.01)  # Reader::setSoft
    assert np.all(q2["soft"] == 0.01)


def test_native_byte_order_is_read(tmp_path):
    p = ics.plummer(40, seed=4, soft=0.05)
    f = str(tmp_path / "c.tipsy")
    tipsy.write_tipsy(f, p, double=False, softening=True)
    raw = bytearray(open(f, "rb").read())
    # rewrite as little-endian: header fields then every 4-byte word of the records
    le = bytearray(raw)
    le[:8] = raw[:8][::-1]
    for o in range(8, len(raw), 4):
        le[o:o + 4] = raw[o:o + 4][::-1]
    g = str(tmp_path / "c_le.tipsy")
    open(g, "wb").write(bytes(le))
    a, _ = tipsy.read_tipsy(f)
    b, _ = tipsy.read_tipsy(g)
    for k in ("x", "vy", "m", "soft"):
        assert np.array_equal(a[k], b[k])


def test_bad_files_are_rejected(tmp_path):
    f = str(tmp_path / "bad.tipsy")
    open(f, "wb").write(b"\0" * 8)
    with pytest.raises(ValueError):
        tipsy.read_tipsy(f)
    p = ics.plummer(10, seed=5, soft=0.1)
    tipsy.write_tipsy(f, p)
    open(f, "ab").write(b"\0" * 3)
    with pytest.raises(ValueError):
        tipsy.read_tipsy(f)


def test_acc_round_trip(tmp_path):
    rng = np.random.default_rng(7)
    a = rng.normal(size=(3, 123)) * 10.0 ** rng.integers(-8, 3, size=(3, 123))
    f = str(tmp_path / "x.acc")
    tipsy.write_acc(f, *a)
    b = tipsy.read_acc(f)
    assert np.allclose(a, b, rtol=1e-13, atol=0)
    assert open(f).readline() == "123\n"


@pytest.mark.skipif(not os.path.exists(REF_GRAVITY), reason="reference checkout not found (set PT_REFERENCE)")
def test_reference_fixture_reads_like_the_known_answer_arrays():
    kat = np.load(os.path.join(GOLD, "lambs_kat.npz"))
    p, h = tipsy.read_tipsy(os.path.join(REF_GRAVITY, "lambs.00200_subsamp_30K"))
    assert h.nbodies == kat["pos"].shape[0] == h.ndark
    assert np.array_equal(np.stack([p["x"], p["y"], p["z"]], 1), kat["pos"].astype(np.float64))
    assert np.array_equal(p["m"], kat["mass"].astype(np.float64))
    assert np.array_equal(p["soft"], kat["eps"].astype(np.float64))
    acc = tipsy.read_acc(os.path.join(REF_GRAVITY, "direct.acc"))
    assert np.array_equal(acc[:, kat["targets"]].T, kat["acc"])


def test_round_trip_random(tmp_path):
    """Any particle count (none included) and type mix, both precisions: what
    the writer stores, the reader returns (cast to the file's precision), gas,
    dark and star in that order."""
    from hypothesis import given, settings, strategies as st

    @settings(max_examples=60, deadline=None)
    @given(st.integers(0, 200), st.booleans(), st.integers(0, 2 ** 31 - 1))
    def check(n, double, seed):
        rng = np.random.default_rng(seed)
        p = {k: rng.normal(0.0, 1.0, n) for k in ("x", "y", "z", "vx", "vy", "vz")}
        p["m"] = rng.uniform(0.1, 1.0, n)
        p["soft"] = rng.uniform(0.001, 0.1, n)
        p["type"] = rng.integers(0, 3, n).astype(np.int8)
        f = str(tmp_path / f"r{seed}.tipsy")
        tipsy.write_tipsy(f, p, time=1.5, double=double, softening=True)
        q, h = tipsy.read_tipsy(f)
        assert h.nbodies == n and h.time == 1.5
        o = np.concatenate([np.flatnonzero(p["type"] == t) for t in (0, 1, 2)]).astype(np.int64)
        cast = (lambda a: a) if double else (lambda a: a.astype(np.float32).astype(np.float64))
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.array_equal(q[k], cast(p[k][o])), k
        assert np.array_equal(q["type"], p["type"][o])
        os.remove(f)

    check()

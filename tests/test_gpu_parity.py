"""GPU parity tests: the CUDA path through the C ABI against the CPU oracle
(and the reference-sources golden digests).

FP64 form: bit-exact keys, tree topology, moments, interaction lists,
accelerations, potentials and kick/perturb state.  Mixed form: same lists,
forces within 1e-5 rms relative of the FP64 form (FP32 interactions).
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from paratreet_b200 import ics

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(f[4:-5] for f in os.listdir(GOLD) if f.startswith("ref_") and f.endswith(".json"))


def sim(**kw):
    from paratreet_b200.gravity import GravitySimulation
    return GravitySimulation(**kw)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def rel_err(a, b):
    num = np.sqrt((a[0] - b[0]) ** 2 + (a[1] - b[1]) ** 2 + (a[2] - b[2]) ** 2)
    den = np.sqrt(b[0] ** 2 + b[1] ** 2 + b[2] ** 2)
    return num / np.where(den > 0, den, 1.0)


@pytest.mark.parametrize("name", CASES)
def test_fp64_matches_reference_golden(name):
    with open(os.path.join(GOLD, f"ref_{name}.json")) as f:
        g = json.load(f)
    p = getattr(ics, g["generator"])(**g["kwargs"])
    with sim(max_particles_per_leaf=g["bucket"], theta=g["theta"], max_timestep=g["dt_max"],
             record_lists=True) as s:
        s.set_particles(p)
        s.start_down()
        h = g["sha256"]
        assert sha(s.keys()) == h["keys"]
        t = O.sort_tree(s.tree())
        assert t.keys.size == g["n_nodes"]
        assert sha(t.keys) == h["node_keys"]
        assert sha(t.types.astype(np.int32)) == h["node_types"]
        assert sha(t.count.astype(np.int32)) == h["node_counts"]
        assert sha(t.moments) == h["node_moments"]
        L = s.lists()
        assert sha(L.bucket_keys) == h["bucket_keys"]
        assert sha(L.offsets.astype(np.int64)) == h["list_offsets"]
        assert sha(L.keys) == h["list_keys"]
        assert sha(L.kinds.astype(np.int32)) == h["list_kinds"]
        a = s.accelerations()
        for k in ("ax", "ay", "az", "pot"):
            assert sha(a[k]) == h[k], k
        c = s.counters()
        assert (c["n_pp"], c["n_pc"]) == (g["n_pp"], g["n_pc"])


@pytest.mark.parametrize("name", CASES)
def test_fp64_steps_match_reference_golden(name):
    with open(os.path.join(GOLD, f"ref_{name}.json")) as f:
        g = json.load(f)
    p = getattr(ics, g["generator"])(**g["kwargs"])
    with sim(max_particles_per_leaf=g["bucket"], theta=g["theta"], max_timestep=g["dt_max"]) as s:
        s.set_particles(p)
        s.run(g["steps"])
        st = s.state()
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            assert sha(st[k]) == g["after_steps"]["sha256"][k], k
        assert s.last_dt() == g["after_steps"]["last_dt"]


@pytest.mark.parametrize("gen,n,bucket,theta", [
    ("plummer", 20000, 16, 0.7), ("mixture", 50000, 16, 0.7), ("plummer", 30000, 32, 0.5),
    ("hernquist", 20000, 32, 1.0), ("plummer", 5000, 4, 0.7), ("mixture", 20000, 1, 0.7),
])
def test_fp64_bit_exact_vs_oracle(gen, n, bucket, theta):
    p = getattr(ics, gen)(n)
    ref = O.PortSim(p, bucket=bucket, theta=theta, dt_max=0.01, threads=8)
    ref.forces(record_lists=True)
    with sim(max_particles_per_leaf=bucket, theta=theta, max_timestep=0.01, record_lists=True) as s:
        s.set_particles(p)
        s.start_down()
        assert np.array_equal(s.keys(), ref.keys())
        lo, hi = s.universe()
        rlo, rhi = ref.universe()
        assert np.array_equal(lo, rlo) and np.array_equal(hi, rhi)
        tg, tr = O.sort_tree(s.tree()), O.sort_tree(ref.tree())
        assert np.array_equal(tg.keys, tr.keys)
        assert np.array_equal(tg.types, tr.types)
        assert np.array_equal(tg.count, tr.count)
        assert np.array_equal(tg.moments, tr.moments)
        Lg, Lr = s.lists(), ref.lists()
        assert np.array_equal(Lg.bucket_keys, Lr.bucket_keys)
        assert np.array_equal(Lg.offsets, Lr.offsets)
        assert np.array_equal(Lg.keys, Lr.keys)
        assert np.array_equal(Lg.kinds, Lr.kinds)
        a = s.accelerations()
        rax, ray, raz, rpot, rpotf = ref.acc()
        assert np.array_equal(a["ax"], rax)
        assert np.array_equal(a["ay"], ray)
        assert np.array_equal(a["az"], raz)
        assert np.array_equal(a["pot"], rpot)
        assert np.array_equal(a["pot_full"], rpotf)


def test_fp64_mixture_1m_ten_steps():
    """The 2^20 mixture workload: 10 kick/perturb steps at dt=1e-4."""
    p = ics.mixture(1 << 20, seed=7, soft=1e-4)
    ref = O.PortSim(p, bucket=16, theta=0.7, dt_max=1e-4, threads=os.cpu_count() or 8)
    ref.run(10)
    with sim(max_particles_per_leaf=16, theta=0.7, max_timestep=1e-4) as s:
        s.set_particles(p)
        s.run(10)
        st = s.state()
        rs = ref.state()
        for k, r in zip(("x", "y", "z", "vx", "vy", "vz"), rs):
            assert np.array_equal(st[k], r), k
        a = s.accelerations()
        rax, ray, raz, rpot, _ = ref.acc()
        assert np.array_equal(a["ax"], rax) and np.array_equal(a["pot"], rpot)


@pytest.mark.parametrize("gen,n,bucket", [("plummer", 20000, 16), ("mixture", 50000, 32), ("hernquist", 20000, 32)])
def test_mixed_matches_fp64(gen, n, bucket):
    p = getattr(ics, gen)(n)
    with sim(max_particles_per_leaf=bucket, record_lists=True) as s64:
        s64.set_particles(p)
        s64.start_down()
        a64 = s64.accelerations()
        L64 = s64.lists()
    with sim(max_particles_per_leaf=bucket, precision="mixed", record_lists=True) as sm:
        sm.set_particles(p)
        sm.start_down()
        am = sm.accelerations()
        Lm = sm.lists()
    # the same interactions per bucket: the mixed form records its two-phase
    # walk's lists (leaves first, then nodes, in that walk's order), the FP64
    # form the reference's pre-order
    assert np.array_equal(L64.offsets, Lm.offsets)
    for b in range(L64.offsets.size - 1):
        o0, o1 = L64.offsets[b], L64.offsets[b + 1]
        k64 = np.lexsort((L64.keys[o0:o1], L64.kinds[o0:o1]))
        km = np.lexsort((Lm.keys[o0:o1], Lm.kinds[o0:o1]))
        assert np.array_equal(L64.keys[o0:o1][k64], Lm.keys[o0:o1][km]), b
        assert np.array_equal(L64.kinds[o0:o1][k64], Lm.kinds[o0:o1][km]), b
    e = rel_err((am["ax"], am["ay"], am["az"]), (a64["ax"], a64["ay"], a64["az"]))
    assert np.sqrt(np.mean(e ** 2)) < 1e-5
    assert np.max(e) < 1e-3
    pe = np.abs(am["pot_full"] - a64["pot_full"]) / np.abs(a64["pot_full"])
    assert np.sqrt(np.mean(pe ** 2)) < 1e-5
    # the reference's potential: quadrupole node() terms only (monopole nodes
    # and leaves apply none), measured against the full potential's size
    qe = np.abs(am["pot"] - a64["pot"]) / np.abs(a64["pot_full"])
    assert np.sqrt(np.mean(qe ** 2)) < 1e-5 and np.max(qe) < 1e-3


def test_mixed_matches_fp64_full_size():
    """The 2^24 Plummer workload (eps 1e-3, bucket 32, theta 0.7): both forms
    make the same interactions (P2P pairs, P2C evaluations and opening tests
    counted on the device, and every bucket's list: the FP64 walk's recorded
    list and the mixed form's two-phase list have equal order-independent
    digests and lengths) and the mixed accelerations stay within 1e-5 RMS of
    the FP64 ones over all particles."""
    p = ics.plummer(1 << 24, seed=42, soft=1e-3)
    out = {}
    for prec in ("fp64", "mixed"):
        with sim(max_particles_per_leaf=32, theta=0.7, precision=prec, record_lists=(prec == "fp64")) as s:
            s.set_particles(p)
            s.start_down()
            dig = s.list_digests("recorded" if prec == "fp64" else "two_phase")
            out[prec] = (s.accelerations(), s.counters(), dig, s.bucket_keys())
    (a64, c64, d64, k64), (am, cm, dm, km) = out["fp64"], out["mixed"]
    for k in ("n_pp", "n_pc", "n_open", "n_nodes", "n_buckets"):
        assert c64[k] == cm[k], k
    assert np.array_equal(k64, km)
    assert np.array_equal(d64[1], dm[1]), "list lengths differ"
    assert np.array_equal(d64[0], dm[0]), "list digests differ"
    assert all(np.all(np.isfinite(am[k])) for k in ("ax", "ay", "az", "pot", "pot_full"))
    e = rel_err((am["ax"], am["ay"], am["az"]), (a64["ax"], a64["ay"], a64["az"]))
    assert np.sqrt(np.mean(e ** 2)) < 1e-5


@pytest.mark.parametrize("prec", ["mixed", "fp64_lists"])
def test_list_relocation_keeps_lists(prec):
    """Warp regions of 64 entries instead of 32768: nearly every bucket's list
    outgrows what is left of its region and moves while the walk writes it.
    The lists (order-independent digests and lengths), the counts and the
    accelerations and potentials are the same bit for bit."""
    p = ics.plummer(200000, seed=21, soft=1e-3)
    res = []
    for region in (32768, 64):
        with sim(max_particles_per_leaf=32, theta=0.5, precision=prec) as s:
            s.set_list_region(region)
            s.set_particles(p)
            s.start_down()
            s.start_down()
            res.append((s.accelerations(), s.counters(), s.list_digests("two_phase")))
    (a, c, d), (b, cb, db) = res
    assert (c["n_pp"], c["n_pc"], c["n_open"]) == (cb["n_pp"], cb["n_pc"], cb["n_open"])
    assert np.array_equal(d[1], db[1]) and np.array_equal(d[0], db[0])
    for k in ("ax", "ay", "az", "pot", "pot_full"):
        assert np.array_equal(a[k], b[k]), k
    with sim() as s:
        with pytest.raises(Exception):
            s.set_list_region(63)


@pytest.mark.parametrize("gen,n,bucket,soft,theta", [("plummer", 200000, 32, 1e-3, 0.7),
                                                      ("mixture", 150000, 16, 1e-4, 0.7),
                                                      ("hernquist", 50000, 16, 0.05, 0.5)])
def test_fp64_lists_matches_ordered_fp64(gen, n, bucket, soft, theta):
    """The FP64 comparator of the mixed form (PT_FP64_LISTS: the two-phase
    lists evaluated in FP64) against the ordered FP64 walk (bit-exact with the
    reference): the same interactions, and accelerations and potentials equal
    up to the order of each particle's sums."""
    p = getattr(ics, gen)(n, seed=9, soft=soft)
    out = {}
    for prec in ("fp64", "fp64_lists"):
        with sim(max_particles_per_leaf=bucket, theta=theta, precision=prec) as s:
            s.set_particles(p)
            s.start_down()
            s.start_down()
            out[prec] = (s.accelerations(), s.counters())
    (a, c), (b, cl) = out["fp64"], out["fp64_lists"]
    assert (c["n_pp"], c["n_pc"], c["n_open"]) == (cl["n_pp"], cl["n_pc"], cl["n_open"])
    da = np.sqrt((b["ax"] - a["ax"]) ** 2 + (b["ay"] - a["ay"]) ** 2 + (b["az"] - a["az"]) ** 2)
    am = np.sqrt(a["ax"] ** 2 + a["ay"] ** 2 + a["az"] ** 2)
    rel = da / am
    print(f"fp64_lists vs fp64 {gen} n={n}: acc rel rms {np.sqrt(np.mean(rel ** 2)):.2e} max {rel.max():.2e}; "
          f"|da| max / rms|a| {da.max() / np.sqrt(np.mean(am ** 2)):.2e}")
    assert np.sqrt(np.mean(rel ** 2)) < 1e-13
    assert rel.max() < 1e-11
    for k in ("pot", "pot_full"):
        dp = np.abs(b[k] - a[k]) / np.abs(a["pot_full"])
        assert dp.max() < 1e-12, k


@pytest.mark.parametrize("gen,n,bucket", [("plummer", 60000, 32), ("mixture", 40000, 16)])
def test_mixed_fused_fallback_matches_two_phase(gen, n, bucket, monkeypatch):
    """The fused walk-and-evaluate kernel (taken when the list pools cannot be
    allocated; PT_MIXED_FUSED=1 forces it) against the default two-phase
    traversal: the same interactions, FP32 sums in another order."""
    p = getattr(ics, gen)(n, seed=5)
    res = []
    for fused in ("0", "1"):
        monkeypatch.setenv("PT_MIXED_FUSED", fused)
        with sim(max_particles_per_leaf=bucket, precision="mixed") as s:
            s.set_particles(p)
            s.start_down()
            s.start_down()  # a second pass: the two-phase pools are sized by the first
            res.append((s.accelerations(), s.counters()))
    (a2, c2), (af, cf) = res
    assert (c2["n_pp"], c2["n_pc"], c2["n_open"]) == (cf["n_pp"], cf["n_pc"], cf["n_open"])
    e = rel_err((af["ax"], af["ay"], af["az"]), (a2["ax"], a2["ay"], a2["az"]))
    assert np.sqrt(np.mean(e ** 2)) < 1e-6
    assert np.max(e) < 1e-4
    pe = np.abs(af["pot_full"] - a2["pot_full"]) / np.abs(a2["pot_full"])
    assert np.sqrt(np.mean(pe ** 2)) < 1e-6


def test_direct_sum_matches_oracle():
    p = ics.plummer(6000, seed=9, soft=0.01)
    tgt = np.arange(0, 6000, 7, dtype=np.int32)
    rax, ray, raz, rpot = O.direct_sum(p, tgt, threads=8)
    with sim() as s:
        s.set_particles(p)
        ax, ay, az, pot = s.direct_sum(tgt)
    # the device sum splits the sources into slices (reassociation only)
    e = rel_err((ax, ay, az), (rax, ray, raz))
    assert e.max() < 1e-12
    assert np.max(np.abs(pot - rpot) / np.abs(rpot)) < 1e-12


def test_direct_sum_split_known_answer():
    """GPU direct sum (source-split) vs the reference's direct.acc."""
    z = np.load(os.path.join(GOLD, "lambs_kat.npz"))
    pos = z["pos"].astype(np.float64)
    n = pos.shape[0]
    p = {"x": pos[:, 0].copy(), "y": pos[:, 1].copy(), "z": pos[:, 2].copy(), "vx": np.zeros(n),
         "vy": np.zeros(n), "vz": np.zeros(n), "m": z["mass"].astype(np.float64),
         "soft": z["eps"].astype(np.float64)}
    with sim() as s:
        s.set_particles(p)
        ax, ay, az, _ = s.direct_sum(z["targets"])
    e = rel_err((ax, ay, az), tuple(z["acc"].T))
    assert e.max() <= 1e-6 and np.sqrt(np.mean(e ** 2)) <= 1e-7


@pytest.mark.parametrize("n", [0, 1, 2, 3, 16, 17, 33])
def test_tiny_inputs(n):
    p = ics.plummer(max(n, 1))
    if n == 0:
        p = {k: v[:0] for k, v in p.items()}
    ref = O.PortSim(p, bucket=16)
    ref.forces()
    with sim(max_particles_per_leaf=16) as s:
        s.set_particles(p)
        s.start_down()
        if n:
            a = s.accelerations()
            rax = ref.acc()[0]
            assert np.array_equal(a["ax"], rax)


def test_duplicate_positions_depth_limit():
    p = ics.plummer(300)
    for k in ("x", "y", "z"):
        p[k][:40] = p[k][0]
    ref = O.PortSim(p, bucket=16)
    ref.forces()
    with sim(max_particles_per_leaf=16) as s:
        s.set_particles(p)
        s.start_down()
        a = s.accelerations()
        assert np.array_equal(a["ax"], ref.acc()[0])
        assert s.tree().depth.max() == 21


def test_nonfinite_input_is_reported():
    from paratreet_b200._lib import PtError
    p = ics.plummer(1000)
    p["y"][17] = np.nan
    with sim() as s:
        s.set_particles(p)
        with pytest.raises(PtError) as e:
            s.start_down()
        assert e.value.code == -6
        # the handle stays usable
        s.set_particles(ics.plummer(1000))
        s.start_down()


def test_bucket_ranges_partition_the_pass():
    p = ics.plummer(30000, seed=4)
    with sim(max_particles_per_leaf=16) as s:
        s.set_particles(p)
        s.start_down()
        full = s.accelerations()
        nb = s.counters()["n_buckets"]
        parts = []
        for b0, b1 in ((0, nb // 3), (nb // 3, nb)):
            s.start_down(buckets=(b0, b1))
            parts.append(s.accelerations())
    ax = parts[0]["ax"] + parts[1]["ax"]
    assert np.array_equal(ax, full["ax"])


def test_zero_mass_particles():
    p = ics.plummer(5000, seed=11)
    p["m"][::3] = 0.0
    ref = O.PortSim(p, bucket=8)
    ref.forces(record_lists=True)
    with sim(max_particles_per_leaf=8, record_lists=True) as s:
        s.set_particles(p)
        s.start_down()
        tg, tr = O.sort_tree(s.tree()), O.sort_tree(ref.tree())
        assert np.array_equal(tg.moments, tr.moments)
        assert np.array_equal(s.accelerations()["ax"], ref.acc()[0])


@pytest.mark.parametrize("gen,n,bucket,theta", [("plummer", 6000, 16, 0.7), ("mixture", 20000, 32, 0.5),
                                                ("hernquist", 3000, 1, 1.0)])
def test_fp64_basic_down_bit_exact_vs_oracle(gen, n, bucket, theta):
    """Partition::startBasicDown: the FP64 walk in breadth-first order matches
    the oracle bit for bit (accelerations, potentials, interaction lists)."""
    p = getattr(ics, gen)(n, seed=13)
    o = O.PortSim(p, bucket=bucket, theta=theta, threads=8)
    o.set_basic_down()
    o.forces(record_lists=True)
    want = o.acc()
    lo = o.lists()
    with sim(max_particles_per_leaf=bucket, theta=theta, traversal="basic", record_lists=True) as s:
        s.set_particles(p)
        s.start_down()
        a = s.accelerations()
        lg = s.lists()
    for k, w in zip(("ax", "ay", "az", "pot", "pot_full"), want):
        assert np.array_equal(a[k], w), k
    assert np.array_equal(lg.offsets, lo.offsets) and np.array_equal(lg.keys, lo.keys)
    assert np.array_equal(lg.kinds, lo.kinds)


@pytest.mark.parametrize("name", sorted(f[6:-5] for f in os.listdir(GOLD) if f.startswith("basic_")))
def test_fp64_basic_down_matches_reference_golden(name):
    with open(os.path.join(GOLD, f"basic_{name}.json")) as f:
        g = json.load(f)
    p = getattr(ics, g["generator"])(**g["kwargs"])
    with sim(max_particles_per_leaf=g["bucket"], theta=g["theta"], traversal="basic") as s:
        s.set_particles(p)
        s.start_down()
        a = s.accelerations()
    for k in ("ax", "ay", "az", "pot"):
        assert sha(a[k]) == g["sha256"][k], k

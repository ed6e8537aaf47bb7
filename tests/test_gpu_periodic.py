"""GPU tests of the periodic path: (2n+1)^3 replica walks (examples/Gravity.C
traversalFn) plus the Ewald correction (examples/Ewald.{h,C}), and the FP64
periodic direct sum used as the force-error yardstick.

The tree part of the FP64 periodic pass is evaluated exactly like the C
oracle; the Ewald correction calls CUDA's erf/erfc/exp/sincos where the
oracle calls the host libm, so the comparison allows 1e-10 relative per
particle (the C oracle itself is bit-exact against the reference's sources,
tests/test_oracle.py)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from paratreet_b200 import ics

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def sim(**kw):
    from paratreet_b200.gravity import GravitySimulation
    return GravitySimulation(**kw)


def vec_rel(a, b):
    """Per-particle |a - b| / |b| over the three acceleration components."""
    d = np.sqrt(sum((a[k] - b[k]) ** 2 for k in range(3)))
    s = np.sqrt(sum(b[k] ** 2 for k in range(3)))
    return d / np.maximum(s, 1e-300)


def port_periodic(p, bucket, theta, nrep, **kw):
    s = O.PortSim(p, bucket=bucket, theta=theta, threads=8)
    s.set_periodic(1.0, nrep, **kw)
    s.forces()
    return s.acc()


@pytest.mark.parametrize("name", sorted(f[9:-5] for f in os.listdir(GOLD) if f.startswith("periodic_")))
def test_fp64_periodic_matches_golden_case(name):
    with open(os.path.join(GOLD, f"periodic_{name}.json")) as f:
        g = json.load(f)
    p = ics.lattice(**g["kwargs"])
    want = port_periodic(p, g["bucket"], g["theta"], g["n_replicas"])
    with sim(max_particles_per_leaf=g["bucket"], theta=g["theta"], periodic=True,
             n_replicas=g["n_replicas"], period=g["period"]) as s:
        s.set_particles(p)
        s.start_down()
        a = s.accelerations()
    e = vec_rel([a["ax"], a["ay"], a["az"]], want[:3])
    print(name, "max rel %.3e" % e.max())
    assert e.max() < 1e-10
    assert np.abs(a["pot"] - want[3]).max() <= 1e-10 * np.abs(want[3]).max()
    assert np.abs(a["pot_full"] - want[4]).max() <= 1e-10 * np.abs(want[4]).max()
    # the sampled values of the reference's own sources
    idx = g["samples"]["idx"]
    assert np.allclose(a["ax"][idx], g["samples"]["ax"], rtol=1e-10, atol=1e-12 * np.abs(want[0]).max())


@pytest.mark.parametrize("nrep,bucket,theta,hcut", [(0, 16, 0.7, 2.8), (1, 8, 1.0, 10 ** 0.5), (2, 32, 0.5, 2.0)])
def test_fp64_periodic_matches_oracle(nrep, bucket, theta, hcut):
    p = ics.lattice(14, seed=4, rms_cells=0.35, soft_cells=0.5)
    want = port_periodic(p, bucket, theta, nrep, hcut=hcut)
    with sim(max_particles_per_leaf=bucket, theta=theta, periodic=True, n_replicas=nrep,
             ewald_hcut=hcut) as s:
        s.set_particles(p)
        s.start_down()
        a = s.accelerations()
    e = vec_rel([a["ax"], a["ay"], a["az"]], want[:3])
    assert e.max() < 1e-10, e.max()
    assert np.abs(a["pot_full"] - want[4]).max() <= 1e-10 * np.abs(want[4]).max()


def test_mixed_periodic_matches_fp64():
    p = ics.lattice(20, seed=11, rms_cells=0.25, soft_cells=0.5)
    out = {}
    for prec in ("fp64", "mixed"):
        with sim(max_particles_per_leaf=32, theta=0.7, periodic=True, n_replicas=1, precision=prec) as s:
            s.set_particles(p)
            s.start_down()
            out[prec] = s.accelerations()
    d, m = out["fp64"], out["mixed"]
    e = vec_rel([m["ax"], m["ay"], m["az"]], [d["ax"], d["ay"], d["az"]])
    print("mixed vs fp64 periodic: rms %.3e max %.3e" % (np.sqrt(np.mean(e * e)), e.max()))
    # the net force on a displaced lattice is a small residual of large terms
    assert np.sqrt(np.mean(e * e)) < 2e-4
    # the periodic potential is a residual of replica sums of size G M / L = 1:
    # FP32 interaction error is relative to those sums, not to the residual
    assert np.abs(m["pot_full"] - d["pot_full"]).max() < 1e-5


def test_periodic_bucket_ranges_partition_the_pass():
    p = ics.lattice(12, seed=2, rms_cells=0.3, soft_cells=0.5)
    with sim(max_particles_per_leaf=16, periodic=True, n_replicas=1) as s:
        s.set_particles(p)
        s.start_down()
        full = s.accelerations()
        nb = s.bucket_keys().size
        parts = []
        for rng in ((0, nb // 3), (nb // 3, nb)):
            s.start_down(buckets=rng)
            parts.append(s.accelerations())
    hit = [np.abs(q["ax"]) + np.abs(q["ay"]) + np.abs(q["az"]) > 0 for q in parts]
    assert not np.any(hit[0] & hit[1])
    assert np.all(hit[0] | hit[1])
    for q, h in zip(parts, hit):
        for k in ("ax", "ay", "az", "pot", "pot_full"):
            assert np.array_equal(q[k][h], full[k][h]), k


def test_ewald_direct_sum_matches_oracle():
    p = ics.lattice(16, seed=11, rms_cells=0.25, soft_cells=0.5)
    tg = np.arange(0, p["x"].size, 61, dtype=np.int32)
    want = O.ewald_direct_sum(p, tg, 1.0, threads=8)
    with sim(periodic=True, n_replicas=1) as s:
        s.set_particles(p)
        got = s.ewald_direct_sum(tg)
    e = vec_rel(got[:3], want[:3])
    assert e.max() < 1e-10, e.max()
    assert np.abs(got[3] - want[3]).max() < 1e-10 * np.abs(want[3]).max()


def test_periodic_tree_converges_to_ewald_direct_sum():
    """Accuracy of the reference method on the GPU: at theta 0.3 with two
    replica shells the tree + Ewald correction is within a few 1e-3 of the
    Ewald direct sum (the residual is the quadrupole truncation of the root
    expansion used for the far images)."""
    p = ics.lattice(16, seed=11, rms_cells=0.25, soft_cells=0.5)
    tg = np.arange(0, p["x"].size, 64, dtype=np.int32)
    with sim(max_particles_per_leaf=16, theta=0.3, periodic=True, n_replicas=2) as s:
        s.set_particles(p)
        s.start_down()
        a = s.accelerations()
        d = s.ewald_direct_sum(tg)
    e = vec_rel([a["ax"][tg], a["ay"][tg], a["az"][tg]], d[:3])
    print("tree vs Ewald direct: rms %.3e max %.3e" % (np.sqrt(np.mean(e * e)), e.max()))
    assert np.sqrt(np.mean(e * e)) < 5e-3
    assert np.abs(a["pot_full"][tg] - d[3]).max() < 1e-3 * np.abs(d[3]).max() + 1e-3


def test_periodic_steps_match_oracle():
    """Driver::run in periodic mode (kick, drift, new universe, rekey)."""
    p = ics.lattice(10, seed=6, rms_cells=0.3, soft_cells=0.5)
    p["vx"][:] = 0.1
    o = O.PortSim(p, bucket=16, theta=0.7, dt_max=1e-3, threads=8)
    o.set_periodic(1.0, 1)
    o.run(2)
    want = o.state()
    with sim(max_particles_per_leaf=16, theta=0.7, periodic=True, n_replicas=1, max_timestep=1e-3,
             integrator="kkd") as s:
        s.set_particles(p)
        s.run(2)
        st = s.state()
    for k, w in zip(("x", "y", "z", "vx", "vy", "vz"), want):
        assert np.allclose(st[k], w, rtol=1e-12, atol=1e-13), k

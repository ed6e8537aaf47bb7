"""GPU tests of the SPH density pass (pt_sph_density): the reference's
DensityVisitor k = 32 neighbour search and DensityFn on the gravity tree.
Neighbour sets, their d2 and the ball radii must equal the C oracle's bit for
bit (which equals the reference's own sources, tests/test_oracle.py);
densities differ only in the summation order of their 32 terms (1e-13)."""
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


@pytest.mark.parametrize("gen,n,bucket", [("plummer", 5000, 16), ("mixture", 12000, 32), ("hernquist", 4000, 8),
                                          ("plummer", 1000, 1)])
def test_sph_density_matches_oracle(gen, n, bucket):
    p = getattr(ics, gen)(n, seed=21)
    with sim(max_particles_per_leaf=bucket) as s:
        s.set_particles(p)
        d, b, nbr, nd2 = s.sph_density(neighbors=True)
    dp, bp, nbp, nd2p = O.sph_density(p, threads=8)
    assert np.array_equal(nbr, nbp)
    assert np.array_equal(nd2, nd2p)
    assert np.array_equal(b, bp)
    assert np.allclose(d, dp, rtol=1e-13, atol=0)


@pytest.mark.parametrize("name", sorted(f[4:-5] for f in os.listdir(GOLD) if f.startswith("sph_")))
def test_sph_density_matches_reference_golden(name):
    import hashlib
    with open(os.path.join(GOLD, f"sph_{name}.json")) as f:
        g = json.load(f)
    p = getattr(ics, g["generator"])(**g["kwargs"])
    with sim(max_particles_per_leaf=g["bucket"]) as s:
        s.set_particles(p)
        d, b, nbr, nd2 = s.sph_density(neighbors=True)
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()  # noqa: E731
    assert sha(nbr.astype(np.int32)) == g["sha256"]["nbr"]
    assert sha(nd2) == g["sha256"]["nbr_d2"]
    assert sha(b) == g["sha256"]["ball_sq"]
    assert np.allclose(d[g["samples"]["idx"]], g["samples"]["density"], rtol=1e-13, atol=0)


def test_sph_density_large_brute_force_sample():
    """N = 2^20 mixture: for 48 seeded particles the 32nd smallest d2 over all
    particles (numpy, same expression) equals the ball radius bit for bit."""
    p = ics.mixture(1 << 20, seed=7)
    with sim(max_particles_per_leaf=16) as s:
        s.set_particles(p)
        d, b = s.sph_density()
    rng = np.random.default_rng(5)
    for i in rng.choice(p["x"].size, 48, replace=False):
        dx, dy, dz = p["x"][i] - p["x"], p["y"][i] - p["y"], p["z"][i] - p["z"]
        d2 = dx * dx + dy * dy + dz * dz
        assert b[i] == np.partition(d2, 31)[31]
    assert np.all(np.isfinite(d)) and np.all(d > 0)


@pytest.mark.parametrize("n", [1, 2, 31, 33])
def test_sph_density_tiny(n):
    p = ics.plummer(max(n, 2), seed=3, soft=0.05)
    p = {k: v[:n].copy() for k, v in p.items()}
    with sim(max_particles_per_leaf=16) as s:
        s.set_particles(p)
        d, b, nbr, nd2 = s.sph_density(neighbors=True)
    dp, bp, nbp, nd2p = O.sph_density(p)
    assert np.array_equal(nbr, nbp) and np.array_equal(b, bp)
    assert np.allclose(d, dp, rtol=1e-13, atol=0, equal_nan=True)


def test_sph_density_then_forces():
    """A density pass re-sorts the particles; the next force pass is unaffected."""
    p = ics.plummer(3000, seed=4, soft=0.01)
    with sim(max_particles_per_leaf=16) as s:
        s.set_particles(p)
        s.start_down()
        a0 = s.accelerations()
        s.sph_density()
        from paratreet_b200._lib import PtError
        with pytest.raises(PtError):
            s.accelerations()
        s.start_down()
        a1 = s.accelerations()
    for k in ("ax", "ay", "az"):
        assert np.array_equal(a0[k], a1[k])

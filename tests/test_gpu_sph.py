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


def _with_velocities(p, seed=8):
    rng = np.random.default_rng(seed)
    n = p["x"].size
    for k in ("vx", "vy", "vz"):
        p[k] = p[k] + rng.normal(0.0, 0.3, n)
    return p, rng.uniform(0.2, 2.0, n)


def _close(got, want, rel):
    scale = max(float(np.abs(want).max()), 1e-300)
    return float(np.abs(got - want).max()) <= rel * scale


@pytest.mark.parametrize("gen,n,bucket", [("plummer", 5000, 16), ("mixture", 12000, 32), ("hernquist", 4000, 8),
                                          ("plummer", 1000, 1)])
def test_sph_pressure_matches_oracle(gen, n, bucket):
    """Pressure accelerations and PdV work against the C oracle's ForceFn /
    doSPHCalc: the neighbour sets are the same, the sums differ in order only
    (warp sums, atomic reactions): within 1e-12 of the largest value."""
    p, u = _with_velocities(getattr(ics, gen)(n, seed=21))
    with sim(max_particles_per_leaf=bucket) as s:
        s.set_particles(p)
        d, ax, ay, az, pdv = s.sph_pressure(u)
    dp, bp, nbp, nd2p = O.sph_density(p, threads=8)
    want = O.sph_pressure(p, u, dp, bp, nbp, nd2p)
    assert np.allclose(d, dp, rtol=1e-13, atol=0)
    for got, w in zip((ax, ay, az, pdv), want):
        assert _close(got, w, 1e-12)


@pytest.mark.parametrize("name", sorted(f[4:-5] for f in os.listdir(GOLD) if f.startswith("sph_")))
def test_sph_pressure_matches_reference_golden(name):
    with open(os.path.join(GOLD, f"sph_{name}.json")) as f:
        g = json.load(f)
    pr = g["pressure"]
    p = getattr(ics, g["generator"])(**g["kwargs"])
    u = np.random.default_rng(17).uniform(0.5, 1.5, p["x"].size)
    with sim(max_particles_per_leaf=g["bucket"]) as s:
        s.set_particles(p)
        out = s.sph_pressure(u)[1:]
    for k, v in zip(("ax", "ay", "az", "pdv"), out):
        scale = max(pr["pdv_scale"] if k == "pdv" else pr["acc_scale"], 1e-300)
        assert np.all(np.abs(v[pr["idx"]] - np.asarray(pr[k])) <= 1e-12 * scale), k
        assert abs(np.abs(v).sum() - pr["l1"][k]) <= 1e-12 * max(pr["l1"][k], 1e-300), k


def test_sph_pressure_large_momentum_and_sample():
    """N = 2^20 mixture: the pass conserves momentum (sum m a = 0 to
    summation order), and for 32 seeded particles whose neighbours' neighbour
    lists are all recomputed by brute force the acceleration and PdV match a
    numpy restatement of ForceFn and doSPHCalc including every reaction."""
    p, u = _with_velocities(ics.mixture(1 << 20, seed=7))
    n = p["x"].size
    with sim(max_particles_per_leaf=16) as s:
        s.set_particles(p)
        _, ball = s.sph_density()
        d, ax, ay, az, pdv = s.sph_pressure(u)
    acc = (ax, ay, az)
    assert all(np.all(np.isfinite(a)) for a in acc + (pdv,))
    mom = [abs(float(np.sum(p["m"] * a))) for a in acc]
    scale = float(np.sum(p["m"] * (np.abs(ax) + np.abs(ay) + np.abs(az))))
    assert max(mom) <= 1e-12 * scale
    # the density pass's own checks cover the neighbour search; here the
    # pressure sums of sampled particles are rebuilt from the pass's densities
    X = np.stack([p["x"], p["y"], p["z"]], 1)
    V = np.stack([p["vx"], p["vy"], p["vz"]], 1)
    rng = np.random.default_rng(5)

    def knn(i):
        d2 = ((X[i] - X) ** 2).sum(1)
        j = np.argpartition(d2, 31)[:32]
        return j, d2[j]

    def terms(i):
        """(reaction on each neighbour j of i, i's own sum) as doSPHCalc forms them."""
        j, d2 = knn(i)
        rsq = d2.max()
        fb = np.sqrt(rsq)
        ih2 = 4.0 / rsq
        dk = lambda a: np.where(a < 1.0, -3 + 2.25 * np.sqrt(a),  # noqa: E731
                                -0.75 * (2.0 - np.sqrt(a)) ** 2 / np.maximum(np.sqrt(a), 1e-300))
        rs = dk(d2 * ih2) * d2 * p["m"][j]
        divvi, divvj = rs.sum() / d[i], (rs / d[j]).sum()
        corr = divvi / divvj if divvj != 0.0 else 1.0
        ih2b = 4.0 / (fb * fb)
        fn = 0.5 / np.pi * ih2b * ih2b / (0.5 * fb)
        dx = X[j] - X[i]
        r2 = (dx * dx).sum(1)
        r1 = dk(r2 * ih2b) * fn * corr
        aP, bP = u[i] * (2.0 / 3.0) / d[j], u[j] * (2.0 / 3.0) / d[i]
        dvdr = ((V[j] - V[i]) * dx).sum(1)
        own_a = ((aP + bP) * r1 * p["m"][j])[:, None] * dx
        own_w = r1 * p["m"][j] * aP * dvdr
        opp_a = -((aP + bP) * r1 * p["m"][i])[:, None] * dx
        opp_w = r1 * p["m"][i] * aP * dvdr
        return j, own_a.sum(0), own_w.sum(), opp_a, opp_w

    amax = max(float(np.abs(a).max()) for a in acc)
    wmax = float(np.abs(pdv).max())
    for i in rng.choice(n, 16, replace=False):
        j_i, own_a, own_w, _, _ = terms(i)
        tot_a, tot_w = own_a.copy(), own_w
        # reactions: every q that has i among its 32 nearest, i.e. whose ball
        # (the pass's 32nd smallest d2) reaches i
        d2i = ((X - X[i]) ** 2).sum(1)
        cand = np.nonzero(d2i <= ball)[0]
        for q in cand:
            if q == i:
                continue
            j_q, _, _, opp_a, opp_w = terms(q)
            hit = np.nonzero(j_q == i)[0]
            if hit.size:
                tot_a += opp_a[hit[0]]
                tot_w += opp_w[hit[0]]
        got = np.array([ax[i], ay[i], az[i]])
        assert np.all(np.abs(got - tot_a) <= 1e-9 * amax), i
        assert abs(pdv[i] - tot_w) <= 1e-9 * max(wmax, 1e-300), i


@pytest.mark.parametrize("n", [2, 31, 33])
def test_sph_pressure_tiny(n):
    p = ics.plummer(max(n, 2), seed=3, soft=0.05)
    p = {k: v[:n].copy() for k, v in p.items()}
    u = np.linspace(0.5, 1.5, n)
    with sim(max_particles_per_leaf=16) as s:
        s.set_particles(p)
        d, ax, ay, az, pdv = s.sph_pressure(u)
    dp, bp, nbp, nd2p = O.sph_density(p)
    want = O.sph_pressure(p, u, dp, bp, nbp, nd2p)
    for got, w in zip((ax, ay, az, pdv), want):
        assert _close(got, w, 1e-12)


@pytest.mark.parametrize("ngrid,bucket", [(8, 16), (16, 32)])
def test_sph_density_exact_ties_on_a_lattice(ngrid, bucket):
    """Exactly equal distances (a perfect lattice): ball^2 bit-exact, density
    to summation order and every neighbour inside the ball as the C oracle's;
    which of the particles at exactly the ball's distance fill the last slots
    is a tie the reference leaves open."""
    p = ics.lattice(ngrid, seed=1, rms_cells=0.0)
    with sim(max_particles_per_leaf=bucket) as s:
        s.set_particles(p)
        d, b, nbr, nd2 = s.sph_density(neighbors=True)
    dp, bp, nbp, nd2p = O.sph_density(p)
    assert np.array_equal(b, bp)
    assert np.allclose(d, dp, rtol=1e-13, atol=0)
    for i in range(p["x"].size):
        assert set(nbr[i][nd2[i] < b[i]].tolist()) == set(nbp[i][nd2p[i] < bp[i]].tolist()), i
        assert np.all(nd2[i][nbr[i] >= 0] <= b[i])


def _step_state(s, u, up, vp):
    st = s.state()
    return dict(st, u=u, u_pred=up, vpx=vp[0], vpy=vp[1], vpz=vp[2])


@pytest.mark.parametrize("gen,n,bucket,steps", [("plummer", 4000, 16, 3), ("mixture", 6000, 32, 2)])
def test_sph_step_matches_oracle(gen, n, bucket, steps):
    """Iterations of the SPH example (pt_sph_step: density, pressure with the
    predicted energies and velocities, kick + perturb with the u updates)
    against the C oracle's: same neighbour sets each step, sums in another
    order (warp sums, atomic reactions), so within 1e-12 of each field's
    largest value."""
    p, u = _with_velocities(getattr(ics, gen)(n, seed=21))
    rng = np.random.default_rng(9)
    up = u * rng.uniform(0.9, 1.1, n)
    vp = tuple(p[k] + rng.normal(0.0, 0.01, n) for k in ("vx", "vy", "vz"))
    with sim(max_particles_per_leaf=bucket, max_timestep=0.01) as s:
        s.set_particles(p)
        gu, gup, gvp = s.sph_run(steps, u, up, vp)
        got = _step_state(s, gu, gup, gvp)
    q, pu, pup, pvp = O.sph_step(p, steps, 0.01, u, up, vp, threads=8)
    want = dict(q, u=pu, u_pred=pup, vpx=pvp[0], vpy=pvp[1], vpz=pvp[2])
    for k in ("x", "y", "z", "vx", "vy", "vz", "u", "u_pred", "vpx", "vpy", "vpz"):
        assert _close(got[k], want[k], 1e-12), k
    assert not np.allclose(got["x"], p["x"])


@pytest.mark.parametrize("name", sorted(f[8:-5] for f in os.listdir(GOLD) if f.startswith("sphstep_")))
def test_sph_step_matches_reference_golden(name):
    with open(os.path.join(GOLD, f"sphstep_{name}.json")) as f:
        g = json.load(f)
    p, u = _with_velocities(getattr(ics, g["generator"])(**g["kwargs"]))
    with sim(max_particles_per_leaf=g["bucket"], max_timestep=g["dt"]) as s:
        s.set_particles(p)
        gu, gup, gvp = s.sph_run(g["steps"], u)
        got = _step_state(s, gu, gup, gvp)
    for k, want in g["samples"].items():
        scale = max(g["scale"][k], 1e-300)
        assert np.all(np.abs(got[k][g["idx"]] - np.asarray(want)) <= 1e-12 * scale), k


def test_sph_step_large_one_step_properties():
    """N = 2^18 Plummer, one step from u_pred = u and v_pred = v: the velocity
    change is a dt from the pressure pass on the same state, u and u_pred
    follow the reference's PdV update, and momentum is conserved."""
    p, u = _with_velocities(ics.plummer(1 << 18, seed=3, soft=1e-3))
    dt = 1e-3
    with sim(max_particles_per_leaf=32, max_timestep=dt) as s:
        s.set_particles(p)
        _, ax, ay, az, pdv = s.sph_pressure(u)
        gu, gup, gvp = s.sph_run(1, u)
        st = s.state()
    for a, k, vpk in ((ax, "vx", 0), (ay, "vy", 1), (az, "vz", 2)):
        dv = st[k] - p[k]
        assert _close(dv, a * dt, 1e-9), k
        assert _close(gvp[vpk] - st[k], a * dt, 1e-9), k
        # sum m a = 0 to summation order; dv also carries the rounding of v + a dt
        bound = float(np.sum(p["m"] * (np.abs(a * dt) + np.abs(p[k]))))
        assert abs(float(np.sum(p["m"] * dv))) <= 1e-12 * bound
    ud = 0.5e-7 * dt
    assert _close(gu, u - pdv * ud, 1e-15) and _close(gup, u - 2 * pdv * ud, 1e-15)
    assert np.all(np.isfinite(st["x"])) and not np.allclose(st["x"], p["x"])


@pytest.mark.parametrize("n", [2, 7, 33])
def test_sph_step_tiny(n):
    """Fewer particles than neighbours: the lists hold every particle (padded
    with -1), and the steps still match the C oracle's."""
    p = ics.plummer(max(n, 2), seed=3, soft=0.05)
    p = {k: v[:n].copy() for k, v in p.items()}
    p, u = _with_velocities(p, seed=1)
    with sim(max_particles_per_leaf=16, max_timestep=0.01) as s:
        s.set_particles(p)
        gu, gup, gvp = s.sph_run(2, u)
        got = _step_state(s, gu, gup, gvp)
    q, pu, pup, pvp = O.sph_step(p, 2, 0.01, u, u, (p["vx"], p["vy"], p["vz"]))
    want = dict(q, u=pu, u_pred=pup, vpx=pvp[0], vpy=pvp[1], vpz=pvp[2])
    for k in want:
        if k in got:
            assert _close(got[k], want[k], 1e-12), k


def test_sph_single_particle_is_reported():
    """One particle: its only neighbour is itself, the ball has zero radius and
    the reference's doSPHCalc fails its isfinite(acc) assertion; here the
    pressure pass and the step return an error and the handle stays usable."""
    from paratreet_b200._lib import PtError
    p = ics.plummer(8, seed=3, soft=0.05)
    one = {k: v[:1].copy() for k, v in p.items()}
    with sim(max_particles_per_leaf=16, max_timestep=0.01) as s:
        s.set_particles(one)
        with pytest.raises(PtError, match="SPH pressure term not finite"):
            s.sph_pressure(np.ones(1))
        with pytest.raises(PtError, match="SPH pressure term not finite"):
            s.sph_run(1, np.ones(1))
        s.set_particles(p)
        d, ax, ay, az, pdv = s.sph_pressure(np.ones(8))
        assert all(np.all(np.isfinite(a)) for a in (d, ax, ay, az, pdv))

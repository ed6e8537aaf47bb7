"""The differentiation workload: loss L = 0.5 sum |x_i(T) - y_i|^2 after K
leapfrog (KDK) steps, with y = the initial positions plus N(0, 1e-3) noise,
and its gradient with respect to the initial positions and masses from the
checkpointed adjoint chain (pt_chain_grad).

Two checks, each on 64 seeded coordinates (48 positions, 16 masses):

* Full size (Hernquist N = 262,144, seed 3, a = 1, truncated at 20a, v = 0,
  eps 0.01, theta 0.6, bucket 16, K = 64 steps of dt = 0.005, a checkpoint
  every 8 steps): the FP64 chain's gradient against central finite
  differences of the FP64 chain.  The chain with FP32 interactions is
  compared with the same finite differences; its largest error is reported
  and bounded.
* Small N (Hernquist N = 2,000, K = 8): the GPU chain's FP64 gradient
  against an FP64 reference gradient that the CPU oracle computes by central
  finite differences of its own KDK chain (the C restatement's force pass,
  bit-identical to the GPU FP64 form).

How the finite differences are taken, and what they are held to:

* The loss difference is summed particle by particle, L(+h) - L(-h) =
  0.5 sum (d+ - d-) . (d+ + d-) with d = x(T) - y, so that the small
  difference is not taken between two large sums.
* The adjoint is the derivative for the interaction lists of the base
  trajectory.  A perturbed run whose lists differ at some step samples a
  different branch of the piecewise-smooth loss; such a coordinate is
  reported and left out (at most 8 of the 48 positions and 6 of the 16
  masses).  On the GPU the finite differences run the FP64 form over the
  two-phase lists (PT_FP64_LISTS: the same interactions, FP64 arithmetic,
  equal to the FP64 chain up to the order of each sum) so that every step's
  lists are compared through their order-independent digests, which also
  tell a monopole node() from a quadrupole one; the oracle compares its
  interaction counts and its count of monopole node() calls.
* Positions: h = 1e-6; the plain relative error |fd - g| / |g| is reported
  and held to 1e-6, unless the finite difference's own error estimate (next
  item) is larger, as it is where a gradient happens to be small.
* Masses: a mass moves the centres of mass of every node that holds the
  particle, and with them opening decisions of many buckets over the steps:
  at full size a step of 1e-8 (0.26% of m = 1/N) changed the lists in 15 of
  16 coordinates on B200, so the step is 1e-10 there, and 1e-6 (0.2% of
  m = 5e-4) at N = 2,000.
* The rounding of the trajectories (about 1e-16 of each of the N positions)
  is part of every loss difference, and where a gradient is small it is a
  visible part: at full size the finite difference's own error reaches
  ~1e-5 of the gradient for some positions and ~1e-2 for some masses.  So
  each mass difference, and each position difference that misses 1e-6
  relative, is also taken with h / 2 and h / 4, and |fd - g| <= 1e-6 |g| +
  3 eta is asserted with eta = max(|fd(h) - fd(h/2)|, |fd(h) - fd(h/4)|):
  the spread of the smaller steps, whose rounding error is two and four
  times that of the step h, estimates the error of fd(h); as a one-sample
  estimate of a random error it can fall short of it (on B200 one position
  of 44 missed 1e-6 |g| + eta by 1.5e-10, a fifth of the rounding error
  expected there), hence three times it.  The plain relative errors are
  reported beside it."""
import numpy as np
import pytest

from paratreet_b200 import ics

pytestmark = pytest.mark.gpu

N, K, DT, CKPT, THETA = 262144, 64, 0.005, 8, 0.6
H_POS = 1e-6


def pick_coords(rng, n, npos=48, nmass=16):
    out = [(int(rng.integers(n)), ("x", "y", "z")[int(rng.integers(3))]) for _ in range(npos)]
    out += [(int(rng.integers(n)), "m") for _ in range(nmass)]
    return out


def loss_diff(fp, fm, y):
    """L(+h) - L(-h) from the two final positions, particle by particle."""
    tot = 0.0
    for k, yk in zip(("x", "y", "z"), y):
        dp, dm = fp[k] - yk, fm[k] - yk
        tot += 0.5 * float(np.sum((dp - dm) * (dp + dm)))
    return tot


def gpu_chain(f, p, steps):
    """Final positions and, per step, a digest of every bucket's interaction
    list (sum of the per-bucket digests mod 2^64, their lengths, the bucket
    count) of the GPU chain (a handle of the two-phase FP64 form)."""
    f.set_particles(p)
    marks = []
    f.start_down()  # the first force pass, at the initial positions
    for k in range(steps + 1):
        if k:
            f.run(1)
        dig, cnt = f.list_digests("two_phase")
        marks.append((int(np.sum(dig, dtype=np.uint64)), int(cnt.sum()), int(dig.size)))
    s = f.state()
    return {k: s[k] for k in ("x", "y", "z")}, marks


def fd_one(chain, p, y, i, c, h, base):
    """Central difference of the loss in coordinate (i, c) with step h, and
    whether both perturbed runs kept the base run's lists."""
    res, same = [], True
    for sgn in (1, -1):
        q = {k: v.copy() for k, v in p.items()}
        q[c][i] += sgn * h
        fin, cnt = chain(q)
        same = same and cnt == base
        res.append(fin)
    return loss_diff(res[0], res[1], y) / (2 * h), same


def fd_check(chain, p, y, coords, g, h_mass):
    """Finite differences against the adjoint gradient g (FP64 chain).  Per
    coordinate: fd, the error estimate max |fd(h) - fd(h/k)| over k = 2, 4
    (taken for every mass and for any position whose plain relative error
    exceeds 1e-6; 0 otherwise) and whether the lists stayed those of the
    base run."""
    base = chain(p)[1]
    out = []
    for (i, c), gk in zip(coords, g):
        h = h_mass if c == "m" else H_POS
        f, same = fd_one(chain, p, y, i, c, h, base)
        eta = 0.0
        if same and (c == "m" or abs(f - gk) > 1e-6 * abs(gk)):
            for k in (2, 4):
                fk, same_k = fd_one(chain, p, y, i, c, h / k, base)
                same = same and same_k
                eta = max(eta, abs(f - fk))
        out.append((f, eta, same))
    return out


def adjoint_at(g, coords):
    return np.array([g["g" + c][i] for i, c in coords])


def assess(fd, g, coords):
    """Errors of the adjoint gradient g against the finite differences: the
    plain relative error, and the slack |fd - g| - (1e-6 |g| + 3 eta), which
    must not be positive."""
    f = np.array([r[0] for r in fd])
    eta = np.array([r[1] for r in fd])
    ok = np.array([r[2] for r in fd])
    is_m = np.array([c == "m" for _, c in coords])
    rel = np.abs(f - g) / np.abs(g)
    slack = np.abs(f - g) - (1e-6 * np.abs(g) + 3.0 * eta)

    def mx(v, sel):
        return float(v[sel].max()) if sel.any() else None

    rep = {"valid_positions": int((ok & ~is_m).sum()), "valid_masses": int((ok & is_m).sum()),
           "lists_changed": [list(coords[k]) for k in np.nonzero(~ok)[0]],
           "max_rel_positions": mx(rel, ok & ~is_m), "max_rel_masses": mx(rel, ok & is_m),
           "median_rel": float(np.median(rel[ok])) if ok.any() else None,
           "positions_over_1e-6_plain": int(((rel > 1e-6) & ok & ~is_m).sum()),
           "max_fd_error_estimate_over_g": mx(eta / np.abs(g), ok),
           "max_slack": mx(slack, ok)}
    return rep, rel, slack, ok, is_m


def test_gradient_workload_hernquist_262k():
    from paratreet_b200.gravity import GravitySimulation

    p = ics.hernquist(N, seed=3, soft=0.01)
    y = ics.perturbed_targets(p, seed=3, sigma=1e-3)
    coords = pick_coords(np.random.default_rng(64), N)
    with GravitySimulation(max_particles_per_leaf=16, theta=THETA, max_timestep=DT, precision="mixed",
                           integrator="kdk", record_lists=True) as s:
        s.set_particles(p)
        loss_m, gm = s.chain_grad(K, DT, y, ckpt_every=CKPT)
        s.set_precision("fp64")
        loss_d, gd = s.chain_grad(K, DT, y, ckpt_every=CKPT)
    ad, am = adjoint_at(gd, coords), adjoint_at(gm, coords)
    with GravitySimulation(max_particles_per_leaf=16, theta=THETA, max_timestep=DT, precision="fp64_lists",
                           integrator="kdk") as f:
        fd = fd_check(lambda q: gpu_chain(f, q, K), p, y, coords, ad, h_mass=1e-10)
    rep_d, rel_d, slack_d, ok, is_m = assess(fd, ad, coords)
    rep_m, rel_m, _, _, _ = assess(fd, am, coords)
    print("gradient workload:", {"fp64_chain_vs_fd": rep_d, "fp32_interaction_chain_vs_fd_of_fp64_chain": rep_m,
                                 "loss": {"fp64": loss_d, "mixed": loss_m}})
    assert abs(loss_m - loss_d) / loss_d < 1e-4
    assert rep_d["valid_positions"] >= 40 and rep_d["valid_masses"] >= 10, rep_d["lists_changed"]
    assert slack_d[ok].max() <= 0.0, rep_d
    # the FP32-interaction chain differentiates a slightly different trajectory
    # (forces within ~1e-7 of FP64 per step); its gradient is held to 1e-3
    # relative, with the same allowance for the finite differences' own error
    f = np.array([r[0] for r in fd])
    eta = np.array([r[1] for r in fd])
    assert (np.abs(f - am) - (1e-3 * np.abs(am) + 3.0 * eta))[ok].max() <= 0.0, rep_m


def oracle_chain(q, steps, dt, theta, bucket):
    """The oracle's KDK chain: v += a dt/2; x += v dt; a = a(x); v += a dt/2,
    each force pass by the C restatement (a fresh tree every step).  Final
    positions and the P2P, P2C and monopole node() counts of every force
    pass."""
    from oracle import oracle as O

    x = [q["x"].copy(), q["y"].copy(), q["z"].copy()]
    v = [q["vx"].copy(), q["vy"].copy(), q["vz"].copy()]
    counts = []

    def acc(xs):
        r = dict(q, x=xs[0], y=xs[1], z=xs[2])
        sim = O.PortSim(r, bucket=bucket, theta=theta, dt_max=dt)
        sim.forces()
        a = sim.acc()[:3]
        c = sim.counters()
        counts.append((c["n_pp"], c["n_pc"], sim.mono_count()))
        sim.close()
        return a

    a = acc(x)
    for _ in range(steps):
        for k in range(3):
            v[k] = v[k] + (0.5 * dt) * a[k]
            x[k] = x[k] + dt * v[k]
        a = acc(x)
        for k in range(3):
            v[k] = v[k] + (0.5 * dt) * a[k]
    return dict(zip(("x", "y", "z"), x)), counts


def test_chain_gradient_against_oracle_fd_small_n():
    from paratreet_b200.gravity import GravitySimulation

    n, steps, bucket = 2000, 8, 16
    p = ics.hernquist(n, seed=3, soft=0.01)
    y = ics.perturbed_targets(p, seed=3, sigma=1e-3)
    coords = pick_coords(np.random.default_rng(65), n)
    with GravitySimulation(max_particles_per_leaf=bucket, theta=THETA, max_timestep=DT, precision="fp64",
                           integrator="kdk", record_lists=True) as s:
        s.set_particles(p)
        _, gd = s.chain_grad(steps, DT, y, ckpt_every=3)
        s.set_precision("mixed")
        _, gm = s.chain_grad(steps, DT, y, ckpt_every=3)
    ad, am = adjoint_at(gd, coords), adjoint_at(gm, coords)
    ref = fd_check(lambda q: oracle_chain(q, steps, DT, THETA, bucket), p, y, coords, ad, h_mass=1e-6)
    rep_d, rel_d, slack_d, ok, is_m = assess(ref, ad, coords)
    rep_m, rel_m, _, _, _ = assess(ref, am, coords)
    print("oracle FD gradient, N=2000 K=8:", {"fp64_chain": rep_d, "fp32_interaction_chain": rep_m})
    assert rep_d["valid_positions"] >= 40 and rep_d["valid_masses"] >= 10, rep_d["lists_changed"]
    assert slack_d[ok].max() <= 0.0, rep_d
    assert rel_m[ok & ~is_m].max() <= 1e-3, rep_m

"""GPU tests of the adjoint force pass and the checkpointed K-step chain.

The adjoint is the exact derivative of the force pass for a FIXED interaction
list, so it is checked against central finite differences of the frozen-list
FP64 replay (pt_forces_frozen), which keeps the tree and the lists while the
moments follow the perturbed positions / masses.  A torch.autograd.Function
(defined here, in the tests only) wraps forward = force pass and backward =
pt_adjoint.
"""
import numpy as np
import pytest

from paratreet_b200 import ics

pytestmark = pytest.mark.gpu


def sim(**kw):
    from paratreet_b200.gravity import GravitySimulation
    return GravitySimulation(**kw)


def frozen_objective(s, p, cot, **changes):
    q = {k: p[k].copy() for k in ("x", "y", "z", "m")}
    q.update(changes)
    a = s.forces_frozen(q["x"], q["y"], q["z"], q["m"])
    return float(np.sum(cot[0] * a["ax"]) + np.sum(cot[1] * a["ay"]) + np.sum(cot[2] * a["az"]))


def test_frozen_replay_reproduces_the_pass():
    p = ics.plummer(8000, seed=5, soft=0.01)
    with sim(max_particles_per_leaf=16, record_lists=True) as s:
        s.set_particles(p)
        s.start_down()
        a0 = s.accelerations()
        a1 = s.forces_frozen(p["x"], p["y"], p["z"], p["m"])
    for k in ("ax", "ay", "az", "pot", "pot_full"):
        assert np.array_equal(a0[k], a1[k]), k


@pytest.mark.parametrize("gen,n,bucket,soft", [("plummer", 3000, 16, 0.01), ("hernquist", 2500, 8, 0.05)])
def test_adjoint_matches_finite_differences(gen, n, bucket, soft):
    p = getattr(ics, gen)(n, soft=soft)
    rng = np.random.default_rng(17)
    cot = rng.normal(size=(3, n))
    with sim(max_particles_per_leaf=bucket, record_lists=True) as s:
        s.set_particles(p)
        s.start_down()
        g = s.adjoint(*cot)
        errs = []
        for _ in range(24):
            i = int(rng.integers(n))
            comp = ("x", "y", "z")[int(rng.integers(3))]
            h = 1e-5 * max(1.0, abs(p[comp][i]))
            xp, xm = p[comp].copy(), p[comp].copy()
            xp[i] += h
            xm[i] -= h
            fd = (frozen_objective(s, p, cot, **{comp: xp}) - frozen_objective(s, p, cot, **{comp: xm})) / (2 * h)
            an = g["g" + comp][i]
            errs.append(abs(fd - an) / max(abs(an), 1e-3 * np.abs(g["g" + comp]).max()))
        for _ in range(8):
            i = int(rng.integers(n))
            h = 1e-4 * p["m"][i]
            mp, mm = p["m"].copy(), p["m"].copy()
            mp[i] += h
            mm[i] -= h
            fd = (frozen_objective(s, p, cot, m=mp) - frozen_objective(s, p, cot, m=mm)) / (2 * h)
            errs.append(abs(fd - g["gm"][i]) / max(abs(g["gm"][i]), 1e-3 * np.abs(g["gm"]).max()))
    print("adjoint vs FD: max rel err %.3e" % max(errs))
    assert max(errs) < 1e-5, errs


def test_autograd_function_wrapper():
    torch = pytest.importorskip("torch")

    class Forces(torch.autograd.Function):
        """forward: positions (3, N), masses (N) -> accelerations (3, N) via the
        GPU force pass (lists recorded); backward: pt_adjoint."""

        @staticmethod
        def forward(ctx, pos, mass, s, base):
            q = dict(base)
            q["x"], q["y"], q["z"] = (pos[k].detach().cpu().numpy().astype(np.float64) for k in range(3))
            q["m"] = mass.detach().cpu().numpy().astype(np.float64)
            s.set_particles(q)
            s.start_down()
            a = s.accelerations()
            ctx.s = s
            return torch.tensor(np.stack([a["ax"], a["ay"], a["az"]]), dtype=torch.float64)

        @staticmethod
        def backward(ctx, grad):
            g = ctx.s.adjoint(*grad.detach().cpu().numpy())
            gpos = torch.tensor(np.stack([g["gx"], g["gy"], g["gz"]]), dtype=torch.float64)
            return gpos, torch.tensor(g["gm"]), None, None

    p = ics.plummer(2000, seed=8, soft=0.02)
    pos = torch.tensor(np.stack([p["x"], p["y"], p["z"]]), requires_grad=True)
    mass = torch.tensor(p["m"], requires_grad=True)
    w = torch.tensor(np.random.default_rng(3).normal(size=(3, 2000)))
    with sim(max_particles_per_leaf=16, record_lists=True) as s:
        acc = Forces.apply(pos, mass, s, p)
        (acc * w).sum().backward()
        g = pos.grad.numpy()
        # the same gradient from the C ABI directly
        ref = s.adjoint(*w.numpy())
    # the adjoint adds source terms with FP64 atomics: equal up to summation
    # order, so entries that cancel are compared against the array's scale
    for got, want in ((g[0], ref["gx"]), (g[1], ref["gy"]), (g[2], ref["gz"]), (mass.grad.numpy(), ref["gm"])):
        assert np.allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


def test_chain_gradient_matches_finite_differences():
    """K-step leapfrog with checkpoints; FD of the full chain (the lists are
    re-walked every step, so a perturbation small enough not to flip any
    opening decision is used)."""
    n, K, dt = 1536, 12, 0.005
    p = ics.hernquist(n, seed=3, soft=0.02)
    rng = np.random.default_rng(5)
    y = [p[k] + rng.normal(0.0, 1e-3, n) for k in ("x", "y", "z")]
    with sim(max_particles_per_leaf=16, theta=0.6, max_timestep=1.0) as s:
        s.set_particles(p)
        loss, g = s.chain_grad(K, dt, y, ckpt_every=4)
        g2 = s.chain_grad(K, dt, y, ckpt_every=12)[1]  # no recomputation
        assert np.allclose(g["gx"], g2["gx"], rtol=1e-12, atol=1e-15)
        errs = []
        for _ in range(12):
            i = int(rng.integers(n))
            comp = ("x", "y", "z")[int(rng.integers(3))]
            h = 1e-6
            vals = []
            for sgn in (1, -1):
                q = {k: v.copy() for k, v in p.items()}
                q[comp][i] += sgn * h
                s.set_particles(q)
                vals.append(s.chain_grad(K, dt, y, ckpt_every=K)[0])
            fd = (vals[0] - vals[1]) / (2 * h)
            an = g["g" + comp][i]
            errs.append(abs(fd - an) / max(abs(an), 1e-2 * np.abs(g["g" + comp]).max()))
    print("chain gradient vs FD: median %.3e max %.3e" % (np.median(errs), max(errs)))
    assert np.median(errs) < 1e-5, errs

"""The periodic workload at full size: N = 256^3 = 16,777,216 particles on a
lattice in a unit box displaced by a Gaussian field with P(k) ~ k^-2 (rms 0.25
cell, seed 11, cut at Nyquist), equal masses, eps = 0.5/256, theta 0.7,
bucket 32, quadrupole moments, one replica shell walked by the tree and the
Ewald correction with |h|^2 <= 10; one force evaluation and one KDK step with
dt = 1e-3.  Errors of the mixed and the FP64 tree against the FP64 Ewald
direct sum on 2048 seeded targets.  PT_PERIODIC_NGRID shrinks the lattice for
a quick run.

The net force on a displaced lattice is a small residual (rms |a| ~ 0.011
G M / L^2 here) and shrinks as 1 / ngrid, while the tree's absolute error at a
given theta does not (about 8e-3 G M / L^2 at theta 0.7 for 16^3 to 64^3 in the
C oracle), so the per-particle relative error of the reference method is of
order one at this size.  The error is therefore also stated relative to the
rms force, |da| / rms|a| (rms and p99), at theta 0.7 and at theta 0.4, where
it falls by a factor of seven."""
import json
import os
import time

import numpy as np
import pytest

from paratreet_b200 import ics

pytestmark = pytest.mark.gpu

NGRID = int(os.environ.get("PT_PERIODIC_NGRID", "256"))
HCUT = 10 ** 0.5


def err_stats(a, d, tg):
    """Per-particle relative error |da| / |a| and the error relative to the
    rms force, |da| / rms|a| (rms and p99 of each)."""
    diff = np.sqrt(sum((a[k][tg] - d[i]) ** 2 for i, k in enumerate(("ax", "ay", "az"))))
    mag = np.sqrt(sum(d[i] ** 2 for i in range(3)))
    e = diff / mag
    frms = float(np.sqrt(np.mean(mag * mag)))
    return {"rms": float(np.sqrt(np.mean(e * e))), "p99": float(np.percentile(e, 99)), "max": float(e.max()),
            "abs_rms": float(np.sqrt(np.mean(diff * diff))), "force_rms": frms,
            "abs_rms_over_force_rms": float(np.sqrt(np.mean(diff * diff))) / frms,
            "abs_p99_over_force_rms": float(np.percentile(diff, 99)) / frms}


def test_periodic_lattice_workload():
    from paratreet_b200.gravity import GravitySimulation

    p = ics.lattice(NGRID, seed=11, rms_cells=0.25, soft_cells=0.5)
    n = p["x"].size
    tg = np.sort(np.random.default_rng(2048).choice(n, 2048, replace=False)).astype(np.int32)
    report = {"workload": "lattice%d^3 periodic" % NGRID, "n": n}
    acc = {}
    d = None
    for theta in (0.7, 0.4):
        for prec in ("fp64", "mixed"):
            with GravitySimulation(max_particles_per_leaf=32, theta=theta, max_timestep=1e-3, precision=prec,
                                   integrator="kdk", periodic=True, n_replicas=1, period=1.0,
                                   ewald_hcut=HCUT) as s:
                s.set_particles(p)
                s.start_down()
                s.start_down()  # second pass timed (first one sizes the buffers)
                acc[theta, prec] = s.accelerations()
                c = s.counters()
                report[f"{prec}_theta{theta}"] = {"ms_total": c["ms_total"], "ms_traverse": c["ms_traverse"],
                                                  "n_pp": c["n_pp"], "n_pc": c["n_pc"]}
                if prec == "mixed" and d is None:
                    t0 = time.perf_counter()
                    d = s.ewald_direct_sum(tg)
                    report["yardstick_s"] = time.perf_counter() - t0
                    s.run(1)  # one KDK step
                    st = s.state()
                    report["kdk_dt"] = s.last_dt()
                    assert all(np.all(np.isfinite(st[k])) for k in st)
    for (theta, prec), a in acc.items():
        report[f"{prec}_theta{theta}"]["vs_ewald_direct"] = err_stats(a, d, tg)
    for theta in (0.7, 0.4):
        m, f = acc[theta, "mixed"], acc[theta, "fp64"]
        dm = np.sqrt(sum((m[k] - f[k]) ** 2 for k in ("ax", "ay", "az")))
        mf = np.sqrt(sum(f[k] ** 2 for k in ("ax", "ay", "az")))
        report[f"mixed_vs_fp64_rms_theta{theta}"] = float(np.sqrt(np.mean((dm / mf) ** 2)))
    print("periodic workload:", json.dumps(report))
    e = {k: report[k]["vs_ewald_direct"] for k in report if k.startswith(("fp64_theta", "mixed_theta"))}
    for theta in (0.7, 0.4):
        assert report[f"mixed_vs_fp64_rms_theta{theta}"] < 1e-3
        # both forms carry the reference method's error, not one of their own
        assert abs(e[f"mixed_theta{theta}"]["abs_rms"] - e[f"fp64_theta{theta}"]["abs_rms"]) < \
            0.01 * e[f"fp64_theta{theta}"]["abs_rms"]
    for prec in ("fp64", "mixed"):
        # the error relative to the rms force falls with theta at this size
        assert e[f"{prec}_theta0.4"]["abs_rms_over_force_rms"] < 0.5 * e[f"{prec}_theta0.7"]["abs_rms_over_force_rms"]
    if NGRID == 256:
        # measured on B200 (both forms): |da| / rms|a| rms 0.714 (p99 1.38) at
        # theta 0.7 and 0.101 (p99 0.198) at theta 0.4; held within a tenth
        for prec in ("fp64", "mixed"):
            assert e[f"{prec}_theta0.7"]["abs_rms_over_force_rms"] < 0.79
            assert e[f"{prec}_theta0.4"]["abs_rms_over_force_rms"] < 0.111
            assert e[f"{prec}_theta0.4"]["abs_p99_over_force_rms"] < 0.22

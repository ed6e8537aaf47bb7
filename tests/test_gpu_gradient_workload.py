"""The differentiation workload at full size: Hernquist halo N = 262,144
(seed 3, a = 1, truncated at 20a, v = 0, eps 0.01, theta 0.6), loss
L = 0.5 sum |x_i(T) - y_i|^2 after K = 64 leapfrog steps of dt = 0.005, with
y = the same initial positions plus N(0, 1e-3) noise; gradient with respect
to the initial positions (checkpoints every 8 steps) against central finite
differences (h = 1e-6) of the FP64 chain on PT_GRAD_COORDS random coordinates
(default 16; 64 for the full check).  Also reports the cost of one adjoint pass
relative to one force pass."""
import os
import time

import numpy as np
import pytest

from paratreet_b200 import ics

pytestmark = pytest.mark.gpu

N, K, DT, CKPT, THETA = 262144, 64, 0.005, 8, 0.6


def test_gradient_workload_hernquist_262k():
    from paratreet_b200.gravity import GravitySimulation

    coords = int(os.environ.get("PT_GRAD_COORDS", "16"))
    p = ics.hernquist(N, seed=3, soft=0.01)
    y = ics.perturbed_targets(p, seed=3, sigma=1e-3)
    rng = np.random.default_rng(64)
    report = {}
    with GravitySimulation(max_particles_per_leaf=16, theta=THETA, max_timestep=DT, precision="mixed",
                           integrator="kdk", record_lists=True) as s:
        s.set_particles(p)
        # cost of one adjoint pass vs one force pass (mixed forward, FP64 adjoint)
        s.start_down()
        t0 = time.perf_counter()
        for _ in range(3):
            s.start_down()
        t_fwd_lists = (time.perf_counter() - t0) / 3
        c = s.counters()
        cot = rng.normal(size=(3, N))
        s.adjoint(*cot)
        t0 = time.perf_counter()
        for _ in range(3):
            s.adjoint(*cot)
        t_adj = (time.perf_counter() - t0) / 3
        report["forward_ms_traverse_mixed"] = c["ms_traverse"]
        report["forward_pass_with_lists_s"] = t_fwd_lists
        report["adjoint_pass_s"] = t_adj
        # gradient of the chain with mixed-precision forces
        t0 = time.perf_counter()
        loss_m, gm = s.chain_grad(K, DT, y, ckpt_every=CKPT)
        report["chain_grad_mixed_s"] = time.perf_counter() - t0
        s.set_precision("fp64")
        t0 = time.perf_counter()
        loss_d, gd = s.chain_grad(K, DT, y, ckpt_every=CKPT)
        report["chain_grad_fp64_s"] = time.perf_counter() - t0
    report["loss_mixed"], report["loss_fp64"] = loss_m, loss_d

    errs_d, errs_m = [], []
    with GravitySimulation(max_particles_per_leaf=16, theta=THETA, max_timestep=DT, precision="fp64",
                           integrator="kdk") as f:
        for _ in range(coords):
            i = int(rng.integers(N))
            comp = ("x", "y", "z")[int(rng.integers(3))]
            vals = []
            for sgn in (1, -1):
                q = {k: v.copy() for k, v in p.items()}
                q[comp][i] += sgn * 1e-6
                f.set_particles(q)
                f.run(K)
                st = f.state()
                vals.append(0.5 * sum(np.sum((st[k] - yk) ** 2) for k, yk in zip(("x", "y", "z"), y)))
            fd = (vals[0] - vals[1]) / 2e-6
            scale = 1e-2 * np.abs(gd["g" + comp]).max()
            errs_d.append(abs(fd - gd["g" + comp][i]) / max(abs(gd["g" + comp][i]), scale))
            errs_m.append(abs(fd - gm["g" + comp][i]) / max(abs(gm["g" + comp][i]), scale))
    report["fd_coords"] = coords
    report["fp64_grad_vs_fd"] = {"median": float(np.median(errs_d)), "max": float(np.max(errs_d))}
    report["mixed_grad_vs_fd"] = {"median": float(np.median(errs_m)), "max": float(np.max(errs_m))}
    print("gradient workload:", report)
    assert abs(loss_m - loss_d) / loss_d < 1e-4
    assert np.median(errs_d) < 1e-5
    assert np.median(errs_m) < 1e-3

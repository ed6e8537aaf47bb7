"""Generate the committed golden fixtures under tests/golden/.

Run in a container where the reference tree is mounted and the
reference-sources oracle (oracle/_ref/libptref.so, ``make -C oracle``) is
built:

    python tests/golden/make_golden.py [--reference PATH]

PATH defaults to $PT_REFERENCE, else <repo>/../reference.

Outputs
-------
lambs_kat.npz
    The reference's own force-accuracy fixture (tests/gravity/
    lambs.00200_subsamp_30K, big-endian Tipsy, 30000 dark particles, eps
    2.5e-4) as FP32 positions, plus the accelerations that the reference's
    tests/gravity/direct.acc holds for 2000 seeded target particles.  It is
    the known-answer test of the FP64 spline direct sum.
ref_<case>.json
    SHA-256 digests (and a few sample values) of every output of the
    reference's own gravity sources, compiled where they lie, on a seeded
    workload: particle keys, the node dump (canonical key order), the
    per-bucket interaction lists, accelerations, partial potentials, and the
    state after the configured number of kick/perturb steps.  The C oracle
    and the CUDA path must reproduce these bit for bit.
basic_<case>.json
    The reference's gravity sources under the basic down traversal
    (Partition::startBasicDown: breadth first per bucket): digests of the
    accelerations, partial potentials and interaction lists.
sph_<case>.json
    The reference's SPH density pass (examples/DensityVisitor.h with a
    restated up-and-down walk, DensityFn of examples/SPH.C, kernelM4 of
    examples/SPHUtils.h): digests of every particle's 32 neighbours (sorted
    by distance, then index), their d2 and the ball radii, and sampled
    densities (which depend on the heap's summation order in the last bits).
    Then the pressure pass (PressureVisitor walk, ForceFn of examples/SPH.C,
    doSPHCalc of examples/SPHUtils.h, the opposing effects added after it)
    for seeded internal energies u: sampled pressure accelerations and PdV
    work, and their L1 norms (summation order again decides the last bits).
sphstep_<case>.json
    Iterations of the reference's SPH example (the density and pressure
    passes above, then the reference's own Particle::kick and
    Particle::perturb of src/Particle.C with dt = max_timestep) from seeded
    velocities and internal energies: sampled positions, velocities,
    predicted velocities, u and u_predicted after the last step, with their
    scales (the pressure pass's summation order decides the last bits).
periodic_<case>.json
    The same sources in periodic mode (examples/Gravity.C replica walks plus
    the Ewald correction of examples/Ewald.{h,C}) on a displaced lattice:
    digests and samples of the accelerations and partial potentials.  The C
    oracle reproduces them bit for bit (same host libm); the CUDA path is
    compared with the C oracle within a tolerance, since the Ewald sums call
    CUDA's erf/erfc/exp/sincos.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import struct
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from paratreet_b200 import ics  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# name -> (generator, kwargs, bucket, theta, dt_max, steps)
CASES = {
    "plummer_10k": (ics.plummer, dict(n=10000, seed=42, soft=0.01), 16, 0.7, 0.01, 1),
    "mixture_16k": (ics.mixture, dict(n=16384, seed=7, soft=1e-4), 16, 0.7, 1e-4, 3),
    "plummer_4k_b32_t05": (ics.plummer, dict(n=4096, seed=5, soft=1e-3), 32, 0.5, 0.01, 1),
    "hernquist_8k_t10": (ics.hernquist, dict(n=8192, seed=3, soft=0.01), 32, 1.0, 0.005, 2),
}

# name -> (generator, kwargs, bucket, theta)
BASIC_CASES = {
    "plummer_4k": (ics.plummer, dict(n=4096, seed=11, soft=0.01), 16, 0.7),
    "hernquist_6k_t05": (ics.hernquist, dict(n=6000, seed=4, soft=0.01), 8, 0.5),
}

# name -> (generator, kwargs, bucket)
SPH_CASES = {
    "plummer_4k": (ics.plummer, dict(n=4096, seed=9, soft=0.01), 16),
    "mixture_8k": (ics.mixture, dict(n=8192, seed=2, soft=1e-4), 32),
}

# name -> (generator, kwargs, bucket, dt, steps)
SPH_STEP_CASES = {
    "plummer_3k": (ics.plummer, dict(n=3000, seed=4, soft=0.01), 16, 0.01, 3),
}

# name -> (lattice kwargs, bucket, theta, n_replicas)
PERIODIC_CASES = {
    "lattice_16_b32_r1": (dict(ngrid=16, seed=11, rms_cells=0.25, soft_cells=0.5), 32, 0.7, 1),
    "lattice_12_b16_t05_r2": (dict(ngrid=12, seed=5, rms_cells=0.4, soft_cells=0.3), 16, 0.5, 2),
}


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_case(name):
    gen, kw, bucket, theta, dt_max, steps = CASES[name]
    p = gen(**kw)
    r = O.RefSim(p, bucket=bucket, theta=theta, dt_max=dt_max, threads=1)
    r.forces(record_lists=True)
    ax, ay, az, pot = r.acc()
    tree = O.sort_tree(r.tree())
    lists = r.lists()
    cnt = r.counters()
    out = {
        "case": name,
        "generator": gen.__name__,
        "kwargs": kw,
        "bucket": bucket,
        "theta": theta,
        "dt_max": dt_max,
        "steps": steps,
        "n_nodes": int(tree.keys.size),
        "n_buckets": int(lists.bucket_keys.size),
        "n_pp": cnt["n_pp"],
        "n_pc": cnt["n_pc"],
        "sha256": {
            "keys": digest(r.keys()),
            "node_keys": digest(tree.keys),
            "node_types": digest(tree.types.astype(np.int32)),
            "node_counts": digest(tree.count.astype(np.int32)),
            "node_moments": digest(tree.moments),
            "bucket_keys": digest(lists.bucket_keys),
            "list_offsets": digest(lists.offsets.astype(np.int64)),
            "list_keys": digest(lists.keys),
            "list_kinds": digest(lists.kinds.astype(np.int32)),
            "ax": digest(ax), "ay": digest(ay), "az": digest(az), "pot": digest(pot),
        },
        "samples": {
            "idx": [0, 1, 2, int(p["x"].size // 2), int(p["x"].size - 1)],
        },
    }
    idx = out["samples"]["idx"]
    out["samples"]["ax"] = [float(ax[i]) for i in idx]
    out["samples"]["pot"] = [float(pot[i]) for i in idx]
    r.close()
    r = O.RefSim(p, bucket=bucket, theta=theta, dt_max=dt_max, threads=1)
    r.run(steps)
    st = r.state()
    a2 = r.acc()
    out["after_steps"] = {
        "last_dt": r.counters()["last_dt"],
        "sha256": {k: digest(v) for k, v in zip(("x", "y", "z", "vx", "vy", "vz"), st)},
        "acc_sha256": {k: digest(v) for k, v in zip(("ax", "ay", "az", "pot"), a2)},
    }
    with open(os.path.join(OUT, f"ref_{name}.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(name, out["n_nodes"], out["n_buckets"], out["n_pp"], out["n_pc"])


def run_periodic_case(name):
    kw, bucket, theta, nrep = PERIODIC_CASES[name]
    p = ics.lattice(**kw)
    r = O.RefSim(p, bucket=bucket, theta=theta, threads=1)
    r.set_periodic(1.0, nrep)
    r.forces()
    ax, ay, az, pot = r.acc()
    idx = [0, 1, 2, int(p["x"].size // 2), int(p["x"].size - 1)]
    out = {
        "case": name, "kwargs": kw, "bucket": bucket, "theta": theta, "n_replicas": nrep, "period": 1.0,
        "sha256": {"ax": digest(ax), "ay": digest(ay), "az": digest(az), "pot": digest(pot)},
        "samples": {"idx": idx, "ax": [float(ax[i]) for i in idx], "pot": [float(pot[i]) for i in idx]},
    }
    with open(os.path.join(OUT, f"periodic_{name}.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(name, p["x"].size)


def run_basic_case(name):
    gen, kw, bucket, theta = BASIC_CASES[name]
    p = gen(**kw)
    r = O.RefSim(p, bucket=bucket, theta=theta, threads=1)
    r.set_basic_down()
    r.forces(record_lists=True)
    ax, ay, az, pot = r.acc()
    lists = r.lists()
    out = {
        "case": name, "generator": gen.__name__, "kwargs": kw, "bucket": bucket, "theta": theta,
        "sha256": {"ax": digest(ax), "ay": digest(ay), "az": digest(az), "pot": digest(pot),
                   "list_offsets": digest(lists.offsets.astype(np.int64)), "list_keys": digest(lists.keys),
                   "list_kinds": digest(lists.kinds.astype(np.int32))},
    }
    with open(os.path.join(OUT, f"basic_{name}.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(name, p["x"].size)


def sph_energies(n):
    """The internal energies of the pressure goldens."""
    return np.random.default_rng(17).uniform(0.5, 1.5, n)


def run_sph_case(name):
    gen, kw, bucket = SPH_CASES[name]
    p = gen(**kw)
    r = O.RefSim(p, bucket=bucket, threads=1)
    dens, ball, nbr, nd2 = r.sph_density()
    idx = [0, 1, 2, int(p["x"].size // 2), int(p["x"].size - 1)]
    out = {
        "case": name, "generator": gen.__name__, "kwargs": kw, "bucket": bucket,
        "sha256": {"nbr": digest(nbr.astype(np.int32)), "nbr_d2": digest(nd2), "ball_sq": digest(ball)},
        "samples": {"idx": idx, "density": [float(dens[i]) for i in idx]},
    }
    n = p["x"].size
    u = sph_energies(n)
    ax, ay, az, pdv = r.sph_pressure(u)
    pidx = sorted(set(idx) | set(int(i) for i in np.random.default_rng(3).choice(n, 27, replace=False)))
    out["pressure"] = {
        "u": "numpy default_rng(17).uniform(0.5, 1.5, n)", "idx": pidx,
        "ax": [float(ax[i]) for i in pidx], "ay": [float(ay[i]) for i in pidx],
        "az": [float(az[i]) for i in pidx], "pdv": [float(pdv[i]) for i in pidx],
        "l1": {k: float(np.abs(v).sum()) for k, v in (("ax", ax), ("ay", ay), ("az", az), ("pdv", pdv))},
        "acc_scale": float(max(np.abs(ax).max(), np.abs(ay).max(), np.abs(az).max())),
        "pdv_scale": float(np.abs(pdv).max()),
    }
    with open(os.path.join(OUT, f"sph_{name}.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(name, p["x"].size)


def sph_step_inputs(p):
    """Seeded velocities (the generator's plus N(0, 0.3)) and internal
    energies of the SPH step goldens."""
    n = p["x"].size
    rng = np.random.default_rng(8)
    q = dict(p)
    for k in ("vx", "vy", "vz"):
        q[k] = p[k] + rng.normal(0.0, 0.3, n)
    return q, rng.uniform(0.2, 2.0, n)


def run_sph_step_case(name):
    gen, kw, bucket, dt, steps = SPH_STEP_CASES[name]
    p, u = sph_step_inputs(gen(**kw))
    n = p["x"].size
    r = O.RefSim(p, bucket=bucket, dt_max=dt, threads=1)
    ru, rup, rvp = r.sph_step(steps, u, u.copy(), (p["vx"], p["vy"], p["vz"]))
    x, y, z, vx, vy, vz = r.state()
    idx = sorted(int(i) for i in np.random.default_rng(5).choice(n, 32, replace=False))
    arrs = {"x": x, "y": y, "z": z, "vx": vx, "vy": vy, "vz": vz, "u": ru, "u_pred": rup,
            "vpx": rvp[0], "vpy": rvp[1], "vpz": rvp[2]}
    out = {
        "case": name, "generator": gen.__name__, "kwargs": kw, "bucket": bucket, "dt": dt, "steps": steps,
        "inputs": "velocities + numpy default_rng(8).normal(0, 0.3, n) per axis, then u = "
                  "default_rng(8).uniform(0.2, 2.0, n) from the same generator; u_pred = u, v_pred = v",
        "idx": idx,
        "samples": {k: [float(v[i]) for i in idx] for k, v in arrs.items()},
        "scale": {k: float(np.abs(v).max()) for k, v in arrs.items()},
    }
    with open(os.path.join(OUT, f"sphstep_{name}.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(name, n)


def read_tipsy_dark(path):
    with open(path, "rb") as f:
        buf = f.read()
    t, n, ndim, nsph, ndark, nstar = struct.unpack(">diiiii", buf[:28])
    assert nsph == 0 and nstar == 0 and n == ndark
    d = np.frombuffer(buf[32:32 + 36 * ndark], dtype=">f4").reshape(ndark, 9)
    return d


def read_acc(path):
    v = np.loadtxt(path)
    n = int(v[0])
    a = v[1:].reshape(3, n)
    return a


def make_kat(reference):
    g = os.path.join(reference, "tests", "gravity")
    d = read_tipsy_dark(os.path.join(g, "lambs.00200_subsamp_30K"))
    acc = read_acc(os.path.join(g, "direct.acc"))
    n = d.shape[0]
    rng = np.random.default_rng(2024)
    tgt = np.sort(rng.choice(n, 2000, replace=False)).astype(np.int32)
    np.savez_compressed(
        os.path.join(OUT, "lambs_kat.npz"),
        pos=d[:, 1:4].astype(np.float32),
        mass=d[:, 0].astype(np.float32),
        eps=d[:, 7].astype(np.float32),
        targets=tgt,
        acc=acc[:, tgt].T.copy(),
    )
    print("kat", n, tgt.size)


def main():
    ap = argparse.ArgumentParser()
    repo = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    ap.add_argument("--reference", default=os.environ.get("PT_REFERENCE", os.path.join(os.path.dirname(repo),
                                                                                       "reference")))
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    ap.add_argument("--periodic-cases", nargs="*", default=list(PERIODIC_CASES))
    ap.add_argument("--sph-cases", nargs="*", default=list(SPH_CASES))
    ap.add_argument("--basic-cases", nargs="*", default=list(BASIC_CASES))
    ap.add_argument("--sph-step-cases", nargs="*", default=list(SPH_STEP_CASES))
    ap.add_argument("--only-sph-step", action="store_true", help="write only the sphstep_ fixtures")
    a = ap.parse_args()
    if not O.ref_available():
        sys.exit("oracle/_ref/libptref.so is missing: run `make -C oracle` with the reference mounted")
    for c in a.sph_step_cases:
        run_sph_step_case(c)
    if a.only_sph_step:
        return
    make_kat(a.reference)
    for c in a.cases:
        run_case(c)
    for c in a.periodic_cases:
        run_periodic_case(c)
    for c in a.sph_cases:
        run_sph_case(c)
    for c in a.basic_cases:
        run_basic_case(c)


if __name__ == "__main__":
    main()

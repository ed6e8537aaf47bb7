"""Force errors of both forms against the FP64 direct sum on the workloads
other than the 2^24 Plummer sphere (which bench.py reports):

  plummer_10k     Plummer N = 10,000, seed 42, eps 0.01, bucket 16, theta 0.7
  mixture_1m      50% uniform cube + 50% in 32 Plummer clumps (a = 0.01),
                  N = 2^20, seed 7, eps 1e-4, bucket 16, theta 0.7
  hernquist_262k  Hernquist N = 262,144, seed 3, eps 0.01, bucket 16, theta 0.6

On 4096 seeded targets (seed 43, as the bench): RMS, 99th percentile and
maximum of |a - a_direct| / |a_direct| for the FP64 tree (the reference's
arithmetic) and the mixed form, and the mixed form's difference from the FP64
tree over all particles.  The tree's own approximation error is the
reference method's; the mixed form must add at most 1e-5 RMS to it."""
import json

import numpy as np
import pytest

from paratreet_b200 import ics

pytestmark = pytest.mark.gpu

CONFIGS = {
    "plummer_10k": (lambda: ics.plummer(10000, seed=42, soft=0.01), 16, 0.7),
    "mixture_1m": (lambda: ics.mixture(1 << 20, seed=7, soft=1e-4), 16, 0.7),
    "hernquist_262k": (lambda: ics.hernquist(262144, seed=3, soft=0.01), 16, 0.6),
}


def rel_errors(a, ref):
    num = np.sqrt(sum((a[k] - ref[i]) ** 2 for i, k in enumerate(("ax", "ay", "az"))))
    den = np.sqrt(sum(ref[i] ** 2 for i in range(3)))
    e = num / den
    return {"rms": float(np.sqrt(np.mean(e * e))), "p99": float(np.percentile(e, 99)), "max": float(e.max())}


@pytest.mark.parametrize("name", list(CONFIGS))
def test_force_errors_vs_direct_sum(name):
    from paratreet_b200.gravity import GravitySimulation

    make, bucket, theta = CONFIGS[name]
    p = make()
    n = p["x"].size
    tgt = np.sort(np.random.default_rng(43).choice(n, size=min(4096, n), replace=False)).astype(np.int32)
    acc, report = {}, {"config": name, "n": n, "theta": theta, "bucket": bucket, "targets": int(tgt.size)}
    direct = None
    for prec in ("fp64", "mixed"):
        with GravitySimulation(max_particles_per_leaf=bucket, theta=theta, precision=prec) as s:
            s.set_particles(p)
            s.start_down()
            acc[prec] = s.accelerations()
            if direct is None:
                direct = s.direct_sum(tgt)[:3]
    for prec in ("fp64", "mixed"):
        report[prec] = rel_errors({k: acc[prec][k][tgt] for k in ("ax", "ay", "az")}, direct)
    report["mixed_vs_fp64_tree"] = rel_errors(acc["mixed"], [acc["fp64"][k] for k in ("ax", "ay", "az")])
    print("force errors:", json.dumps(report))
    assert report["mixed_vs_fp64_tree"]["rms"] < 1e-5
    assert abs(report["mixed"]["rms"] - report["fp64"]["rms"]) <= 1e-5 + 1e-3 * report["fp64"]["rms"]
    # a sanity bound on the quadrupole tree itself at theta 0.6-0.7
    assert report["fp64"]["rms"] < 5e-2

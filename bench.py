"""Benchmark of the B200 Barnes-Hut gravity path.

Headline: force evaluations / s of one force pass (universe, keys, sort,
octree build, upward pass, traversal) at N = 16,777,216 (Plummer sphere, seed
42, eps 1e-3, bucket 32, theta 0.7) in the mixed-precision form, with inputs
resident in HBM.  A "step" is one force pass.  Also reported: the same pass
end to end through the C ABI with host buffers (e2e), the FP64 form, force
errors of both against the FP64 direct sum on 4096 seeded targets, the
traversal kernel's roofline, and the reference CPU path on the host cores.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU (torchrun): every rank holds the whole system, builds the whole
tree and traverses its contiguous share of the DFS-ordered buckets (strong
scaling of one force pass); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "force_evals_per_s"
UNIT = "force evaluations/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1 << 24)
    ap.add_argument("--workload", default="plummer")
    ap.add_argument("--theta", type=float, default=0.7)
    ap.add_argument("--bucket", type=int, default=32)
    ap.add_argument("--soft", type=float, default=1e-3)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64", "fp64_lists"])
    ap.add_argument("--targets", type=int, default=4096)
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--no-extras", action="store_true", help="skip e2e, fp64 comparison, errors, cpu baseline")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--sweep", default="0.5,0.7,1.0",
                    help="theta values of the accuracy / throughput sweep ('' to skip)")
    ap.add_argument("--sph", action="store_true",
                    help="time only the SPH density and pressure passes on the workload (1 GPU)")
    return ap.parse_args()


def make_ics(a):
    from paratreet_b200 import ics
    if a.workload == "plummer":
        return ics.plummer(a.n, seed=42, soft=a.soft)
    if a.workload == "mixture":
        return ics.mixture(a.n, seed=7, soft=a.soft)
    if a.workload == "hernquist":
        return ics.hernquist(a.n, seed=3, soft=a.soft)
    raise SystemExit(f"unknown workload {a.workload}")


def workload_config(a, world):
    return {"workload": f"{a.workload} N={a.n} eps={a.soft} bucket={a.bucket} theta={a.theta}",
            "n_particles": a.n, "bucket": a.bucket, "theta": a.theta, "precision": a.precision,
            "parallelism": f"buckets sharded over {world} GPU(s)" if world > 1 else "1 GPU",
            "l2": "inputs (>=1 GiB particle SoA, >=128 MiB node records) exceed the 126 MB L2"}


class ClockSampler:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def dist_init(a):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def max_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def rel_errors(a, ref):
    num = np.sqrt((a[0] - ref[0]) ** 2 + (a[1] - ref[1]) ** 2 + (a[2] - ref[2]) ** 2)
    den = np.sqrt(ref[0] ** 2 + ref[1] ** 2 + ref[2] ** 2)
    e = num / den
    return {"rms": float(np.sqrt(np.mean(e * e))), "p99": float(np.percentile(e, 99)), "max": float(e.max())}


# ----------------------------------------------------------------- reference arm
def run_reference(a):
    world, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return 0
    from oracle import oracle as O
    cfg = workload_config(a, 1)
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "metric": METRIC,
                          "unavailable": "reference-sources oracle (oracle/_ref) was not built"}))
        return 0
    cfg["precision"] = "fp64"  # the reference's gravity sources built with -DUSE_DOUBLE_FP
    p = make_ics(a)
    threads = os.cpu_count() or 1
    vals = []
    info = None
    for s in range(a.warmup + a.steps):
        v, info = reference_sample(p, a, threads, seconds=a.cpu_seconds / 2)
        if s >= a.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    out = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
           "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "data": "synthetic",
           "dtype": "f64", "config": cfg, "vs_baseline": None,
           "cpu_baseline": dict({"value": value, "unit": UNIT, "cores": threads, "kind": "reference"}, **info),
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


REF_FLAGS = "-O3 -ffp-contract=off -fno-fast-math -DUSE_DOUBLE_FP (FP64)"


def reference_sample(p, a, threads, seconds=10.0, bucket=None, theta=None, label=None):
    """Reference CPU path (the reference's own gravity sources): full tree
    build at N, then the traversal of bucket groups of 16 buckets (one
    Partition each; the reference's defaults give 8 partitions per PE) in a
    seeded random order until `seconds` are spent, scaled to all buckets.
    Returns (force evaluations/s, description dict)."""
    from oracle import oracle as O
    bucket = a.bucket if bucket is None else bucket
    theta = a.theta if theta is None else theta
    n = p["x"].size
    r = O.RefSim(p, bucket=bucket, theta=theta, dt_max=0.01, group=16, threads=threads)
    t_build, t_trav, frac = r.forces_sample(stride=0, budget_s=seconds)
    r.close()
    t_est = t_build + t_trav / max(frac, 1e-12)
    desc = (f"reference gravity sources (oracle/_ref, {REF_FLAGS}) on {threads} thread(s): full tree build at "
            f"N={n} ({t_build:.2f} s) + traversal of {100 * frac:.3f}% of the particles' buckets "
            f"({t_trav:.2f} s), traversal scaled to all buckets")
    info = {"sample": desc, "workload": label or workload_config(a, 1)["workload"],
            "sampled_fraction": frac, "build_s": t_build, "traversal_s_sampled": t_trav,
            "traversal_s_scaled": t_trav / max(frac, 1e-12), "threads": threads,
            "charm_equivalent": f"+p {threads} (one PE per host thread; the reference's defaults then cut "
                                f"{8 * threads} partitions, examples/Main.C:27-28)",
            "flags": REF_FLAGS, "tree_build": "restated serial build around the reference's own "
                                             "CentroidData / MultipoleMoments (oracle/ref_driver.cpp)"}
    return n / t_est, info


# ----------------------------------------------------------------- our arm
def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    world, rank, local = dist_init(a)
    import torch
    torch.cuda.set_device(local)
    from paratreet_b200.gravity import GravitySimulation

    p = make_ics(a)
    n = a.n
    sim = GravitySimulation(max_particles_per_leaf=a.bucket, theta=a.theta, max_timestep=0.01,
                            precision=a.precision, device=local)
    stream = torch.cuda.current_stream()
    sim.set_stream(stream.cuda_stream)
    sim.set_particles(p)
    if a.sph:
        out = {"workload": workload_config(a, world)["workload"], "sph_density": sph_density_rate(a, sim, stream),
               "sph_pressure": sph_pressure_rate(a, sim, stream), "sph_step": sph_step_rate(a, sim, stream)}
        if rank == 0:
            print(json.dumps(out))
        return

    shard = None
    if world > 1:  # buckets cut by measured work; results summed over the ranks (NCCL)
        from paratreet_b200.sharding import DeviceEngine, ShardedGravity
        shard = ShardedGravity(DeviceEngine(sim), world, rank)

    def pass_range():
        if shard is None:
            sim.start_down()
        else:
            shard.forces()

    sim.start_down()  # a full pass on every rank: bucket count and per-bucket work
    if shard is not None:
        shard.balance(sim.bucket_work().astype(np.int64))
    for _ in range(a.warmup):
        pass_range()
    torch.cuda.synchronize()
    barrier(world)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    trav_ms, cnts, launches = [], None, 0
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        barrier(world)
        for k in range(a.steps):
            ev[k][0].record(stream)
            pass_range()
            ev[k][1].record(stream)
            c = sim.counters()
            trav_ms.append(c["ms_traverse"])
            launches += int(c["launches"])  # kernels the library launched for this pass
            cnts = c
        torch.cuda.synchronize()
    step_ms = [s.elapsed_time(e) for s, e in ev]
    t_local = sum(step_ms) / 1e3
    t = max_over_ranks(t_local, world)
    barrier(world)
    value = n * a.steps / t

    # roofline of the traversal (dominant kernel)
    flops = 20.0 * cnts["n_pp"] + 66.0 * cnts["n_pc"]
    t_trav = float(np.mean(trav_ms)) / 1e3
    peaks = measured_peaks()
    clocks = clk.summary()
    sm_max = (peaks.get("sm_max_mhz") or clocks.get("sm_max_mhz") or 1965.0)
    import torch.cuda as tc
    nsm = tc.get_device_properties(local).multi_processor_count
    lanes = 128 if a.precision == "mixed" else 64
    peak_tf = nsm * lanes * 2 * sm_max * 1e6 / 1e12
    achieved = flops / t_trav / 1e12
    traffic = traversal_traffic(a)
    hbm = peaks.get("hbm_gbs") or 6650.0
    roofline = {"bound": "fp32" if a.precision == "mixed" else "fp64", "achieved": achieved,
                "peak": peak_tf, "unit": "TFLOP/s", "frac": achieved / peak_tf, "traffic": traffic,
                "traffic_source": TRAVERSE_MIXED_DRAM_SOURCE if traffic else None,
                "dram_gbs": (traffic / t_trav / 1e9) if traffic else None,
                "dram_frac_of_hbm": (traffic / t_trav / 1e9 / hbm) if traffic else None,
                "kernel": {"mixed": "walk_lists + eval_p2c2 + eval_p2p", "fp64": "traverse_f64",
                           "fp64_lists": "walk_lists + eval_p2c_f64 + eval_p2p_f64"}[a.precision],
                "flops_per_launch": flops,
                "flop_model": "20 per P2P pair + 66 per P2C evaluation",
                "peak_source": f"nominal: {nsm} SMs x {lanes} {'FP32' if lanes == 128 else 'FP64'} lanes x 2 x "
                               f"{sm_max:.0f} MHz (no measured FP32/FP64 figure in MEASURED_PEAKS.json)"}

    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": t * 1e3 / a.steps,
           "step_ms": [round(x, 3) for x in step_ms], "higher_is_better": True,
           "scaling": "strong", "vs_baseline": None, "dtype": "f32 interactions / f64 tree"
           if a.precision == "mixed" else "f64", "data": "synthetic (seeded Plummer sphere)",
           "config": workload_config(a, world), "gpu_launches": launches,
           "roofline": roofline, "clocks": clocks,
           "phases_ms": {k: cnts[k] for k in ("ms_keys", "ms_sort", "ms_build", "ms_upward", "ms_traverse",
                                              "ms_total")},
           "interactions": {"n_pp": cnts["n_pp"], "n_pc": cnts["n_pc"], "n_open": cnts["n_open"],
                            "n_nodes": cnts["n_nodes"], "n_buckets": cnts["n_buckets"]},
           "interactions_per_s": (cnts["n_pp"] + cnts["n_pc"]) / t_trav,
           "phases_roofline": phase_rooflines(cnts, n, peaks)}

    if not a.no_extras:
        out.update(extras(a, sim, p, world, rank, stream, value, shard))
    sim.close()
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


# DRAM bytes (read + write) per particle of the three kernels of one mixed
# traversal, Plummer sphere, bucket 32, theta 0.7, eps 1e-3: ncu
# dram__bytes_read.sum + dram__bytes_write.sum of one launch of each kernel on
# the N = 2^21 pass, divided by N (profiles/traversal_kernels_plummer_2m.md
# holds the commands and the figures).  Every kernel reads and writes in
# proportion to the interactions, which grow with N in the same proportion at
# fixed theta, so the per-particle figure scales to the bench size.
TRAVERSE_MIXED_DRAM_PER_PARTICLE = {
    "walk_lists": (67588352 + 893458432) / 2097152.0,
    "eval_p2c2": (900244480 + 80266240) / 2097152.0,
    "eval_p2p": (413512448 + 60272640) / 2097152.0,
}
TRAVERSE_MIXED_DRAM_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of each kernel at "
                              "N = 2^21, scaled by N (profiles/traversal_kernels_plummer_2m.md)")


def traversal_traffic(a):
    """DRAM bytes of one mixed traversal at the bench size, from the
    per-particle figures measured at N = 2^21; None for other workloads."""
    if (a.workload, a.theta, a.bucket, a.precision, a.soft) == ("plummer", 0.7, 32, "mixed", 1e-3):
        return sum(TRAVERSE_MIXED_DRAM_PER_PARTICLE.values()) * a.n
    return None


def sph_density_rate(a, sim, stream):
    """The SPH example's density pass (k = 32 neighbours + M4 density) on
    the same particles: particles/s through pt_sph_density (tree build,
    neighbour search, density and the D2H of density and ball^2)."""
    import torch
    sim.sph_density()
    ts = []
    for _ in range(2):
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        sim.sph_density()
        s1.record(stream)
        torch.cuda.synchronize()
        ts.append(s0.elapsed_time(s1) / 1e3)
    sim.start_down()  # leave the handle with a force pass, as the other extras expect
    return {"particles_per_s": a.n / float(np.mean(ts)), "ms_per_pass": 1e3 * float(np.mean(ts)),
            "neighbours": 32, "note": "density pass of the SPH example: tree build + kNN + density + D2H"}


def sph_pressure_rate(a, sim, stream):
    """The SPH example's pressure pass after its density pass (ForceFn +
    doSPHCalc with the opposing reactions): particles/s through
    pt_sph_pressure (density pass, H2D of u, pressure kernel, D2H of density,
    accelerations and PdV), seeded internal energies."""
    import torch
    u = np.random.default_rng(17).uniform(0.5, 1.5, a.n)
    sim.sph_pressure(u)
    ts = []
    for _ in range(2):
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        sim.sph_pressure(u)
        s1.record(stream)
        torch.cuda.synchronize()
        ts.append(s0.elapsed_time(s1) / 1e3)
    sim.start_down()
    return {"particles_per_s": a.n / float(np.mean(ts)), "ms_per_pass": 1e3 * float(np.mean(ts)),
            "neighbours": 32, "note": "density pass + pressure pass of the SPH example, host in and out"}


def driver_step_rate(a, sim, stream, steps=20):
    """Seconds per Driver::run iteration (pt_step: force pass, time step from
    the maximum speed, the reference's kick and perturb) on the bench
    particles, over `steps` consecutive iterations after two warm-up ones
    (median, mean and max).  Moves the particles: run it after the extras
    that read them."""
    import torch
    sim.run(2)
    ts, tf = [], []
    for _ in range(steps):
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        sim.run(1)
        s1.record(stream)
        torch.cuda.synchronize()
        ts.append(s0.elapsed_time(s1))
        tf.append(float(sim.counters()["ms_total"]))
    k = int(np.argsort(ts)[len(ts) // 2])  # the median step and its own force pass
    step, force = float(ts[k]), float(tf[k])
    return {"s_per_step": step / 1e3, "s_per_step_mean": float(np.mean(ts)) / 1e3,
            "s_per_step_max": float(np.max(ts)) / 1e3, "max_over_median": float(np.max(ts)) / step,
            "force_pass_ms": force, "rest_ms": step - force,
            "steps_ms": [round(t, 3) for t in ts], "force_pass_ms_per_step": [round(t, 3) for t in tf],
            "warmup_steps": 2,
            "note": f"median, mean and max of {steps} consecutive steps; rest = time step (max-speed "
                    "reduction) + kick/perturb kernel + host synchronisation of the median step"}


def sph_step_rate(a, sim, stream):
    """Iterations of the SPH example (pt_sph_step: density pass, pressure
    pass, kick + perturb with the internal-energy updates, dt = 0.01) on the
    same particles, seeded internal energies; the SPH state goes in and out
    through host memory once per call.  Moves the particles: run it last."""
    import torch
    u = np.random.default_rng(17).uniform(0.5, 1.5, a.n)
    u, up, vp = sim.sph_run(1, u)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    sim.sph_run(2, u, up, vp)
    s1.record(stream)
    torch.cuda.synchronize()
    t = s0.elapsed_time(s1) / 1e3 / 2
    return {"particles_per_s": a.n / t, "ms_per_step": 1e3 * t, "neighbours": 32,
            "note": "SPH example iteration: tree build + kNN + density + pressure + kick/perturb"}


def phase_rooflines(c, n, peaks):
    """HBM roofline of the bandwidth-bound phases of the last pass: their
    algorithmic bytes (keys 36 B/particle; sort 8 + 8 x 24 B and permute of
    the eight FP64 arrays + order 132 B per particle; build 8 B/particle +
    32 B/node; upward 32 B/particle + 160 B/node) over the phase's event time,
    against the measured copy bandwidth."""
    hbm = peaks.get("hbm_gbs") or 6650.0
    nodes = c["n_nodes"]
    rows = {"keys": (36.0 * n, c["ms_keys"]), "sort_permute": ((200.0 + 132.0) * n, c["ms_sort"]),
            "build": (8.0 * n + 32.0 * nodes, c["ms_build"]), "upward": (32.0 * n + 160.0 * nodes, c["ms_upward"])}
    out = {}
    for k, (b, ms) in rows.items():
        gbs = b / (ms / 1e3) / 1e9 if ms > 0 else None
        out[k] = {"bytes": b, "ms": ms, "achieved_gbs": gbs, "frac": (gbs / hbm) if gbs else None}
    out["peak_gbs"] = hbm
    out["peak_source"] = "measured (MEASURED_PEAKS.json hbm_gbs)" if peaks.get("hbm_gbs") else "fallback 6650 GB/s"
    return out


def theta_sweep(a, sim, tgt, direct, stream):
    """Force evaluations/s and errors vs the FP64 direct sum of the three
    forms (mixed; FP64 over the same two-phase lists; the ordered FP64 walk)
    over the theta values of --sweep (same particles and targets)."""
    rows = []
    for th in [float(v) for v in a.sweep.split(",") if v]:
        sim.set_theta(th)
        row = {"theta": th}
        for prec, reps in (("mixed", 2), ("fp64_lists", 1), ("fp64", 1)):
            row[prec] = timed_form(a, sim, tgt, direct, stream, prec, reps)
        row["ratio_mixed_over_fp64"] = row["mixed"]["force_evals_per_s"] / row["fp64"]["force_evals_per_s"]
        row["ratio_mixed_over_fp64_lists"] = (row["mixed"]["force_evals_per_s"] /
                                              row["fp64_lists"]["force_evals_per_s"])
        rows.append(row)
    sim.set_theta(a.theta)
    sim.set_precision(a.precision)
    return rows


def timed_form(a, sim, tgt, direct, stream, prec, reps):
    """Force evaluations/s (mean of reps passes after one untimed pass) and
    the force error against the direct sum, of one form at the current theta."""
    import torch
    sim.set_precision(prec)
    sim.start_down()
    ts = []
    for _ in range(reps):
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        sim.start_down()
        s1.record(stream)
        torch.cuda.synchronize()
        ts.append(s0.elapsed_time(s1) / 1e3)
    acc = sim.accelerations()
    c = sim.counters()
    return {"force_evals_per_s": a.n / float(np.mean(ts)), "ms_per_pass": 1e3 * float(np.mean(ts)),
            "ms_traverse": c["ms_traverse"],
            "err_vs_direct": rel_errors((acc["ax"][tgt], acc["ay"][tgt], acc["az"][tgt]), direct),
            "interactions_per_particle": (c["n_pp"] + c["n_pc"]) / a.n}


def accuracy_clause(a, sim, tgt, direct, stream, bound=1e-4, lo=0.35, hi=0.50):
    """The headline metric under its own accuracy clause: the largest theta on
    a 0.01 grid in [lo, hi] at which the tree's RMS relative force error
    against the FP64 direct sum (the seeded targets) is <= bound, found by
    bisection on the mixed form (whose error equals the FP64 form's to about
    1e-7 relative), then both forms timed and their errors measured there,
    and the errors one grid step above it."""
    grid = [round(lo + 0.01 * k, 2) for k in range(int(round((hi - lo) / 0.01)) + 1)]
    probes = {}

    def rms(th):
        if th not in probes:
            sim.set_theta(th)
            sim.set_precision("mixed")
            sim.start_down()
            acc = sim.accelerations()
            probes[th] = rel_errors((acc["ax"][tgt], acc["ay"][tgt], acc["az"][tgt]), direct)["rms"]
        return probes[th]

    out = {"bound_rms": bound, "grid": [grid[0], grid[-1], 0.01]}
    if rms(grid[0]) > bound:
        out["theta"] = None
        out["note"] = f"rms {probes[grid[0]]:.3e} > bound already at theta {grid[0]}"
    else:
        i, j = 0, len(grid) - 1  # rms(grid[i]) <= bound; grid[j] unknown or above
        if rms(grid[j]) <= bound:
            i = j
        while j - i > 1:
            k = (i + j) // 2
            if rms(grid[k]) <= bound:
                i = k
            else:
                j = k
        th = grid[i]
        sim.set_theta(th)
        row = {"theta": th}
        row["mixed"] = timed_form(a, sim, tgt, direct, stream, "mixed", 2)
        row["fp64_lists"] = timed_form(a, sim, tgt, direct, stream, "fp64_lists", 1)
        row["fp64"] = timed_form(a, sim, tgt, direct, stream, "fp64", 1)
        row["ratio_mixed_over_fp64"] = row["mixed"]["force_evals_per_s"] / row["fp64"]["force_evals_per_s"]
        row["ratio_mixed_over_fp64_lists"] = (row["mixed"]["force_evals_per_s"] /
                                              row["fp64_lists"]["force_evals_per_s"])
        row["all_within_bound"] = bool(all(row[f]["err_vs_direct"]["rms"] <= bound
                                           for f in ("mixed", "fp64_lists", "fp64")))
        out.update(row)
        if i + 1 < len(grid):
            out["next_theta_mixed_rms"] = {"theta": grid[i + 1], "rms": rms(grid[i + 1])}
    out["probes_mixed_rms"] = {str(k): v for k, v in sorted(probes.items())}
    sim.set_theta(a.theta)
    sim.set_precision(a.precision)
    return out


def adjoint_cost(a, stream):
    """Cost of one adjoint force pass against one forward pass on the
    differentiation workload (Hernquist N = 262,144, seed 3, eps 0.01,
    theta 0.6, bucket 16), each through the C ABI with its host data in
    pinned buffers: the forward pass with its accelerations read back (the
    plain two-phase mixed pass, and the pass that also records the
    interaction lists the adjoint differentiates), and pt_adjoint with the
    cotangent in and the gradients out.  Each the mean of 5 calls after two
    untimed ones."""
    import torch
    from paratreet_b200 import ics
    from paratreet_b200.gravity import GravitySimulation
    n = 262144
    q = ics.hernquist(n, seed=3, soft=0.01)
    cot = np.random.default_rng(64).normal(size=(3, n))

    def timed(f, reps=5):
        f()
        f()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(reps):
            f()
        s1.record(stream)
        torch.cuda.synchronize()
        return s0.elapsed_time(s1) / reps

    # pinned host buffers, allocated once: the timed calls measure the
    # library and its copies, not numpy's page faults
    def pinned(k):
        return torch.empty(n, dtype=torch.float64).pin_memory().numpy()

    acc_out = {k: pinned(k) for k in ("ax", "ay", "az", "pot", "pot_full")}
    grad_out = {k: pinned(k) for k in ("gx", "gy", "gz", "gm")}
    cot_in = [pinned(k) for k in range(3)]
    for k in range(3):
        cot_in[k][:] = cot[k]

    def forward(sim):
        sim.start_down()
        sim.accelerations(acc_out)

    out = {"workload": "hernquist N=262144 eps=0.01 bucket=16 theta=0.6",
           "note": "each call through the C ABI with its host data in pinned buffers allocated once "
                   "(accelerations read back; cotangent in, gradients out)"}
    with GravitySimulation(max_particles_per_leaf=16, theta=0.6, precision="mixed") as plain:
        plain.set_stream(stream.cuda_stream)
        plain.set_particles(q)
        out["forward_ms_two_phase"] = timed(lambda: forward(plain))
    with GravitySimulation(max_particles_per_leaf=16, theta=0.6, precision="mixed", record_lists=True) as s:
        s.set_stream(stream.cuda_stream)
        s.set_particles(q)
        out["forward_ms_recording_lists"] = timed(lambda: forward(s))
        s.start_down()
        out["adjoint_ms"] = timed(lambda: s.adjoint(*cot_in, out=grad_out))
    out["adjoint_over_recording_forward"] = out["adjoint_ms"] / out["forward_ms_recording_lists"]
    out["adjoint_over_two_phase_forward"] = out["adjoint_ms"] / out["forward_ms_two_phase"]
    out["target"] = "adjoint <= 2.5 x one forward pass"
    return out


def extras(a, sim, p, world, rank, stream, value, shard=None):
    import torch
    n = a.n
    res = {}
    # e2e through the C ABI with pinned host buffers
    fields = ("x", "y", "z", "vx", "vy", "vz", "m", "soft")
    pinned = {k: torch.from_numpy(np.ascontiguousarray(p[k])).pin_memory() for k in fields}
    outs = {k: torch.empty(n, dtype=torch.float64).pin_memory() for k in ("ax", "ay", "az", "pot_full")}
    host = {k: pinned[k].numpy() for k in fields}
    hout = {k: outs[k].numpy() for k in outs}
    torch.cuda.synchronize()
    steps = max(1, min(a.steps, 3))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    e0.record(stream)
    for _ in range(steps):
        sim.set_particles(host)
        if shard is None:
            sim.start_down()
        else:
            shard.forces()
        sim.accelerations({"ax": hout["ax"], "ay": hout["ay"], "az": hout["az"], "pot": None,
                           "pot_full": hout["pot_full"]})
    e1.record(stream)
    torch.cuda.synchronize()
    t = max_over_ranks(e0.elapsed_time(e1) / 1e3, world)
    res["e2e"] = {"value": n * steps / t, "unit": UNIT, "h2d_bytes_per_step": 8 * 8 * n,
                  "d2h_bytes_per_step": 4 * 8 * n, "steps": steps,
                  "path": "pt_set_particles (pinned H2D) + pt_compute_forces + pt_get_accel (D2H)"}
    if world > 1:
        # the accuracy, FP64, sweep, SPH and CPU-baseline extras belong to the
        # 1-GPU run; every rank stops here so that none holds its GPU waiting
        return res
    # force errors vs the FP64 direct sum on seeded targets, mixed and FP64
    rng = np.random.default_rng(43)
    tgt = np.sort(rng.choice(n, size=min(a.targets, n), replace=False)).astype(np.int32)
    dax, day, daz, _ = sim.direct_sum(tgt)
    sim.start_down()
    am = sim.accelerations()
    err_m = rel_errors((am["ax"][tgt], am["ay"][tgt], am["az"][tgt]), (dax, day, daz))
    other = "fp64" if a.precision == "mixed" else "mixed"
    sim.set_precision(other)
    sim.start_down()
    t64 = []
    for _ in range(a.fp64_steps):
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        sim.start_down()
        s1.record(stream)
        torch.cuda.synchronize()
        t64.append(s0.elapsed_time(s1) / 1e3)
    a64 = sim.accelerations()
    c64 = sim.counters()
    err_o = rel_errors((a64["ax"][tgt], a64["ay"][tgt], a64["az"][tgt]), (dax, day, daz))
    diff = rel_errors((am["ax"], am["ay"], am["az"]), (a64["ax"], a64["ay"], a64["az"]))
    sim.set_precision(a.precision)
    v_other = n / float(np.mean(t64))
    res["precision_comparison"] = {
        f"{a.precision}_force_evals_per_s": value, f"{other}_force_evals_per_s": v_other,
        "ratio_mixed_over_fp64": (value / v_other) if a.precision == "mixed" else (v_other / value),
        f"{a.precision}_err_vs_direct": err_m, f"{other}_err_vs_direct": err_o,
        "mixed_vs_fp64_all_particles": diff, "targets": int(tgt.size), "target_seed": 43,
        f"{other}_ms_traverse": c64["ms_traverse"]}
    import torch.cuda as tc
    nsm = tc.get_device_properties(torch.cuda.current_device()).multi_processor_count
    sm_max = measured_peaks().get("sm_max_mhz") or 1965.0
    peak64 = nsm * 64 * 2 * sm_max * 1e6 / 1e12

    def fp64_roofline(c, kernel):
        ach = (20.0 * c["n_pp"] + 66.0 * c["n_pc"]) / (c["ms_traverse"] / 1e3) / 1e12
        return {"bound": "fp64", "achieved": ach, "peak": peak64, "unit": "TFLOP/s", "frac": ach / peak64,
                "kernel": kernel, "flop_model": "20 per P2P pair + 66 per P2C evaluation",
                "peak_source": f"nominal: {nsm} SMs x 64 FP64 lanes x 2 x {sm_max:.0f} MHz"}

    if other == "fp64":
        res["precision_comparison"]["fp64_roofline"] = fp64_roofline(c64, "traverse_f64")
    if a.precision == "mixed":
        # the FP64 comparator built like the mixed form (same lists and layout)
        fl = timed_form(a, sim, tgt, (dax, day, daz), stream, "fp64_lists", 2)
        cl = sim.counters()
        sim.set_precision(a.precision)
        pc = res["precision_comparison"]
        pc["fp64_lists_force_evals_per_s"] = fl["force_evals_per_s"]
        pc["fp64_lists_err_vs_direct"] = fl["err_vs_direct"]
        pc["fp64_lists_ms_traverse"] = cl["ms_traverse"]
        pc["ratio_mixed_over_fp64_lists"] = value / fl["force_evals_per_s"]
        pc["fp64_lists_roofline"] = fp64_roofline(cl, "walk_lists + eval_p2c_f64 + eval_p2p_f64")
        pc["forms"] = {"mixed": "FP32 interactions over the two-phase lists",
                       "fp64_lists": "FP64 interactions over the same two-phase lists and work layout",
                       "fp64": "the ordered FP64 walk, bit-exact with the reference"}
    res["theta_sweep"] = theta_sweep(a, sim, tgt, (dax, day, daz), stream) if a.sweep else []
    res["accuracy_clause"] = accuracy_clause(a, sim, tgt, (dax, day, daz), stream)
    res["sph_density"] = sph_density_rate(a, sim, stream)
    res["sph_pressure"] = sph_pressure_rate(a, sim, stream)
    res["driver_step"] = driver_step_rate(a, sim, stream)
    res["adjoint_cost"] = adjoint_cost(a, stream)
    # CPU baseline: the reference's gravity sources on the host cores
    try:
        threads = os.cpu_count() or 1
        v, info = reference_sample(p, a, threads, seconds=a.cpu_seconds)
        res["cpu_baseline"] = dict({"value": v, "unit": UNIT, "cores": threads, "kind": "reference"}, **info)
        # one core, for the scaling of the reference's own code over the host threads
        v1, info1 = reference_sample(p, a, 1, seconds=max(1.0, a.cpu_seconds / 4))
        res["cpu_baseline"]["single_core"] = dict({"value": v1, "threads_speedup": v / v1 if v1 else None}, **info1)
        res["cpu_baseline"]["configs"] = cpu_baseline_configs(a, threads, v, info)
    except Exception as e:  # reported, not fatal
        res["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                               "sample": f"failed: {e}"}
    return res


def cpu_baseline_configs(a, threads, v_c2, info_c2):
    """The reference's CPU path at the smaller workloads as well: the 10,000
    particle Plummer sphere (eps 0.01, bucket 16) and the 2^20 mixture (eps
    1e-4, bucket 16), theta 0.7, one full force pass each on all host threads
    and on one, beside the bench workload's own figure."""
    from paratreet_b200 import ics
    rows = {}
    for name, gen, kw in (("plummer_10k", ics.plummer, dict(n=10000, seed=42, soft=0.01)),
                          ("mixture_1m", ics.mixture, dict(n=1 << 20, seed=7, soft=1e-4))):
        q = gen(**kw)
        label = f"{name}: N={kw['n']} eps={kw['soft']} bucket=16 theta=0.7"
        row = {}
        for th, budget in ((threads, 60.0), (1, 20.0)):
            v, info = reference_sample(q, a, th, seconds=budget, bucket=16, theta=0.7, label=label)
            row[f"threads_{th}"] = {"value": v, "sampled_fraction": info["sampled_fraction"],
                                   "build_s": info["build_s"], "traversal_s_scaled": info["traversal_s_scaled"],
                                   "charm_equivalent": f"+p {th}"}
        rows[name] = dict(row, workload=label, unit=UNIT)
    rows["plummer_16m"] = {"workload": info_c2["workload"], "unit": UNIT,
                           f"threads_{threads}": {"value": v_c2, "sampled_fraction": info_c2["sampled_fraction"],
                                                  "build_s": info_c2["build_s"],
                                                  "traversal_s_scaled": info_c2["traversal_s_scaled"],
                                                  "charm_equivalent": f"+p {threads}"}}
    return rows


if __name__ == "__main__":
    sys.exit(main())

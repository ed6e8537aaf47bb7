"""The C++ host facade (include/paratreet_gpu.hpp) compiled into a small host
program (tests/cpp/gravity_demo.cpp) with g++ and linked against the library:
Tipsy interoperability with the Python reader/writer on the CPU, and on the
GPU a force pass through run_gravity and Driver::run steps compared with the
same calls made from Python."""
import os
import subprocess

import numpy as np
import pytest

from paratreet_b200 import ics, tipsy

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "paratreet_b200")


@pytest.fixture(scope="module")
def demo(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "gravity_demo")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "gravity_demo.cpp"), "-L", LIBDIR, "-lpt_gravity",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def typed(n, seed):
    p = ics.plummer(n, seed=seed, soft=0.02)
    p["type"] = np.random.default_rng(seed).integers(0, 3, n).astype(np.int8)
    return p


def test_cpp_reads_and_writes_tipsy_like_python(demo, tmp_path):
    p = typed(500, 3)
    src, dst = str(tmp_path / "in.tipsy"), str(tmp_path / "out.tipsy")
    tipsy.write_tipsy(src, p, time=0.5, softening=True)
    r = subprocess.run([demo, "copy", src, dst], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "read 500 particles" in r.stdout
    a, ha = tipsy.read_tipsy(src)
    b, hb = tipsy.read_tipsy(dst)
    assert (ha.nsph, ha.ndark, ha.nstar, ha.time) == (hb.nsph, hb.ndark, hb.nstar, hb.time)
    for k in ("x", "y", "z", "vx", "vy", "vz", "m", "type"):
        assert np.array_equal(a[k], b[k]), k
    # like the reference's TipsyWriter, the C++ writer leaves softening unset
    assert np.all(b["soft"] == 0.0)
    # and the Python writer reproduces the C++ file byte for byte
    again = str(tmp_path / "again.tipsy")
    tipsy.write_tipsy(again, dict(b, type=b["type"]), time=0.5)
    assert open(again, "rb").read() == open(dst, "rb").read()


def test_cpp_rejects_a_bad_file(demo, tmp_path):
    bad = str(tmp_path / "bad.tipsy")
    open(bad, "wb").write(b"\x01" * 40)
    r = subprocess.run([demo, "copy", bad, str(tmp_path / "o")], capture_output=True, text=True)
    assert r.returncode == 1 and "not a Tipsy file" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_cpp_run_gravity_matches_python(demo, tmp_path, prec):
    from paratreet_b200.gravity import GravitySimulation
    p = ics.plummer(6000, seed=9, soft=0.01)
    f = str(tmp_path / "p.tipsy")
    tipsy.write_tipsy(f, p, softening=True)
    q, _ = tipsy.read_tipsy(f)  # float32 mass / softening as the C++ host sees them
    acc = str(tmp_path / "p.acc")
    args = [demo, "forces", f, acc, "0.6", "16"] + (["mixed"] if prec == "mixed" else [])
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = tipsy.read_acc(acc)
    with GravitySimulation(max_particles_per_leaf=16, theta=0.6, precision=prec) as s:
        s.set_particles(q)
        s.start_down()
        a = s.accelerations()
    want = np.stack([a["ax"], a["ay"], a["az"]])
    assert np.allclose(got, want, rtol=1e-13, atol=0)  # %.14g output: 14 significant digits


@pytest.mark.gpu
def test_cpp_driver_steps_match_python(demo, tmp_path):
    from paratreet_b200.gravity import GravitySimulation
    p = ics.plummer(3000, seed=2, soft=0.02)
    f, out = str(tmp_path / "s.tipsy"), str(tmp_path / "s_out.tipsy")
    tipsy.write_tipsy(f, p, softening=True)
    q, _ = tipsy.read_tipsy(f)
    r = subprocess.run([demo, "steps", f, out, "0.7", "16", "0.01", "3"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got, _ = tipsy.read_tipsy(out)
    with GravitySimulation(max_particles_per_leaf=16, theta=0.7, max_timestep=0.01) as s:
        s.set_particles(q)
        s.run(3)
        st = s.state()
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(got[k], st[k]), k


@pytest.mark.gpu
def test_cpp_sph_pressure_matches_python(demo, tmp_path):
    """Gravity::sph_pressure (the SPH example's traversalFn) from C++ against
    the same pass through the Python binding: densities to 1e-13, pressure
    accelerations and PdV to 1e-12 of the largest value (atomic summation
    order of the reactions)."""
    from paratreet_b200.gravity import GravitySimulation
    p = ics.plummer(5000, seed=6, soft=0.02)
    f, out = str(tmp_path / "g.tipsy"), str(tmp_path / "sph.txt")
    tipsy.write_tipsy(f, p, softening=True)
    q, _ = tipsy.read_tipsy(f)
    r = subprocess.run([demo, "sph", f, out, "16"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.loadtxt(out).T
    u = 1.0 + (np.arange(q["x"].size) % 7) / 10.0
    with GravitySimulation(max_particles_per_leaf=16) as s:
        s.set_particles(q)
        want = s.sph_pressure(u)
    assert np.allclose(got[0], want[0], rtol=1e-13, atol=0)
    for g, w in zip(got[1:], want[1:]):
        assert np.abs(g - w).max() <= 1e-12 * max(np.abs(w).max(), 1e-300)


@pytest.mark.gpu
def test_cpp_sph_run_matches_python(demo, tmp_path):
    """Gravity::sph_run (iterations of the SPH example) from C++ against
    GravitySimulation.sph_run through the Python binding: positions,
    velocities and energies within 1e-12 of each field's largest value (the
    reactions' atomic summation order differs between the two runs)."""
    from paratreet_b200.gravity import GravitySimulation
    p = ics.plummer(4000, seed=6, soft=0.02)
    f, out = str(tmp_path / "g.tipsy"), str(tmp_path / "sphsteps.txt")
    tipsy.write_tipsy(f, p, softening=True)
    q, _ = tipsy.read_tipsy(f)
    r = subprocess.run([demo, "sphsteps", f, out, "16", "0.01", "2"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.loadtxt(out).T
    u = 1.0 + (np.arange(q["x"].size) % 7) / 10.0
    with GravitySimulation(max_particles_per_leaf=16, max_timestep=0.01) as s:
        s.set_particles(q)
        wu, wup, _ = s.sph_run(2, u)
        st = s.state()
    want = [st[k] for k in ("x", "y", "z", "vx", "vy", "vz")] + [wu, wup]
    for g, w in zip(got, want):
        assert np.abs(g - w).max() <= 1e-12 * max(np.abs(w).max(), 1e-300)
    assert not np.allclose(got[0], q["x"])

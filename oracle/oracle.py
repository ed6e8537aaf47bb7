"""ctypes front-end for the CPU oracles -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` may import this module, and only as the checker or as the timed
CPU baseline; the product (``paratreet_b200``) never imports it.

Two oracles share one interface:

* ``PortSim``  -- ``oracle/libpt_oracle.so``, the plain-C restatement.
* ``RefSim``   -- ``oracle/_ref/libptref.so``, the reference's own gravity
  sources (examples/GravityVisitor.h, CentroidData.h, MultipoleMoments.h,
  src/Node.h, src/Particle.{h,C}) compiled where they lie, driven by a
  restated build/traversal.  Present only where it was built.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "libpt_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libptref.so")

_dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")

NODE_LEAF, NODE_EMPTY, NODE_INTERNAL = 1, 2, 6


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def _bind(lib, prefix: str):
    f = lambda name: getattr(lib, prefix + name)  # noqa: E731
    f("create").restype = C.c_void_p
    f("destroy").argtypes = [C.c_void_p]
    f("get_acc").argtypes = [C.c_void_p] + [_dp] * 4 + ([_dp] if prefix == "pto_" else [])
    f("get_keys").argtypes = [C.c_void_p, _u64p]
    f("get_state").argtypes = [C.c_void_p] + [_dp] * 6
    f("get_universe").argtypes = [C.c_void_p, _dp, _dp]
    f("get_counters").argtypes = [C.c_void_p, _u64p, _dp, _dp]
    f("num_nodes").argtypes = [C.c_void_p]
    f("num_nodes").restype = C.c_long
    f("get_nodes").argtypes = [C.c_void_p, _u64p, _i32p, _dp]
    f("num_buckets").argtypes = [C.c_void_p]
    f("num_buckets").restype = C.c_long
    f("get_bucket_keys").argtypes = [C.c_void_p, _u64p]
    f("list_total").argtypes = [C.c_void_p]
    f("list_total").restype = C.c_long
    f("get_lists").argtypes = [C.c_void_p, _i64p, _u64p, _i32p]


_port = None
_ref = None


def _port_lib():
    global _port
    if _port is None:
        lib = C.CDLL(PORT_LIB)
        _bind(lib, "pto_")
        lib.pto_create.argtypes = [C.c_int] + [_dp] * 8 + [C.c_int, C.c_double, C.c_double, C.c_int]
        lib.pto_forces.argtypes = [C.c_void_p, C.c_int]
        lib.pto_run.argtypes = [C.c_void_p, C.c_int]
        lib.pto_direct.argtypes = [C.c_int] + [_dp] * 5 + [C.c_int, _i32p] + [_dp] * 4 + [C.c_int]
        lib.pto_sph_density.argtypes = [C.c_int] + [_dp] * 4 + [C.c_int, C.c_int, _dp, _dp, _i32p, _dp]
        lib.pto_sph_pressure.argtypes = [C.c_int] + [_dp] * 10 + [_i32p, _dp, C.c_int] + [_dp] * 4
        lib.pto_set_periodic.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_double, C.c_double]
        lib.pto_set_traversal.argtypes = [C.c_void_p, C.c_int]
        lib.pto_get_mono.argtypes = [C.c_void_p]
        lib.pto_get_mono.restype = C.c_ulonglong
        lib.pto_ewald_direct.argtypes = [C.c_int] + [_dp] * 5 + [C.c_double, C.c_int, _i32p] + [_dp] * 4 + [C.c_int]
        _port = lib
    return _port


def _ref_lib():
    global _ref
    if _ref is None:
        lib = C.CDLL(REF_LIB)
        _bind(lib, "ptref_")
        lib.ptref_create.argtypes = [C.c_int] + [_dp] * 8 + [C.c_int, C.c_double, C.c_double, C.c_int, C.c_int]
        lib.ptref_run.argtypes = [C.c_void_p, C.c_int]
        lib.ptref_set_record_lists.argtypes = [C.c_void_p, C.c_int]
        lib.ptref_forces_sample.argtypes = [C.c_void_p, C.c_double] + [C.POINTER(C.c_double)] * 3
        lib.ptref_set_periodic.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int]
        lib.ptref_set_traversal.argtypes = [C.c_void_p, C.c_int]
        lib.ptref_dual.argtypes = [C.c_void_p, _dp, _dp, _dp, _u64p]
        lib.ptref_sph_pressure.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
        lib.ptref_sph_density.argtypes = [C.c_void_p, _dp, _dp, _i32p, _dp]
        lib.ptref_sph_step.argtypes = [C.c_void_p, C.c_int] + [_dp] * 5
        _ref = lib
    return _ref


@dataclass
class Tree:
    keys: np.ndarray      # u64 node keys
    types: np.ndarray     # int32 node types (1 leaf, 2 empty, 6 internal)
    depth: np.ndarray
    count: np.ndarray
    moments: np.ndarray   # (n, 18) float64


@dataclass
class Lists:
    bucket_keys: np.ndarray
    offsets: np.ndarray
    keys: np.ndarray
    kinds: np.ndarray


def _arrs(p):
    return [np.ascontiguousarray(p[k], dtype=np.float64) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "soft")]


class _Sim:
    prefix = ""

    def __init__(self, lib, handle, n):
        self._lib, self._h, self.n = lib, handle, n

    def _f(self, name):
        return getattr(self._lib, self.prefix + name)

    def close(self):
        if self._h:
            self._f("destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def keys(self):
        k = np.zeros(self.n, np.uint64)
        self._f("get_keys")(self._h, k)
        return k

    def state(self):
        a = [np.zeros(self.n) for _ in range(6)]
        self._f("get_state")(self._h, *a)
        return a

    def universe(self):
        lo, hi = np.zeros(3), np.zeros(3)
        self._f("get_universe")(self._h, lo, hi)
        return lo, hi

    def counters(self):
        c = np.zeros(4, np.uint64)
        t = np.zeros(2)
        dt = np.zeros(1)
        self._f("get_counters")(self._h, c, t, dt)
        return {"n_pp": int(c[0]), "n_pc": int(c[1]), "n_open": int(c[2]), "n_buckets": int(c[3]),
                "t_build": float(t[0]), "t_traverse": float(t[1]), "last_dt": float(dt[0])}

    def tree(self) -> Tree:
        nn = self._f("num_nodes")(self._h)
        k = np.zeros(nn, np.uint64)
        ints = np.zeros(4 * nn, np.int32)
        d = np.zeros(18 * nn)
        self._f("get_nodes")(self._h, k, ints, d)
        ints = ints.reshape(nn, 4)
        return Tree(k, ints[:, 0].copy(), ints[:, 1].copy(), ints[:, 2].copy(), d.reshape(nn, 18))

    def lists(self) -> Lists:
        nb = self._f("num_buckets")(self._h)
        bk = np.zeros(nb, np.uint64)
        self._f("get_bucket_keys")(self._h, bk)
        tot = self._f("list_total")(self._h)
        off = np.zeros(nb + 1, np.int64)
        keys = np.zeros(max(tot, 1), np.uint64)
        kinds = np.zeros(max(tot, 1), np.int32)
        self._f("get_lists")(self._h, off, keys, kinds)
        return Lists(bk, off, keys[:tot], kinds[:tot])


class PortSim(_Sim):
    """The plain-C restatement (oracle/pt_oracle.c)."""
    prefix = "pto_"

    def __init__(self, p: dict, bucket=16, theta=0.7, dt_max=0.01, threads=1):
        lib = _port_lib()
        n = p["x"].size
        h = lib.pto_create(n, *_arrs(p), bucket, theta, dt_max, threads)
        super().__init__(lib, h, n)

    def set_basic_down(self, on=True):
        """Breadth-first per-bucket order (Partition::startBasicDown)."""
        self._lib.pto_set_traversal(self._h, 1 if on else 0)

    def set_periodic(self, period=1.0, n_replicas=1, rcut=2.6, hcut=2.8):
        """Periodic cube: replica walks plus the Ewald correction."""
        self._lib.pto_set_periodic(self._h, 1, period, n_replicas, rcut, hcut)

    def forces(self, record_lists=False):
        self._lib.pto_forces(self._h, 1 if record_lists else 0)

    def mono_count(self):
        """node() calls of the last pass that took the monopole fallback."""
        return int(self._lib.pto_get_mono(self._h))

    def run(self, nsteps):
        self._lib.pto_run(self._h, nsteps)

    def acc(self):
        a = [np.zeros(self.n) for _ in range(5)]
        self._lib.pto_get_acc(self._h, *a)
        return a  # ax, ay, az, pot (reference partial potential), pot_full


class RefSim(_Sim):
    """The reference's own gravity sources (oracle/_ref/libptref.so)."""
    prefix = "ptref_"

    def __init__(self, p: dict, bucket=16, theta=0.7, dt_max=0.01, group=64, threads=1):
        lib = _ref_lib()
        n = p["x"].size
        h = lib.ptref_create(n, *_arrs(p), bucket, theta, dt_max, group, threads)
        super().__init__(lib, h, n)

    def set_basic_down(self, on=True):
        """Breadth-first per-bucket order (Partition::startBasicDown)."""
        self._lib.ptref_set_traversal(self._h, 1 if on else 0)

    def set_periodic(self, period=1.0, n_replicas=1):
        """Periodic cube (the reference's fEwCut 2.6 and |h| <= 2.8)."""
        self._lib.ptref_set_periodic(self._h, 1, period, n_replicas)

    def dual(self):
        """Subtree::startDual<GravityVisitor> (one subtree): ax, ay, az and
        (P2P pairs, P2C evaluations)."""
        a = [np.zeros(self.n) for _ in range(3)]
        c = np.zeros(2, np.uint64)
        self._lib.ptref_dual(self._h, *a, c)
        return a, (int(c[0]), int(c[1]))

    def sph_density(self):
        """The reference's DensityVisitor + DensityFn (k = 32): density, ball^2,
        neighbours (caller order, sorted by (d2, index)) and their d2."""
        n, k = self.n, 32
        d, b, nd2 = np.zeros(n), np.zeros(n), np.zeros(n * k)
        nbr = np.zeros(n * k, np.int32)
        self._lib.ptref_sph_density(self._h, d, b, nbr, nd2)
        return d, b, nbr.reshape(n, k), nd2.reshape(n, k)

    def sph_pressure(self, u):
        """The reference's PressureVisitor + ForceFn + doSPHCalc after
        sph_density(): pressure accelerations and PdV work (caller order)."""
        out = [np.zeros(self.n) for _ in range(4)]
        self._lib.ptref_sph_pressure(self._h, np.ascontiguousarray(u, dtype=np.float64), *out)
        return out

    def sph_step(self, nsteps, u, u_pred, v_pred):
        """nsteps iterations of the reference's SPH example (density pass,
        pressure pass, Particle::kick / perturb with dt = dt_max): returns the
        SPH state (u, u_pred, (vpx, vpy, vpz)) in caller order; positions and
        velocities through state()."""
        st = [np.array(a, dtype=np.float64, copy=True) for a in [u, u_pred] + list(v_pred)]
        self._lib.ptref_sph_step(self._h, int(nsteps), *st)
        return st[0], st[1], tuple(st[2:])

    def forces(self, record_lists=False):
        self._lib.ptref_set_record_lists(self._h, 1 if record_lists else 0)
        self._lib.ptref_run(self._h, 0)

    def run(self, nsteps):
        self._lib.ptref_set_record_lists(self._h, 0)
        self._lib.ptref_run(self._h, nsteps)

    def acc(self):
        a = [np.zeros(self.n) for _ in range(4)]
        self._lib.ptref_get_acc(self._h, *a)
        return a  # ax, ay, az, pot (partial potential)

    def forces_sample(self, stride=0, budget_s=10.0):
        """Timed bounded sample: full build, then bucket groups until budget_s.
        Returns (build seconds, traversal seconds, traversed particle share)."""
        tb, tt, fr = C.c_double(), C.c_double(), C.c_double()
        self._lib.ptref_forces_sample(self._h, budget_s, C.byref(tb), C.byref(tt), C.byref(fr))
        return tb.value, tt.value, fr.value


def direct_sum(p: dict, targets: np.ndarray, threads: int = 1):
    """FP64 isolated spline direct sum at the given target indices."""
    lib = _port_lib()
    t = np.ascontiguousarray(targets, dtype=np.int32)
    out = [np.zeros(t.size) for _ in range(4)]
    a = _arrs(p)
    lib.pto_direct(p["x"].size, a[0], a[1], a[2], a[6], a[7], t.size, t, *out, threads)
    return out


def ewald_direct_sum(p: dict, targets: np.ndarray, period: float = 1.0, threads: int = 1):
    """FP64 periodic (Ewald) direct sum at the given target indices."""
    lib = _port_lib()
    t = np.ascontiguousarray(targets, dtype=np.int32)
    out = [np.zeros(t.size) for _ in range(4)]
    a = _arrs(p)
    lib.pto_ewald_direct(p["x"].size, a[0], a[1], a[2], a[6], a[7], period, t.size, t, *out, threads)
    return out


def sph_density(p: dict, k: int = 32, threads: int = 1):
    """Brute-force k-nearest-neighbour SPH density (the C restatement)."""
    lib = _port_lib()
    n = p["x"].size
    a = _arrs(p)
    d, b, nd2 = np.zeros(n), np.zeros(n), np.zeros(n * k)
    nbr = np.zeros(n * k, np.int32)
    lib.pto_sph_density(n, a[0], a[1], a[2], a[6], k, threads, d, b, nbr, nd2)
    return d, b, nbr.reshape(n, k), nd2.reshape(n, k)


def sph_pressure(p: dict, u, density, ballsq, nbr, nd2):
    """The SPH pressure pass (C restatement) after sph_density(): pressure
    accelerations and PdV work with the opposite reactions added."""
    lib = _port_lib()
    n, k = p["x"].size, nbr.shape[1]
    a = _arrs(p)
    out = [np.zeros(n) for _ in range(4)]
    lib.pto_sph_pressure(n, a[0], a[1], a[2], a[3], a[4], a[5], a[6], np.ascontiguousarray(u, dtype=np.float64),
                         np.ascontiguousarray(density), np.ascontiguousarray(ballsq),
                         np.ascontiguousarray(nbr, dtype=np.int32).ravel(), np.ascontiguousarray(nd2).ravel(), k, *out)
    return out


def sph_step(p: dict, nsteps: int, dt: float, u, u_pred, v_pred, threads: int = 1):
    """nsteps iterations of the SPH example on the C restatement: the density
    and pressure passes above (the pressure pass reading u_pred and v_pred as
    u_predicted and velocity_predicted), then Particle::kick and
    Particle::perturb (src/Particle.C:7-21) elementwise in FP64 with the
    reference's association.  Returns (particles, u, u_pred, (vpx, vpy, vpz))
    in caller order."""
    q = {k: np.array(v, copy=True) for k, v in p.items()}
    u = np.array(u, dtype=np.float64, copy=True)
    up = np.array(u_pred, dtype=np.float64, copy=True)
    vp = [np.array(v, dtype=np.float64, copy=True) for v in v_pred]
    for _ in range(nsteps):
        dens, ball, nbr, nd2 = sph_density(q, threads=threads)
        pv = dict(q, vx=vp[0], vy=vp[1], vz=vp[2])
        acc = sph_pressure(pv, up, dens, ball, nbr, nd2)
        for d, (xk, vk) in enumerate((("x", "vx"), ("y", "vy"), ("z", "vz"))):
            a = acc[d]
            v = q[vk] + a * dt / 2      # kick
            v = v + (a * dt / 2)         # perturb
            vp[d] = v + (a * dt)
            q[xk] = q[xk] + (v * dt)
            q[vk] = v
        u_delta = 0.5e-7 * dt
        u = u - acc[3] * u_delta
        up = u - acc[3] * u_delta
    return q, u, up, tuple(vp)


def sort_tree(t: Tree) -> Tree:
    """Canonical node order (by key) so trees from different layouts compare."""
    o = np.argsort(t.keys, kind="stable")
    return Tree(t.keys[o], t.types[o], t.depth[o], t.count[o], t.moments[o])

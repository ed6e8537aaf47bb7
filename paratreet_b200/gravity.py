"""Host-side mirror of ParaTreeT's Gravity example interface, over the C ABI.

The reference's user-facing pieces for this path and what stands in for them:

* ``GravityVisitor(offset, theta)`` (examples/GravityVisitor.h:9-31): same
  traits (CallSelfLeaf, ForceEvenDepth, TargetMustBeLeaf), same opening
  factors; here it configures the device traversal instead of being called
  per node.
* ``Configuration`` fields used by the path (src/Configuration.h:131-153:
  max_particles_per_leaf ``-l``, num_iterations ``-i``) and ExMain's
  ``theta`` / ``max_timestep`` ``-j`` (examples/Main.C:55-57, :64-78).
* ``Partition<Data>::startDown<Visitor>(Visitor)`` (src/Partition.h:129-134):
  ``GravitySimulation.start_down(visitor)`` runs one force pass.
* ``Driver<Data>::run`` (src/Driver.h:183-288): ``GravitySimulation.run``.
* ``outputParticleAccelerations`` (src/Paratreet.h:242-249):
  ``GravitySimulation.accelerations``.

All compute runs in libpt_gravity.so on the GPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L

PRECISIONS = {"fp64": L.PT_FP64, "mixed": L.PT_MIXED, "fp64_lists": L.PT_FP64_LISTS}
INTEGRATORS = {"kkd": L.PT_KKD, "kdk": L.PT_KDK}


class GravityVisitor:
    """Parameters of examples/GravityVisitor.h for the device traversal."""

    CallSelfLeaf = True
    ForceEvenDepth = True
    TargetMustBeLeaf = True
    opening_geometry_factor_squared = 4.0 / 3.0

    def __init__(self, offset=(0.0, 0.0, 0.0), theta: float = 0.7):
        if not theta > 0:
            raise ValueError("theta must be positive")
        self.offset = tuple(float(v) for v in offset)
        self.theta = float(theta)
        self.gravity_factor = self.opening_geometry_factor_squared / (self.theta * self.theta)
        self.monopole_gravity_factor = np.sqrt(self.opening_geometry_factor_squared) / self.theta ** 4


@dataclass
class Configuration:
    max_particles_per_leaf: int = 16
    theta: float = 0.7
    max_timestep: float = 1e-5
    precision: str = "fp64"
    integrator: str = "kkd"
    device: int = 0
    record_lists: bool = False
    periodic: bool = False        # Configuration::periodic
    n_replicas: int = 0           # Configuration::nReplicas
    period: float = 1.0           # Configuration::fPeriod (cubic)
    ewald_rcut: float = 2.6       # fEwCut, examples/Ewald.h:26
    ewald_hcut: float = 2.8       # dEwhCut, examples/Ewald.C:86
    traversal: str = "transposed"  # "transposed" (Partition::startDown) or "basic" (startBasicDown)


@dataclass
class TreeDump:
    keys: np.ndarray
    types: np.ndarray
    depth: np.ndarray
    count: np.ndarray
    moments: np.ndarray  # (n, 18): mass, cm3, soft, radius, xx, xy, xz, yy, yz, zz, lo3, hi3


@dataclass
class InteractionLists:
    bucket_keys: np.ndarray
    offsets: np.ndarray
    keys: np.ndarray
    kinds: np.ndarray  # 0 leaf() P2P, 1 node() P2C


_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "m", "soft")


class GravitySimulation:
    """One simulation's device state (one handle of the C ABI)."""

    def __init__(self, conf: Configuration | None = None, **kw):
        conf = conf or Configuration(**kw)
        self.conf = conf
        self._lib = L.load()
        cfg = L.PtConfig()
        self._check(self._lib.pt_config_default(C.byref(cfg)))
        cfg.theta = conf.theta
        cfg.bucket = conf.max_particles_per_leaf
        cfg.precision = PRECISIONS[conf.precision]
        cfg.integrator = INTEGRATORS[conf.integrator]
        cfg.dt_max = conf.max_timestep
        cfg.device = conf.device
        cfg.record_lists = 1 if conf.record_lists else 0
        cfg.periodic = 1 if conf.periodic else 0
        cfg.n_replicas = conf.n_replicas
        cfg.period = conf.period
        cfg.ewald_rcut = conf.ewald_rcut
        cfg.ewald_hcut = conf.ewald_hcut
        cfg.traversal = {"transposed": L.PT_TRANSPOSED_DOWN, "basic": L.PT_BASIC_DOWN}[conf.traversal]
        h = C.c_void_p()
        rc = self._lib.pt_create(C.byref(cfg), C.byref(h))
        if rc != L.PT_OK:
            raise L.PtError(rc, "pt_create failed (CUDA device or configuration)")
        self._h = h
        self.n = 0

    # -- plumbing -----------------------------------------------------------
    def _check(self, rc: int):
        if rc != L.PT_OK:
            msg = self._lib.pt_last_error(getattr(self, "_h", None)) if hasattr(self, "_h") else b""
            raise L.PtError(rc, (msg or b"").decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream_ptr: int | None):
        self._check(self._lib.pt_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def set_theta(self, theta: float):
        self._check(self._lib.pt_set_theta(self._h, theta))
        self.conf.theta = theta

    def set_precision(self, precision: str):
        self._check(self._lib.pt_set_precision(self._h, PRECISIONS[precision]))
        self.conf.precision = precision

    def set_sort_spin_limit(self, polls: int = 1 << 21):
        """Failure-path control of the key sort (tests): the polls a look-back
        makes on an unpublished tile before the pass gives up with an error."""
        self._check(self._lib.pt_set_sort_spin_limit(self._h, int(polls)))

    def set_list_region(self, entries: int = 32768):
        """Entries per warp region of the two-phase list pools (tuning and
        tests: smaller regions move the buckets' lists more often)."""
        self._check(self._lib.pt_set_list_region(self._h, int(entries)))

    # -- particles ----------------------------------------------------------
    def set_particles(self, p: dict):
        arrs = [np.ascontiguousarray(p[k], dtype=np.float64) for k in _FIELDS]
        n = arrs[0].size
        self._keep = arrs
        self._check(self._lib.pt_set_particles(self._h, n, *[L.ptr(a) for a in arrs]))
        self.n = n

    def set_particles_device(self, n: int, ptrs):
        """ptrs: 8 device pointers (x, y, z, vx, vy, vz, m, soft), FP64."""
        self._check(self._lib.pt_set_particles_device(self._h, n, *[C.c_void_p(int(q)) for q in ptrs]))
        self.n = n

    # -- force pass ---------------------------------------------------------
    def start_down(self, visitor: GravityVisitor | None = None, buckets: tuple[int, int] | None = None):
        """Partition::startDown<GravityVisitor>: one force evaluation."""
        if visitor is not None:
            if any(visitor.offset):
                raise ValueError("replica offsets are generated by the periodic configuration "
                                 "(periodic=True, n_replicas, period), as traversalFn does")
            if visitor.theta != self.conf.theta:
                self.set_theta(visitor.theta)
        if buckets is None:
            self._check(self._lib.pt_compute_forces(self._h))
        else:
            self._check(self._lib.pt_compute_forces_range(self._h, int(buckets[0]), int(buckets[1])))

    compute_forces = start_down

    def accelerations(self, out=None):
        n = self.n
        out = out or {k: np.empty(n) for k in ("ax", "ay", "az", "pot", "pot_full")}
        self._check(self._lib.pt_get_accel(self._h, *[L.ptr(out.get(k)) for k in ("ax", "ay", "az", "pot", "pot_full")]))
        return out

    def run(self, num_iterations: int):
        """Driver::run: num_iterations of forces, kick, perturb."""
        self._check(self._lib.pt_step(self._h, int(num_iterations)))

    def advance(self) -> float:
        """Kick + perturb with the accelerations now on the device (after a
        force pass, possibly summed over ranks); returns dt."""
        v = C.c_double()
        self._check(self._lib.pt_advance(self._h, C.byref(v)))
        return v.value

    def bucket_work(self):
        """P2P pairs + P2C evaluations per bucket (DFS order) of the last pass."""
        nn, nb = C.c_int64(), C.c_int64()
        self._check(self._lib.pt_get_tree_size(self._h, C.byref(nn), C.byref(nb)))
        w = np.zeros(nb.value, np.uint64)
        if nb.value:
            self._check(self._lib.pt_get_bucket_work(self._h, L.ptr(w)))
        return w

    def state(self):
        out = {k: np.empty(self.n) for k in ("x", "y", "z", "vx", "vy", "vz")}
        self._check(self._lib.pt_get_state(self._h, *[L.ptr(out[k]) for k in ("x", "y", "z", "vx", "vy", "vz")]))
        return out

    def last_dt(self) -> float:
        v = C.c_double()
        self._check(self._lib.pt_last_dt(self._h, C.byref(v)))
        return v.value

    # -- inspection ---------------------------------------------------------
    def keys(self):
        k = np.empty(self.n, np.uint64)
        self._check(self._lib.pt_get_keys(self._h, L.ptr(k)))
        return k

    def universe(self):
        lo, hi = np.empty(3), np.empty(3)
        self._check(self._lib.pt_get_universe(self._h, L.ptr(lo), L.ptr(hi)))
        return lo, hi

    def tree(self) -> TreeDump:
        nn, nb = C.c_int64(), C.c_int64()
        self._check(self._lib.pt_get_tree_size(self._h, C.byref(nn), C.byref(nb)))
        n = nn.value
        k = np.empty(n, np.uint64)
        ints = np.empty(4 * n, np.int32)
        d = np.empty(18 * n)
        self._check(self._lib.pt_get_tree(self._h, L.ptr(k), L.ptr(ints), L.ptr(d)))
        ints = ints.reshape(n, 4)
        return TreeDump(k, ints[:, 0].copy(), ints[:, 1].copy(), ints[:, 2].copy(), d.reshape(n, 18))

    def bucket_keys(self):
        nn, nb = C.c_int64(), C.c_int64()
        self._check(self._lib.pt_get_tree_size(self._h, C.byref(nn), C.byref(nb)))
        k = np.empty(nb.value, np.uint64)
        self._check(self._lib.pt_get_bucket_keys(self._h, L.ptr(k)))
        return k

    def lists(self) -> InteractionLists:
        bk = self.bucket_keys()
        tot = C.c_int64()
        self._check(self._lib.pt_get_lists_size(self._h, C.byref(tot)))
        off = np.empty(bk.size + 1, np.int64)
        keys = np.empty(max(tot.value, 1), np.uint64)
        kinds = np.empty(max(tot.value, 1), np.int32)
        self._check(self._lib.pt_get_lists(self._h, L.ptr(off), L.ptr(keys), L.ptr(kinds)))
        return InteractionLists(bk, off, keys[: tot.value], kinds[: tot.value])

    def list_digests(self, which: str = "two_phase"):
        """Per bucket (DFS order): an order-independent digest of its
        interaction list in the last pass and the list's length.  which =
        "recorded" (record_lists) or "two_phase" (the mixed form's lists)."""
        nb = self.bucket_keys().size
        dig = np.empty(max(nb, 1), np.uint64)
        cnt = np.empty(max(nb, 1), np.int64)
        self._check(self._lib.pt_get_list_digests(self._h, {"recorded": 0, "two_phase": 1}[which],
                                                   L.ptr(dig), L.ptr(cnt)))
        return dig[:nb], cnt[:nb]

    def counters(self) -> dict:
        c = L.PtCounters()
        self._check(self._lib.pt_get_counters(self._h, C.byref(c)))
        return {f: getattr(c, f) for f, _ in L.PtCounters._fields_ if f != "reserved"}

    def ewald_direct_sum(self, targets):
        """FP64 periodic (Ewald) direct sum in the configured cube at target indices."""
        t = np.ascontiguousarray(targets, dtype=np.int32)
        out = [np.empty(t.size) for _ in range(4)]
        self._check(self._lib.pt_ewald_direct_sum(self._h, t.size, L.ptr(t), *[L.ptr(o) for o in out]))
        return out

    def sph_density(self, neighbors: bool = False):
        """Density pass of the SPH example (DensityVisitor + DensityFn, k = 32):
        density and ball^2 per particle, and with neighbors=True the 32
        neighbours (caller indices, sorted by (d2, index)) and their d2."""
        n = self.n
        d, b = np.empty(n), np.empty(n)
        nbr = np.empty((n, 32), np.int32) if neighbors else None
        nd2 = np.empty((n, 32)) if neighbors else None
        self._check(self._lib.pt_sph_density(self._h, L.ptr(d), L.ptr(b), L.ptr(nbr), L.ptr(nd2)))
        return (d, b, nbr, nd2) if neighbors else (d, b)

    def sph_pressure(self, u):
        """Pressure pass of the SPH example (ForceFn + doSPHCalc after the
        density pass): (density, ax, ay, az, pdv) per particle for internal
        energies u."""
        n = self.n
        uu = np.ascontiguousarray(u, dtype=np.float64)
        if uu.shape != (n,):
            raise ValueError("u must hold one value per particle")
        out = [np.empty(n) for _ in range(5)]
        self._check(self._lib.pt_sph_pressure(self._h, L.ptr(uu), *[L.ptr(o) for o in out]))
        return tuple(out)

    def sph_run(self, iterations: int, u, u_pred=None, v_pred=None):
        """Iterations of the SPH example (density pass, pressure pass, kick and
        perturb with the internal-energy updates; dt = max_timestep).  u,
        u_pred (default u) and v_pred (3 arrays, default the current
        velocities) are the particles' SPH state in caller order; returns the
        updated (u, u_pred, (vpx, vpy, vpz)).  Positions and velocities stay in
        the simulation (state())."""
        n = self.n
        uu = np.array(u, dtype=np.float64, copy=True)
        up = uu.copy() if u_pred is None else np.array(u_pred, dtype=np.float64, copy=True)
        if v_pred is None:
            st = self.state()
            vp = [st["vx"].copy(), st["vy"].copy(), st["vz"].copy()]
        else:
            vp = [np.array(v, dtype=np.float64, copy=True) for v in v_pred]
        if any(a.shape != (n,) for a in [uu, up] + vp):
            raise ValueError("u, u_pred and each v_pred component must hold one value per particle")
        self._check(self._lib.pt_sph_step(self._h, int(iterations), L.ptr(uu), L.ptr(up), *[L.ptr(v) for v in vp]))
        return uu, up, tuple(vp)

    def direct_sum(self, targets):
        t = np.ascontiguousarray(targets, dtype=np.int32)
        out = [np.empty(t.size) for _ in range(4)]
        self._check(self._lib.pt_direct_sum(self._h, t.size, L.ptr(t), *[L.ptr(o) for o in out]))
        return out

    # -- differentiation (needs record_lists) --------------------------------
    def forces_frozen(self, x=None, y=None, z=None, m=None):
        """Re-evaluate the recorded interaction lists (FP64) with new positions /
        masses on the same tree; returns accelerations like accelerations()."""
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, m)]
        self._check(self._lib.pt_forces_frozen(self._h, *[L.ptr(a) for a in arrs]))
        return self.accelerations()

    def adjoint(self, cax, cay, caz, out=None):
        """Gradient of sum_i cot_i . a_i w.r.t. positions and masses (fixed lists);
        ``out`` may hold preallocated arrays "gx", "gy", "gz", "gm"."""
        c = [np.ascontiguousarray(a, dtype=np.float64) for a in (cax, cay, caz)]
        out = out or {k: np.empty(self.n) for k in ("gx", "gy", "gz", "gm")}
        self._check(self._lib.pt_adjoint(self._h, *[L.ptr(a) for a in c],
                                         *[L.ptr(out[k]) for k in ("gx", "gy", "gz", "gm")]))
        return out

    def chain_grad(self, nsteps: int, dt: float, targets, ckpt_every: int = 0):
        """Loss 0.5 sum |x(T) - y|^2 after nsteps KDK steps and its gradient w.r.t.
        the initial positions, velocities and masses (checkpointed adjoint)."""
        y = [np.ascontiguousarray(t, dtype=np.float64) for t in targets]
        out = [np.empty(self.n) for _ in range(7)]
        loss = C.c_double()
        self._check(self._lib.pt_chain_grad(self._h, int(nsteps), float(dt), int(ckpt_every),
                                            *[L.ptr(a) for a in y], C.byref(loss), *[L.ptr(o) for o in out]))
        keys = ("gx", "gy", "gz", "gvx", "gvy", "gvz", "gm")
        return loss.value, dict(zip(keys, out))

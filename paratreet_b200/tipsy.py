"""Tipsy particle files and the ``.acc`` acceleration output of the Gravity
example: host-side I/O that feeds the device path and reads its results back.

Mirrors
  * ``Reader::load`` (src/Reader.C:11-107): header (time, nbodies, ndim, nsph,
    ndark, nstar), then gas, dark and star records in that order; softening
    from gas ``hsmooth`` and dark ``eps``, zero for stars (the reference leaves
    star softening unset); ``order`` = position in the file;
  * ``Reader::setSoft`` (src/Reader.C:110-116): one softening for every
    particle when the configuration gives ``dSoft``;
  * ``TipsyWriter::do_write`` (src/Writer.C:87-159): standard (big-endian)
    Tipsy with FP64 positions and velocities when ``Real`` is double, only
    mass, position and velocity filled, particles in ``order``;
  * ``Writer::do_write`` (src/Writer.C:31-72): ``<name>.acc`` = N, then all x,
    all y, all z accelerations, one ``%.14g`` value per line.

Record layouts (standard Tipsy, big-endian; P = position type, V = velocity
type, each float32 or float64; the rest float32):
  header 32 B: f64 time, i32 nbodies, ndim, nsph, ndark, nstar, pad
  gas:  mass, pos[3]:P, vel[3]:V, rho, temp, hsmooth, metals, phi
  dark: mass, pos[3]:P, vel[3]:V, eps, phi
  star: mass, pos[3]:P, vel[3]:V, metals, tform, eps, phi
The reader detects byte order from the header's counts and the position /
velocity widths from the file size, as the reference's Tipsy reader accepts
both native and standard files."""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

HEADER_BYTES = 32
_GAS_TAIL = ("rho", "temp", "hsmooth", "metals", "phi")
_DARK_TAIL = ("eps", "phi")
_STAR_TAIL = ("metals", "tform", "eps", "phi")


@dataclass
class TipsyHeader:
    time: float
    nbodies: int
    ndim: int
    nsph: int
    ndark: int
    nstar: int


def _dtype(kind: str, endian: str, pos: str, vel: str) -> np.dtype:
    tail = {"gas": _GAS_TAIL, "dark": _DARK_TAIL, "star": _STAR_TAIL}[kind]
    f32 = endian + "f4"
    fields = [("mass", f32), ("pos", endian + pos, (3,)), ("vel", endian + vel, (3,))]
    fields += [(t, f32) for t in tail]
    return np.dtype(fields)


def _record_bytes(h: TipsyHeader, pos: str, vel: str) -> int:
    return sum(cnt * _dtype(k, ">", pos, vel).itemsize
               for k, cnt in (("gas", h.nsph), ("dark", h.ndark), ("star", h.nstar)))


def read_header(buf: bytes) -> tuple[TipsyHeader, str]:
    """Header and byte order ('>' standard, '<' native little-endian)."""
    if len(buf) < HEADER_BYTES:
        raise ValueError("not a Tipsy file: shorter than its 32-byte header")
    for endian in (">", "<"):
        t = np.frombuffer(buf[:8], dtype=endian + "f8")[0]
        nb, nd, ns, ndk, nst = np.frombuffer(buf[8:28], dtype=endian + "i4")
        if nb >= 0 and min(ns, ndk, nst) >= 0 and nb == ns + ndk + nst and nd in (1, 2, 3):
            return TipsyHeader(float(t), int(nb), int(nd), int(ns), int(ndk), int(nst)), endian
    raise ValueError("not a Tipsy file: header counts are inconsistent in either byte order")


def read_tipsy(path: str, soft: float | None = None) -> tuple[dict, TipsyHeader]:
    """Particles of a Tipsy file as FP64 SoA (x y z vx vy vz m soft, plus
    ``type``: 0 gas, 1 dark, 2 star, and ``order``) and its header.  ``soft``
    replaces every softening (Reader::setSoft)."""
    with open(path, "rb") as f:
        buf = f.read()
    h, endian = read_header(buf)
    body = len(buf) - HEADER_BYTES
    for pos, vel in (("f4", "f4"), ("f8", "f4"), ("f8", "f8")):
        if _record_bytes(h, pos, vel) == body:
            break
    else:
        raise ValueError("Tipsy file size matches neither float nor double positions / velocities")
    off = HEADER_BYTES
    parts = []
    for kind, cnt in (("gas", h.nsph), ("dark", h.ndark), ("star", h.nstar)):
        dt = _dtype(kind, endian, pos, vel)
        rec = np.frombuffer(buf, dtype=dt, count=cnt, offset=off)
        off += cnt * dt.itemsize
        parts.append((kind, rec))
    n = h.nbodies
    out = {k: np.empty(n) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "soft")}
    out["type"] = np.empty(n, np.int8)
    i = 0
    for t, (kind, rec) in enumerate(parts):
        c = rec.shape[0]
        sl = slice(i, i + c)
        out["m"][sl] = rec["mass"]
        for d, ax in enumerate("xyz"):
            out[ax][sl] = rec["pos"][:, d]
            out["v" + ax][sl] = rec["vel"][:, d]
        if kind == "gas":
            out["soft"][sl] = rec["hsmooth"]
        elif kind == "dark":
            out["soft"][sl] = rec["eps"]
        else:
            out["soft"][sl] = 0.0
        out["type"][sl] = t
        i += c
    out["order"] = np.arange(n, dtype=np.int64)
    if soft is not None:
        out["soft"][:] = soft
    return out, h


def write_tipsy(path: str, p: dict, time: float = 0.0, double: bool = True, softening: bool = False) -> None:
    """Standard (big-endian) Tipsy in ``order``: gas, dark, star by
    ``p["type"]`` (all dark when absent).  Like TipsyWriter, only mass,
    position and velocity are written unless ``softening`` also stores the
    softening as gas ``hsmooth`` / dark and star ``eps``."""
    n = p["x"].size
    typ = np.asarray(p.get("type", np.ones(n, np.int8)))
    order = np.argsort(np.asarray(p.get("order", np.arange(n))), kind="stable")
    pos = vel = "f8" if double else "f4"
    counts = [int(np.count_nonzero(typ == t)) for t in (0, 1, 2)]
    hdr = bytearray(HEADER_BYTES)
    hdr[:8] = np.array([time], ">f8").tobytes()
    hdr[8:28] = np.array([n, 3, counts[0], counts[1], counts[2]], ">i4").tobytes()
    chunks = [bytes(hdr)]
    for t, kind in enumerate(("gas", "dark", "star")):
        idx = order[typ[order] == t]
        rec = np.zeros(idx.size, dtype=_dtype(kind, ">", pos, vel))
        rec["mass"] = p["m"][idx]
        rec["pos"] = np.stack([p[a][idx] for a in "xyz"], 1)
        rec["vel"] = np.stack([p["v" + a][idx] for a in "xyz"], 1)
        if softening:
            rec["hsmooth" if kind == "gas" else "eps"] = p["soft"][idx]
        chunks.append(rec.tobytes())
    with open(path, "wb") as f:
        for c in chunks:
            f.write(c)


def write_acc(path: str, ax, ay, az) -> None:
    """``.acc`` output of the Gravity example's ``-v`` option: N, then the x,
    y and z blocks, ``%.14g`` per line, in particle order."""
    ax, ay, az = (np.asarray(a, dtype=np.float64) for a in (ax, ay, az))
    with open(path, "w") as f:
        f.write("%d\n" % ax.size)
        for block in (ax, ay, az):
            f.write("".join("%.14g\n" % v for v in block))


def read_acc(path: str) -> np.ndarray:
    """Accelerations of an ``.acc`` file as a (3, N) array."""
    v = np.loadtxt(path)
    n = int(v[0])
    if v.size != 1 + 3 * n:
        raise ValueError(f"{os.path.basename(path)}: expected {1 + 3 * n} values, found {v.size}")
    return v[1:].reshape(3, n)

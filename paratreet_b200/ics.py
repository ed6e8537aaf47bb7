"""Seeded synthetic initial conditions for the Barnes-Hut gravity workloads.

These stand in for the Tipsy inputs the reference reads (src/Reader.C:11-107):
every generator returns FP64 structure-of-arrays particle data
``{x, y, z, vx, vy, vz, m, soft}`` in the input ("order") numbering.  The
random stream is numpy's PCG64 ``default_rng(seed)``; draws are made in fixed
batches so the same seed always gives the same particles.

Workloads (sizes as used by the tests and the benchmark):

* ``plummer``   -- Plummer sphere, a=1, radii a/sqrt(X^(-2/3)-1) rejecting
  r > 10a, isotropic directions, velocities by Aarseth rejection sampling of
  q with g(q)=q^2(1-q^2)^(7/2), v = q*sqrt(2)*(1+r^2)^(-1/4).
* ``mixture``   -- half uniform in [0,1)^3, half in 32 equal Plummer clumps
  (scale radius 0.01, centres uniform in the cube), zero velocities.
* ``hernquist`` -- Hernquist halo r = a*sqrt(X)/(1-sqrt(X)) truncated at 20a,
  isotropic, zero velocities.
* ``lattice``   -- n^3 lattice in a periodic box displaced by a curl-free
  Gaussian random field with P(k) ~ k^-2, cut at the Nyquist wavenumber.

All masses are equal and sum to 1 (G = 1).
"""
from __future__ import annotations

import numpy as np

_BATCH = 1 << 16


def _isotropic(rng: np.random.Generator, n: int):
    cz = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    sz = np.sqrt(1.0 - cz * cz)
    return sz * np.cos(phi), sz * np.sin(phi), cz


def _plummer_radii(rng: np.random.Generator, n: int, a: float, rmax: float) -> np.ndarray:
    out = np.empty(n)
    k = 0
    while k < n:
        x = rng.uniform(0.0, 1.0, _BATCH)
        with np.errstate(divide="ignore", invalid="ignore"):
            r = a / np.sqrt(x ** (-2.0 / 3.0) - 1.0)
        r = r[np.isfinite(r) & (r <= rmax * a) & (x > 0.0)]
        take = min(n - k, r.size)
        out[k:k + take] = r[:take]
        k += take
    return out


def _aarseth_q(rng: np.random.Generator, n: int) -> np.ndarray:
    out = np.empty(n)
    k = 0
    while k < n:
        q = rng.uniform(0.0, 1.0, _BATCH)
        y = rng.uniform(0.0, 0.1, _BATCH)
        q = q[y < q * q * (1.0 - q * q) ** 3.5]
        take = min(n - k, q.size)
        out[k:k + take] = q[:take]
        k += take
    return out


def _pack(x, y, z, vx, vy, vz, soft):
    n = x.size
    return {
        "x": np.ascontiguousarray(x, dtype=np.float64),
        "y": np.ascontiguousarray(y, dtype=np.float64),
        "z": np.ascontiguousarray(z, dtype=np.float64),
        "vx": np.ascontiguousarray(vx, dtype=np.float64),
        "vy": np.ascontiguousarray(vy, dtype=np.float64),
        "vz": np.ascontiguousarray(vz, dtype=np.float64),
        "m": np.full(n, 1.0 / n),
        "soft": np.full(n, float(soft)),
    }


def plummer(n: int, seed: int = 42, a: float = 1.0, rmax: float = 10.0, soft: float = 0.01,
            velocities: bool = True):
    rng = np.random.default_rng(seed)
    r = _plummer_radii(rng, n, a, rmax)
    ux, uy, uz = _isotropic(rng, n)
    if velocities:
        q = _aarseth_q(rng, n)
        v = q * np.sqrt(2.0) * (1.0 + r * r) ** (-0.25)
        wx, wy, wz = _isotropic(rng, n)
        vx, vy, vz = v * wx, v * wy, v * wz
    else:
        vx = vy = vz = np.zeros(n)
    return _pack(r * ux, r * uy, r * uz, vx, vy, vz, soft)


def mixture(n: int, seed: int = 7, n_clumps: int = 32, clump_a: float = 0.01, soft: float = 1e-4):
    rng = np.random.default_rng(seed)
    n_uni = n // 2
    n_clump_total = n - n_uni
    per = n_clump_total // n_clumps
    counts = np.full(n_clumps, per)
    counts[: n_clump_total - per * n_clumps] += 1
    uni = rng.uniform(0.0, 1.0, (n_uni, 3))
    centres = rng.uniform(0.0, 1.0, (n_clumps, 3))
    parts = [uni]
    for c in range(n_clumps):
        k = int(counts[c])
        r = _plummer_radii(rng, k, clump_a, 10.0)
        ux, uy, uz = _isotropic(rng, k)
        parts.append(np.stack([centres[c, 0] + r * ux, centres[c, 1] + r * uy,
                               centres[c, 2] + r * uz], axis=1))
    p = np.concatenate(parts, axis=0)
    z = np.zeros(n)
    return _pack(p[:, 0], p[:, 1], p[:, 2], z, z, z, soft)


def hernquist(n: int, seed: int = 3, a: float = 1.0, rmax: float = 20.0, soft: float = 0.01):
    rng = np.random.default_rng(seed)
    out = np.empty(n)
    k = 0
    while k < n:
        s = np.sqrt(rng.uniform(0.0, 1.0, _BATCH))
        with np.errstate(divide="ignore"):
            r = a * s / (1.0 - s)
        r = r[np.isfinite(r) & (r <= rmax * a)]
        take = min(n - k, r.size)
        out[k:k + take] = r[:take]
        k += take
    ux, uy, uz = _isotropic(rng, n)
    z = np.zeros(n)
    return _pack(out * ux, out * uy, out * uz, z, z, z, soft)


def perturbed_targets(ics: dict, seed: int = 3, sigma: float = 1e-3):
    """Target positions y_i = x_i + N(0, sigma) for the adjoint loss."""
    rng = np.random.default_rng(seed + 1000003)
    n = ics["x"].size
    d = rng.normal(0.0, sigma, (3, n))
    return ics["x"] + d[0], ics["y"] + d[1], ics["z"] + d[2]


def lattice(ngrid: int = 256, seed: int = 11, box: float = 1.0, rms_cells: float = 0.25,
            soft_cells: float = 0.5):
    """Displaced lattice in a periodic box (positions wrapped into [0, box))."""
    rng = np.random.default_rng(seed)
    k1 = np.fft.fftfreq(ngrid) * ngrid
    k1z = np.fft.rfftfreq(ngrid) * ngrid
    kx, ky, kz = np.meshgrid(k1, k1, k1z, indexing="ij")
    k2 = kx * kx + ky * ky + kz * kz
    nyq = ngrid // 2
    keep = (np.abs(kx) < nyq) & (np.abs(ky) < nyq) & (kz < nyq) & (k2 > 0)
    white = rng.normal(size=(ngrid, ngrid, ngrid))
    wk = np.fft.rfftn(white)
    with np.errstate(divide="ignore", invalid="ignore"):
        amp = np.where(keep, 1.0 / k2, 0.0)  # |psi(k)|^2 ~ k^2 / k^4 = k^-2
    disp = []
    for kk in (kx, ky, kz):
        comp = np.fft.irfftn(1j * kk * amp * wk, s=(ngrid, ngrid, ngrid), axes=(0, 1, 2))
        disp.append(comp)
    disp = np.stack(disp)
    rms = np.sqrt(np.mean(np.sum(disp * disp, axis=0)))
    cell = box / ngrid
    disp *= rms_cells * cell / rms
    g = (np.arange(ngrid) + 0.5) * cell
    gx, gy, gz = np.meshgrid(g, g, g, indexing="ij")
    x = np.mod(gx + disp[0], box).ravel()
    y = np.mod(gy + disp[1], box).ravel()
    z = np.mod(gz + disp[2], box).ravel()
    n = x.size
    zz = np.zeros(n)
    return _pack(x, y, z, zz, zz, zz, soft_cells * cell)


WORKLOADS = {
    "plummer": plummer,
    "mixture": mixture,
    "hernquist": hernquist,
}

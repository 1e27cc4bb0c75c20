"""Seeded synthetic inputs shared by the tests and the benchmark.

There is no public dataset on this path: the reference is driven by models and
wavelets its users supply.  These generators produce the workloads' shapes
and value distributions (layered velocities with smooth perturbations, Gardner
density, Ricker wavelets, surface receiver lines) from numpy seeds.
"""
from __future__ import annotations

import numpy as np


def ricker(nt: int, dt: float, f0: float, dtype=np.float32) -> np.ndarray:
    """(1 - 2a) exp(-a), a = (pi f0 (t - t0))^2, t0 = 1.2 / f0."""
    t = np.arange(nt) * dt - 1.2 / f0
    a = (np.pi * f0 * t) ** 2
    return ((1 - 2 * a) * np.exp(-a)).astype(dtype)


def gardner(vp: np.ndarray) -> np.ndarray:
    return (310.0 * vp.astype(np.float64) ** 0.25).astype(vp.dtype)


def _smooth_noise(rng, nz, nx, sigma_cells):
    f = rng.standard_normal((nz, nx))
    # separable Gaussian smoothing in the Fourier domain
    kz = np.fft.fftfreq(nz)[:, None]
    kx = np.fft.fftfreq(nx)[None, :]
    g = np.exp(-2 * (np.pi * sigma_cells) ** 2 * (kz ** 2 + kx ** 2))
    s = np.real(np.fft.ifft2(np.fft.fft2(f) * g))
    return s / (np.abs(s).max() + 1e-30)


def layered_vp(nx: int, nz: int, dx: float, vmin=1500.0, vmax=4500.0, nlayers=6, pert=0.05, sigma_m=150.0,
               seed=1, vclip=None, dtype=np.float32) -> np.ndarray:
    """Flat layers vmin..vmax plus a smooth seeded Gaussian perturbation (fraction `pert`)."""
    rng = np.random.default_rng(seed)
    edges = np.linspace(0, nz, nlayers + 1).astype(int)
    vp = np.empty((nz, nx))
    for k in range(nlayers):
        vp[edges[k]:edges[k + 1], :] = vmin + (vmax - vmin) * k / max(1, nlayers - 1)
    vp *= 1.0 + pert * _smooth_noise(rng, nz, nx, sigma_m / dx)
    if vclip is not None:
        vp = np.minimum(vp, vclip)
    return vp.astype(dtype)


def elastic_model(nx: int, nz: int, dx: float, seed=2, vclip=4450.0, nlenses=6, dtype=np.float32):
    """Layered vp (<= vclip), vp/vs in [1.7, 2.0], Gardner density, random elliptical lenses."""
    rng = np.random.default_rng(seed)
    vp = layered_vp(nx, nz, dx, 1500.0, 4400.0, 6, 0.03, 100.0, seed, None, np.float64)
    zz, xx = np.mgrid[0:nz, 0:nx]
    for _ in range(nlenses):
        cx, cz = rng.uniform(0.1, 0.9) * nx, rng.uniform(0.2, 0.9) * nz
        ax, az = rng.uniform(0.03, 0.12) * nx, rng.uniform(0.02, 0.08) * nz
        m = ((xx - cx) / ax) ** 2 + ((zz - cz) / az) ** 2 < 1
        vp[m] *= rng.uniform(0.9, 1.1)
    vp = np.minimum(vp, vclip)
    ratio = 1.7 + 0.3 * (0.5 + 0.5 * _smooth_noise(rng, nz, nx, 20))
    vs = vp / ratio
    rho = 310.0 * vp ** 0.25
    return vp.astype(dtype), vs.astype(dtype), rho.astype(dtype)


def surface_line(n: int, x0: float, dxr: float, z: float) -> np.ndarray:
    """n positions (x, z) starting at x0 with spacing dxr at depth z."""
    return np.stack([x0 + dxr * np.arange(n), np.full(n, z)], axis=1)


def _gauss_smooth(a: np.ndarray, sigma_cells: float) -> np.ndarray:
    """Gaussian smoothing with reflected edges (Fourier domain on the mirrored array)."""
    nz, nx = a.shape
    m = np.concatenate([a, a[::-1]], axis=0)
    m = np.concatenate([m, m[:, ::-1]], axis=1)
    kz = np.fft.fftfreq(2 * nz)[:, None]
    kx = np.fft.fftfreq(2 * nx)[None, :]
    g = np.exp(-2 * (np.pi * sigma_cells) ** 2 * (kz ** 2 + kx ** 2))
    return np.real(np.fft.ifft2(np.fft.fft2(m) * g))[:nz, :nx]


def fwi_models(nx: int, nz: int, dx: float, seed=4, nanom=8, amp=0.08, smooth_m=200.0, vmin=1500.0, vmax=3500.0,
               dtype=np.float32):
    """True model = smooth depth-increasing background + `nanom` Gaussian anomalies of
    +-amp (seeded); starting model = the true model smoothed with sigma = smooth_m.
    Returns (vp_true, vp_start); density follows Gardner's relation in both."""
    rng = np.random.default_rng(seed)
    z = np.arange(nz)[:, None] / max(1, nz - 1)
    bg = vmin + (vmax - vmin) * z * np.ones((1, nx))
    zz, xx = np.mgrid[0:nz, 0:nx]
    pert = np.zeros((nz, nx))
    for _ in range(nanom):
        cx, cz = rng.uniform(0.1, 0.9) * nx, rng.uniform(0.2, 0.85) * nz
        r = rng.uniform(0.03, 0.08) * min(nx, 3 * nz)
        pert += rng.choice([-1.0, 1.0]) * amp * np.exp(-(((xx - cx) ** 2 + (zz - cz) ** 2) / (2 * r * r)))
    vt = bg * (1.0 + pert)
    vs = _gauss_smooth(vt, smooth_m / dx)
    return vt.astype(dtype), vs.astype(dtype)


def dipping_vp_3d(nx: int, ny: int, nz: int, dx: float, seed=5, vmin=1500.0, vmax=5000.0, ninterfaces=3,
                  vclip=None, dtype=np.float32) -> np.ndarray:
    """Layered 3D velocity [nz][ny][nx]: ninterfaces planar interfaces with seeded
    dips, velocity stepping from vmin to vmax across them (clipped at vclip)."""
    rng = np.random.default_rng(seed)
    z = np.arange(nz)[:, None, None] * dx
    y = np.arange(ny)[None, :, None] * dx
    x = np.arange(nx)[None, None, :] * dx
    depth = nz * dx
    layer = np.zeros((nz, ny, nx), np.int32)
    for k in range(ninterfaces):
        z0 = depth * (k + 1) / (ninterfaces + 1)
        gx, gy = rng.uniform(-0.15, 0.15, 2)
        layer += (z > z0 + gx * (x - nx * dx / 2) + gy * (y - ny * dx / 2)).astype(np.int32)
    vp = vmin + (vmax - vmin) * layer / ninterfaces
    if vclip is not None:
        vp = np.minimum(vp, vclip)
    return vp.astype(dtype)


def elastic_blobs_3d(nx: int, ny: int, nz: int, dx: float, seed=7, vmin=1800.0, vmax=4000.0, nlayers=4, nblobs=12,
                     blobs=True, dtype=np.float32):
    """Elastic 3D model [nz][ny][nx]: flat layers from vmin to vmax, optionally with
    nblobs seeded Gaussian blobs of +-8 % vp; vp/vs drawn per layer in [1.7, 2.0];
    Gardner density.  Returns vp, vs, rho."""
    rng = np.random.default_rng(seed)
    z = np.arange(nz, dtype=np.float32) * dx
    edges = np.sort(rng.uniform(0.1, 0.9, nlayers - 1)) * nz * dx
    layer = np.searchsorted(edges, z)
    v1 = (vmin + (vmax - vmin) * layer / max(1, nlayers - 1)).astype(np.float32)
    ratio = rng.uniform(1.7, 2.0, nlayers).astype(np.float32)[layer]
    vp = np.broadcast_to(v1[:, None, None], (nz, ny, nx)).copy()
    vsr = np.broadcast_to(ratio[:, None, None], (nz, ny, nx))
    centres = rng.uniform(0.15, 0.85, (nblobs, 3)) * np.array([nz, ny, nx])
    radii = rng.uniform(0.04, 0.1, nblobs) * min(nx, ny, nz)
    amps = rng.uniform(-0.08, 0.08, nblobs)
    if blobs:
        iz, iy, ix = (np.arange(n, dtype=np.float32) for n in (nz, ny, nx))
        for (cz, cy, cx), r, a in zip(centres, radii, amps):
            g = (np.exp(-((iz - cz) / r) ** 2)[:, None, None] * np.exp(-((iy - cy) / r) ** 2)[None, :, None] *
                 np.exp(-((ix - cx) / r) ** 2)[None, None, :])
            vp *= (1.0 + a * g).astype(np.float32)
    vp = np.minimum(vp, vmax).astype(dtype)
    vs = (vp / vsr).astype(dtype)
    return vp, vs, gardner(vp).astype(dtype)

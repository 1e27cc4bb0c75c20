"""The synthetic workloads the benchmark and the full-size parity tests share.

Each function returns plain numpy inputs (models, source and receiver
coordinates, wavelets) for one of the benchmark configurations, seeded so that
the GPU runs, the reference runs that produced the committed digests and the
benchmark all see identical inputs:

  acoustic2d_c1   acoustic 2D forward, one shot, 501 x 301, dx = 10 m, 20-cell
                  C-PML, order 8, dt = 1 ms, nt = 2000; six flat layers
                  1500 -> 4500 m/s with a 5 % smooth perturbation, clipped at
                  4450 m/s (the reference's stability guard,
                  ModellingAcoustic2D::checkStability, lib/modelling.cpp:181-194);
                  10 Hz Ricker at z = 20 m, x = 2500 m; 251 receivers every 20 m.
  elastic2d_c2    elastic 2D forward, 16 shots, 801 x 401, dx = 5 m, 30-cell
                  C-PML, dt = 0.5 ms, nt = 4000; layered vp <= 4450 with lenses,
                  vp/vs 1.7-2.0, Gardner density; explosive source at z = 10 m,
                  400 Vx receivers every 10 m.
  fwi_c3          acoustic 2D FWI gradient, 64 shots, 601 x 201, dx = 10 m,
                  20-cell C-PML, dt = 1 ms, nt = 3000, Revolve with 50
                  snapshots; true model = smooth background + 8 anomalies,
                  starting model = the true model smoothed.
  elastic3d_c5    elastic 3D FWI gradient, 16 shots, 256^3, dx = 10 m, 20-cell
                  C-PML, dt = 0.8 ms, nt = 2000; four flat layers 1800 -> 4000
                  m/s with vp/vs 1.7-2.0 per layer and Gardner density; true
                  model = layers + 12 Gaussian blobs of +-8 % vp (seed 7),
                  starting model = the layers 4 % slower (vp and vs); explosive
                  sources on a 4 x 4 grid
                  at z = 20 m; 20 x 20 receivers (Ux, Uy, Uz) every 120 m at
                  z = 10 m.
"""
from __future__ import annotations

import numpy as np

from . import synth

C1 = dict(nx=501, nz=301, dx=10.0, lpml=20, order=8, dt=1e-3, nt=2000, f0=10.0, sx=2500.0, sz=20.0, nrec=251,
          drec=20.0, vclip=4450.0)
C2 = dict(nx=801, nz=401, dx=5.0, lpml=30, order=8, dt=5e-4, nt=4000, nshots=16, nrec=400, drec=10.0, f0=15.0,
          sz=10.0)
C3 = dict(nx=601, nz=201, dx=10.0, lpml=20, order=8, nt=3000, dt=1e-3, nshots=64, ncheck=50, f0=10.0, sz=20.0,
          nrec=601)
C5 = dict(nx=256, ny=256, nz=256, dx=10.0, lpml=20, order=8, dt=8e-4, nt=2000, nshots=16, f0=10.0, sz=20.0,
          nrec_side=20, drec=120.0, rz=10.0)


def acoustic2d_c1(nt=None):
    """vp, rho [nz][nx], source (x, z) [1][2], wavelet [1][nt], receivers [nrec][2]."""
    c = C1
    nt = nt or c["nt"]
    vp = synth.layered_vp(c["nx"], c["nz"], c["dx"], 1500.0, 4500.0, 6, 0.05, 150.0, seed=1, vclip=c["vclip"])
    rho = synth.gardner(vp)
    src = np.array([[c["sx"], c["sz"]]])
    wav = synth.ricker(nt, c["dt"], c["f0"])[None, :]
    rec = synth.surface_line(c["nrec"], 0.0, c["drec"], 0.0)
    return vp, rho, src, wav, rec


def elastic2d_c2(nt=None):
    """vp, vs, rho [nz][nx], source x positions [nshots], wavelet [nt], receivers [nrec][2]."""
    c = C2
    nt = nt or c["nt"]
    vp, vs, rho = synth.elastic_model(c["nx"], c["nz"], c["dx"], seed=2)
    sx = np.sort(np.random.default_rng(3).uniform(200.0, (c["nx"] - 1) * c["dx"] - 200.0, c["nshots"]))
    wav = synth.ricker(nt, c["dt"], c["f0"])
    rec = synth.surface_line(c["nrec"], 0.0, c["drec"], 0.0)
    return vp, vs, rho, sx, wav, rec


def fwi_c3(nt=None):
    """vp_true, vp_start [nz][nx], source x positions [nshots], wavelet [nt], receivers [nrec][2]."""
    c = C3
    nt = nt or c["nt"]
    vt, vs = synth.fwi_models(c["nx"], c["nz"], c["dx"])
    sx = np.linspace(60.0, (c["nx"] - 1) * c["dx"] - 60.0, c["nshots"])
    wav = synth.ricker(nt, c["dt"], c["f0"])
    rec = synth.surface_line(c["nrec"], 0.0, c["dx"], 0.0)
    return vt, vs, sx, wav, rec


def elastic3d_c5(nt=None, true_model=False):
    """vp, vs, rho [nz][ny][nx] (starting model, or the true one), sources [nshots][3],
    wavelet [nt], receivers [nrec][3]."""
    c = C5
    nt = nt or c["nt"]
    vp, vs, rho = synth.elastic_blobs_3d(c["nx"], c["ny"], c["nz"], c["dx"], seed=7, blobs=true_model)
    if not true_model:
        vp *= np.float32(0.96)
        vs *= np.float32(0.96)
    ext = (c["nx"] - 1) * c["dx"]
    g = np.linspace(0.2, 0.8, 4) * ext
    src = np.array([[x, y, c["sz"]] for y in g for x in g]) + np.random.default_rng(8).uniform(-40, 40, (16, 3)) * \
        np.array([1.0, 1.0, 0.0])
    r1 = (ext - (c["nrec_side"] - 1) * c["drec"]) / 2 + np.arange(c["nrec_side"]) * c["drec"]
    rec = np.array([[x, y, c["rz"]] for y in r1 for x in r1])
    wav = synth.ricker(nt, c["dt"], c["f0"])
    return vp, vs, rho, src, wav, rec


def digest(a: np.ndarray) -> str:
    """SHA-256 of an array's bytes in C order (the bit pattern, not the values)."""
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()

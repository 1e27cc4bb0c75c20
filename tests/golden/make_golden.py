"""Generate the golden fixtures of the propagation path from the reference library itself.

Run where the reference sources are present (the reference library is built
from them into oracle/_ref by `make -C oracle ref`):

    python tests/golden/make_golden.py

Every array in reference.npz is an output of the unmodified reference code
(oracle/_ref/librsref.so driving Der, Pml, Model*::staggerModels,
Data2D::makeMap, Revolve, ModellingAcoustic2D/ModellingElastic2D::run,
FwiAcoustic2D::run_optimal and RtmAcoustic2D::run_optimal) on seeded inputs
from rockseis_b200.synth, together with those inputs.  The CPU tests check the
C restatement (oracle/rs_oracle.c) and this library's host preprocessing
against these arrays, so they run without the reference tree.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import api  # noqa: E402
from rockseis_b200 import synth  # noqa: E402

PRESSURE, VX, VZ = 0, 1, 3
OUT = os.path.join(HERE, "reference.npz")


def grid(nx, nz, lpml, dx, dz, dt, nt, order=8, fs=0, ox=0.0, oz=0.0):
    return api.RefGrid(nx, 1, nz, lpml, order, fs, dx, 1.0, dz, ox, 0.0, oz, dt, nt)


def der_cases(g):
    rng = np.random.default_rng(11)
    nx, nz = 29, 23
    f = rng.standard_normal((nz, nx)).astype(np.float32)
    g["der_in"] = f
    g["der_dx_dz"] = np.array([7.5, 5.0])
    out = np.zeros((8, 4, nz, nx), np.float32)
    for order in range(1, 9):
        for k, which in enumerate((0, 2, 3, 5)):
            api.ref().ref_der_f(nx, 1, nz, 7.5, 1.0, 5.0, order, which, f.ctypes.data, out[order - 1, k].ctypes.data)
    g["der_out"] = out          # [order-1][ddx_fw, ddz_fw, ddx_bw, ddz_bw]


def pml_cases(g):
    for lpml, dt in ((10, 1e-3), (30, 5e-4)):
        t = np.zeros(12 * lpml, np.float32)
        api.ref().ref_pml_tables_f(lpml, dt, t.ctypes.data)
        g[f"pml_{lpml}"] = t
        g[f"pml_{lpml}_dt"] = np.array([dt])


def stagger_cases(g):
    nx, nz, lpml = 17, 13, 5
    vp = synth.layered_vp(nx, nz, 10.0, 1500, 3500, 3, 0.05, 50, 4)
    vs = (vp / 1.8).astype(np.float32)
    rho = synth.gardner(vp)
    g["stag_vp"], g["stag_vs"], g["stag_rho"] = vp, vs, rho
    n = (nx + 2 * lpml) * (nz + 2 * lpml)
    for fs in (0, 1):
        rg = grid(nx, nz, lpml, 10.0, 10.0, 1e-3, 10, fs=fs)
        a = np.zeros((3, n), np.float32)
        api.ref().ref_stagger_a2d_f(C.byref(rg), vp.ctypes.data, rho.ctypes.data, *[a[i].ctypes.data for i in range(3)])
        e = np.zeros((5, n), np.float32)
        api.ref().ref_stagger_e2d_f(C.byref(rg), vp.ctypes.data, vs.ctypes.data, rho.ctypes.data,
                                    *[e[i].ctypes.data for i in range(5)])
        g[f"stag_a2d_fs{fs}"] = a.reshape(3, nz + 2 * lpml, nx + 2 * lpml)
        g[f"stag_e2d_fs{fs}"] = e.reshape(5, nz + 2 * lpml, nx + 2 * lpml)


def makemap_cases(g):
    nx, nz, lpml, dx, dz, ox, oz = 41, 31, 8, 10.0, 7.5, -100.0, 20.0
    rng = np.random.default_rng(5)
    coords = np.stack([rng.uniform(ox - 30, ox + (nx - 1) * dx + 30, 40),
                       rng.uniform(oz - 20, oz + (nz - 1) * dz + 20, 40)], 1)
    coords = coords.astype(np.float32).astype(np.float64)    # the reference holds T-typed coordinates
    g["map_coords"] = coords
    g["map_grid"] = np.array([nx, nz, lpml, dx, dz, ox, oz])
    rg = grid(nx, nz, lpml, dx, dz, 1e-3, 10, ox=ox, oz=oz)
    for which in (0, 1):
        for field in (PRESSURE, VX, VZ):
            mp = np.zeros((40, 2), np.int32)
            sh = np.zeros((40, 2), np.float32)
            api.ref().ref_makemap2d_field_f(C.byref(rg), 40, coords.ctypes.data, which, field, mp.ctypes.data,
                                            sh.ctypes.data)
            g[f"map_w{which}_f{field}"], g[f"shift_w{which}_f{field}"] = mp, sh


def revolve_cases(g):
    pairs = [(10, 3), (50, 5), (123, 7), (200, 10), (31, 31), (64, 2)]
    g["rev_pairs"] = np.array(pairs, np.int32)
    for nt, nc in pairs:
        a, c, k = api.ref_revolve_trace(nt, nc)
        g[f"rev_{nt}_{nc}"] = np.stack([a, c, k])
        g[f"rev_numforw_{nt}_{nc}"] = np.array([api.ref().ref_revolve_numforw(nt, nc)])


# ---------------------------------------------------------------- shot-level cases
SHOT = dict(nx=41, nz=31, lpml=8, dx=10.0, dt=1e-3, nt=150, order=8)


def shot_inputs(seed, elastic):
    s = SHOT
    vp = synth.layered_vp(s["nx"], s["nz"], s["dx"], 1500, 3000, 3, 0.05, 60, seed)
    rho = synth.gardner(vp)
    vs = (vp / 1.8).astype(np.float32) if elastic else None
    sc = np.array([[203.3, 31.7]], np.float64)
    gc = synth.surface_line(12, 15.2, 30.0, 12.4).astype(np.float32).astype(np.float64)
    wav = synth.ricker(s["nt"], s["dt"], 20.0)[None, :]
    return vp, vs, rho, sc, gc, wav


def prep(g, key, fs, vp, vs, rho, sc, gc, sfield, rfield):
    """Reference-made oracle inputs: staggered padded models, C-PML tables, maps."""
    s = SHOT
    rg = grid(s["nx"], s["nz"], s["lpml"], s["dx"], s["dx"], s["dt"], s["nt"], s["order"], fs)
    nxp, nzp = s["nx"] + 2 * s["lpml"], s["nz"] + 2 * s["lpml"]
    if vs is None:
        m = np.zeros((3, nzp, nxp), np.float32)
        api.ref().ref_stagger_a2d_f(C.byref(rg), vp.ctypes.data, rho.ctypes.data, *[m[i].ctypes.data for i in range(3)])
    else:
        m = np.zeros((5, nzp, nxp), np.float32)
        api.ref().ref_stagger_e2d_f(C.byref(rg), vp.ctypes.data, vs.ctypes.data, rho.ctypes.data,
                                    *[m[i].ctypes.data for i in range(5)])
    tab = np.zeros(12 * s["lpml"], np.float32)
    api.ref().ref_pml_tables_f(s["lpml"], s["dt"], tab.ctypes.data)
    maps = {}
    for which, coords, field in ((0, sc, sfield), (1, gc, rfield)):
        mp = np.zeros((len(coords), 2), np.int32)
        sh = np.zeros((len(coords), 2), np.float32)
        api.ref().ref_makemap2d_field_f(C.byref(rg), len(coords), np.ascontiguousarray(coords).ctypes.data, which,
                                        field, mp.ctypes.data, sh.ctypes.data)
        maps[which] = (mp, sh)
    g[f"{key}_models"], g[f"{key}_tab"] = m, tab
    g[f"{key}_smap"], g[f"{key}_sshift"] = maps[0]
    g[f"{key}_gmap"], g[f"{key}_gshift"] = maps[1]


def problem(fs, vp, vs, rho):
    s = SHOT
    return api.Problem2D(s["nx"], s["nz"], s["dx"], s["dx"], s["lpml"], s["order"], fs, s["dt"], s["nt"], vp, rho, vs)


def modelling_cases(g):
    cases = [("mod_a2d_pp_fs0", False, 0, PRESSURE, PRESSURE), ("mod_a2d_pp_fs1", False, 1, PRESSURE, PRESSURE),
             ("mod_a2d_pvx_fs0", False, 0, PRESSURE, VX), ("mod_e2d_pvx_fs0", True, 0, PRESSURE, VX),
             ("mod_e2d_vzvz_fs1", True, 1, VZ, VZ), ("mod_e2d_vxp_fs0", True, 0, VX, PRESSURE)]
    names = []
    for i, (key, elastic, fs, sf, rf) in enumerate(cases):
        vp, vs, rho, sc, gc, wav = shot_inputs(20 + i, elastic)
        pb = problem(fs, vp, vs, rho)
        if elastic:
            out = api.ref_modelling_e2d(pb, sc, wav, sf, gc, rf)
        else:
            out = api.ref_modelling_a2d(pb, sc, wav, sf, gc, rf)
        g[f"{key}_vp"], g[f"{key}_rho"], g[f"{key}_wav"] = vp, rho, wav
        if elastic:
            g[f"{key}_vs"] = vs
        g[f"{key}_sc"], g[f"{key}_gc"] = sc, gc
        g[f"{key}_meta"] = np.array([int(elastic), fs, sf, rf], np.int32)
        prep(g, key, fs, vp, vs, rho, sc, gc, sf, rf)
        g[f"{key}_traces"] = out
        names.append(key)
    g["mod_cases"] = np.array(names)


def adjoint_cases(g):
    vp, _, rho, sc, gc, wav = shot_inputs(40, False)
    # observed data: the shot in a model with a slow lens, so the residual is nonzero
    vtrue = vp.copy()
    vtrue[10:18, 15:26] *= 0.93
    obs = api.ref_modelling_a2d(problem(0, vtrue, None, rho), sc, wav, PRESSURE, gc, PRESSURE)
    pb = problem(0, vp, None, rho)
    fwi = api.ref_fwi_a2d(pb, sc, wav, gc, obs, 5)
    g["fwi_vp"], g["fwi_rho"], g["fwi_wav"], g["fwi_sc"], g["fwi_gc"], g["fwi_obs"] = vp, rho, wav, sc, gc, obs
    prep(g, "fwi", 0, vp, None, rho, sc, gc, PRESSURE, PRESSURE)
    for k, v in fwi.items():
        g[f"fwi_out_{k}"] = np.asarray(v)
    # the CORRELATION misfit (misfit type 1) on the same shot
    for k, v in api.ref_fwi_a2d(pb, sc, wav, gc, obs, 5, misfit=1).items():
        g[f"fwi_corr_out_{k}"] = np.asarray(v)
    img = api.ref_rtm_a2d(pb, sc, wav, gc, obs, 5, nhx=3, nhz=1)
    g["rtm_image_h3"] = img


def e2d_fwi_cases(g):
    """FwiElastic2D::run_optimal (P, Ux, Uz data) on the small shot, observed data
    modelled by the reference in a model with a slow lens."""
    vp, vs, rho, sc, gc, wav = shot_inputs(41, True)
    vtrue = vp.copy()
    vtrue[10:18, 15:26] *= 0.93
    pbt = problem(0, vtrue, vs, rho)
    obs3 = [api.ref_modelling_e2d(pbt, sc, wav, PRESSURE, gc, f) for f in (PRESSURE, VX, VZ)]
    pb = problem(0, vp, vs, rho)
    g["e2dfwi_vp"], g["e2dfwi_vs"], g["e2dfwi_rho"], g["e2dfwi_wav"] = vp, vs, rho, wav
    g["e2dfwi_sc"], g["e2dfwi_gc"], g["e2dfwi_obs"] = sc, gc, np.stack(obs3)
    prep(g, "e2dfwi", 0, vp, vs, rho, sc, gc, PRESSURE, PRESSURE)
    s = SHOT
    rg = grid(s["nx"], s["nz"], s["lpml"], s["dx"], s["dx"], s["dt"], s["nt"], s["order"], 0)
    for name, field in (("vx", VX), ("vz", VZ)):
        mp = np.zeros((len(gc), 2), np.int32)
        sh = np.zeros((len(gc), 2), np.float32)
        api.ref().ref_makemap2d_field_f(C.byref(rg), len(gc), np.ascontiguousarray(gc).ctypes.data, 1, field,
                                        mp.ctypes.data, sh.ctypes.data)
        g[f"e2dfwi_gmap_{name}"], g[f"e2dfwi_gshift_{name}"] = mp, sh
    for k, v in api.ref_fwi_e2d(pb, sc, wav, PRESSURE, gc, obs3, 5).items():
        g[f"e2dfwi_out_{k}"] = np.asarray(v)
    for k, v in api.ref_fwi_e2d(pb, sc, wav, PRESSURE, gc, obs3, 5, misfit=1).items():
        g[f"e2dfwi_corr_{k}"] = np.asarray(v)


INTERP_AXES = ((800, 0.0, 1e-3), (333, 0.0103, 2.37e-3), (120, -0.05, 7e-3))


def interp_cases(g):
    """Interp<float>::interp, LINEAR / BSPLINE / SINC, onto finer, irregular-ratio and
    coarser time axes (the last one starting before the input trace)."""
    rng = np.random.default_rng(3)
    n1, d1 = 400, 2e-3
    data = np.stack([synth.ricker(n1, d1, 25.0) * (k + 1) for k in range(5)]).astype(np.float32)
    data += (rng.standard_normal((5, n1)) * 0.01).astype(np.float32)
    g["interp_in"] = data
    g["interp_axis_in"] = np.array([n1, 0.0, d1])
    for mode in (0, 1, 2):
        for a, (n2, o2, d2) in enumerate(INTERP_AXES):
            g[f"interp_m{mode}_a{a}"] = api.ref_interp(mode, data, np.float32(0.0), np.float32(d1), n2,
                                                       np.float32(o2), np.float32(d2))


def a3d_cases(g):
    """Acoustic 3D shots (ModellingAcoustic3D::run) with reference-made inputs."""
    nx, ny, nz, L, nt, dx = 15, 13, 14, 4, 70, 10.0
    vp = np.stack([synth.layered_vp(nx, nz, dx, 1500, 3000, 3, 0.05, 40, 60 + k) for k in range(ny)], 1)
    vp = np.ascontiguousarray(vp.astype(np.float32))
    rho = synth.gardner(vp)
    sc = np.array([[71.3, 63.9, 52.2]])
    gc = np.stack([np.linspace(4.0, 131.0, 6), np.linspace(9.0, 111.0, 6), np.full(6, 7.3)], 1)
    gc = gc.astype(np.float32).astype(np.float64)
    wav = synth.ricker(nt, 1e-3, 30.0)[None, :]
    g["a3d_vp"], g["a3d_rho"], g["a3d_sc"], g["a3d_gc"], g["a3d_wav"] = vp, rho, sc, gc, wav
    g["a3d_grid"] = np.array([nx, ny, nz, L, nt, dx])
    tab = np.zeros(12 * L, np.float32)
    api.ref().ref_pml_tables_f(L, 1e-3, tab.ctypes.data)
    g["a3d_tab"] = tab
    for fs, sf, rf in ((0, PRESSURE, PRESSURE), (1, PRESSURE, VZ), (0, VX, PRESSURE)):
        key = f"a3d_fs{fs}_s{sf}_r{rf}"
        pb = api.Problem3D(nx, ny, nz, dx, dx, dx, L, 8, fs, 1e-3, nt, vp, rho)
        g[f"{key}_traces"] = api.ref_modelling_a3d(pb, sc, wav, sf, gc, rf)
        g[f"{key}_models"] = api.ref_stagger_a3d(pb)
        g[f"{key}_smap"], g[f"{key}_sshift"] = api.ref_makemap3d(pb, sc, 0, sf)
        g[f"{key}_gmap"], g[f"{key}_gshift"] = api.ref_makemap3d(pb, gc, 1, rf)
    # extended 3D RTM image of the first case's gather
    pb = api.Problem3D(nx, ny, nz, dx, dx, dx, L, 8, 0, 1e-3, nt, vp, rho)
    g["a3d_rtm_image"] = api.ref_rtm_a3d(pb, sc, wav, gc, g["a3d_fs0_s0_r0_traces"], 5, 3, 1, 3)
    # FWI gradient against an observed gather from a model with a slow block
    vt = vp.copy()
    vt[5:9, 4:8, 5:10] *= 0.92
    pbt = api.Problem3D(nx, ny, nz, dx, dx, dx, L, 8, 0, 1e-3, nt, vt, rho)
    obs = api.ref_modelling_a3d(pbt, sc, wav, PRESSURE, gc, PRESSURE)
    g["a3d_fwi_obs"] = obs
    for k, v in api.ref_fwi_a3d(pb, sc, wav, gc, obs, 5).items():
        g[f"a3d_fwi_{k}"] = np.asarray(v)
    for k, v in api.ref_fwi_a3d(pb, sc, wav, gc, obs, 5, misfit=1).items():
        g[f"a3d_fwi_corr_{k}"] = np.asarray(v)
    g["a3d_cases"] = np.array([f"a3d_fs{fs}_s{sf}_r{rf}" for fs, sf, rf in ((0, 0, 0), (1, 0, 3), (0, 1, 0))])


def main():
    if not api.ref_available():
        raise SystemExit("oracle/_ref/librsref.so is missing: build it with `make -C oracle ref`")
    g: dict = {}
    der_cases(g)
    pml_cases(g)
    stagger_cases(g)
    makemap_cases(g)
    revolve_cases(g)
    modelling_cases(g)
    adjoint_cases(g)
    e2d_fwi_cases(g)
    interp_cases(g)
    a3d_cases(g)
    np.savez_compressed(OUT, **g)
    print(f"wrote {OUT}: {len(g)} arrays, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main()

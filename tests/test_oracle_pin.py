"""Pins of the CPU oracle and of the host preprocessing (no GPU needed).

tests/golden/reference.npz holds outputs of the unmodified reference library
on seeded inputs (generated by tests/golden/make_golden.py).  Here:

* the C restatement (oracle/rs_oracle.c) must reproduce them bit for bit:
  Der stencils (lib/der.cpp), acoustic and elastic 2D shot gathers
  (lib/modelling.cpp:197-291, 545-645), the acoustic FWI gradient
  (lib/fwi.cpp:1150-1332) and the extended RTM image (lib/rtm.cpp:423-545);
* this library's host preprocessing (include/rsgpu.h: rsgpu_pml_tables,
  rsgpu_stagger_model, rsgpu_make_map, rsgpu_revolve_trace) must reproduce
  Pml::computeABC, Model*::staggerModels, Data2D::makeMap and Revolve bit for
  bit, since the GPU path consumes exactly those arrays;
* where the reference library is built here (oracle/_ref), the oracle is also
  compared with it live on inputs not in the fixtures.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import api
from rockseis_b200 import abi, synth
from rockseis_b200.rockseis import Data2D, ModelAcoustic2D, ModelElastic2D

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference.npz"))
SHOT = dict(nx=41, nz=31, lpml=8, dx=10.0, dt=1e-3, nt=150, order=8)


def problem(fs, vp, rho, vs=None):
    s = SHOT
    return api.Problem2D(s["nx"], s["nz"], s["dx"], s["dx"], s["lpml"], s["order"], fs, s["dt"], s["nt"], vp, rho, vs)


# ---------------------------------------------------------------- oracle vs reference fixtures
@pytest.mark.parametrize("order", range(1, 9))
def test_oracle_der_matches_reference(order):
    f = GOLD["der_in"]
    dx, dz = GOLD["der_dx_dz"]
    nz, nx = f.shape
    for k, which in enumerate((0, 2, 3, 5)):
        out = np.zeros_like(f)
        api.oracle().orc_der2d(nx, nz, order, float(dx), float(dz), which, f.ctypes.data, out.ctypes.data)
        assert np.array_equal(out, GOLD["der_out"][order - 1, k]), f"which={which}"


@pytest.mark.parametrize("case", [str(c) for c in GOLD["mod_cases"]])
def test_oracle_shot_gather_matches_reference(case):
    g = lambda k: GOLD[f"{case}_{k}"]  # noqa: E731
    elastic, fs, sf, rf = (int(x) for x in g("meta"))
    pb = problem(fs, g("vp"), g("rho"), g("vs") if elastic else None)
    models = list(g("models"))
    args = (pb, models, g("tab"), g("smap"), g("sshift"), g("wav"), sf, g("gmap"), g("gshift"), rf)
    out = api.orc_modelling_e2d(*args) if elastic else api.orc_modelling_a2d(*args)
    ref = g("traces")
    assert np.abs(ref).max() > 0
    assert np.array_equal(out, ref), f"max abs diff {np.abs(out - ref).max()}"


def test_oracle_fwi_gradient_matches_reference():
    g = lambda k: GOLD[f"fwi_{k}"]  # noqa: E731
    pb = problem(0, g("vp"), g("rho"))
    r = api.orc_fwi_a2d(pb, list(g("models")), g("tab"), g("smap"), g("sshift"), g("wav"), g("gmap"), g("gshift"),
                        g("obs"))
    for k in ("vpgrad", "rhograd", "wavgrad", "datamod", "datares"):
        ref = g(f"out_{k}")
        assert np.abs(ref).max() > 0, k
        assert np.array_equal(r[k], ref), f"{k}: max abs diff {np.abs(r[k] - ref).max()}"
    assert r["misfit"] == float(g("out_misfit"))


def test_oracle_correlation_misfit_gradient_matches_reference():
    g = lambda k: GOLD[f"fwi_{k}"]  # noqa: E731
    pb = problem(0, g("vp"), g("rho"))
    r = api.orc_fwi_a2d(pb, list(g("models")), g("tab"), g("smap"), g("sshift"), g("wav"), g("gmap"), g("gshift"),
                        g("obs"), misfit=1)
    for k in ("vpgrad", "rhograd", "wavgrad", "datamod", "datares"):
        ref = g(f"corr_out_{k}")
        assert np.abs(ref).max() > 0, k
        assert np.array_equal(r[k], ref), f"{k}: max abs diff {np.abs(r[k] - ref).max()}"
    assert r["misfit"] == float(g("corr_out_misfit")) and r["misfit"] < 0
    # the 97th-percentile clip zeroed at least 3 % of the residual samples
    assert (r["datares"] == 0).mean() >= 0.03


def test_oracle_rtm_image_matches_reference():
    g = lambda k: GOLD[f"fwi_{k}"]  # noqa: E731
    pb = problem(0, g("vp"), g("rho"))
    img = api.orc_rtm_a2d(pb, list(g("models")), g("tab"), g("smap"), g("sshift"), g("wav"), g("gmap"), g("gshift"),
                          g("obs"), nhx=3, nhz=1)
    ref = GOLD["rtm_image_h3"]
    assert np.abs(ref).max() > 0
    assert np.array_equal(img, ref), f"max abs diff {np.abs(img - ref).max()}"


# ---------------------------------------------------------------- host preprocessing vs reference fixtures
@pytest.mark.parametrize("lpml", [10, 30])
def test_pml_tables_match_reference(lpml):
    t = np.zeros(12 * lpml, np.float32)
    abi.check(abi.lib.rsgpu_pml_tables(lpml, float(GOLD[f"pml_{lpml}_dt"][0]), abi.F32_EXACT, t.ctypes.data))
    assert np.array_equal(t, GOLD[f"pml_{lpml}"])


@pytest.mark.parametrize("fs", [0, 1])
def test_stagger_models_match_reference(fs):
    vp, vs, rho = GOLD["stag_vp"], GOLD["stag_vs"], GOLD["stag_rho"]
    nz, nx = vp.shape
    a = ModelAcoustic2D(nx, nz, 5, 10.0, 10.0, 0.0, 0.0, fs)
    a.createModel()
    a.Vp[:], a.R[:] = vp, rho
    for got, ref in zip(a.padded(), GOLD[f"stag_a2d_fs{fs}"]):
        assert np.array_equal(got, ref)
    e = ModelElastic2D(nx, nz, 5, 10.0, 10.0, 0.0, 0.0, fs)
    e.createModel()
    e.Vp[:], e.Vs[:], e.R[:] = vp, vs, rho
    for name, got, ref in zip(e.names, e.padded(), GOLD[f"stag_e2d_fs{fs}"]):
        assert np.array_equal(got, ref), name


@pytest.mark.parametrize("which", [0, 1])
@pytest.mark.parametrize("field", [abi.PRESSURE, abi.VX, abi.VZ])
def test_make_map_matches_reference(which, field):
    nx, nz, lpml, dx, dz, ox, oz = GOLD["map_grid"]
    m = ModelAcoustic2D(int(nx), int(nz), int(lpml), dx, dz, ox, oz, 0)
    coords = GOLD["map_coords"]
    d = Data2D(len(coords), 10, 1e-3, 0.0)
    (d.scoords if which == 0 else d.gcoords)[:] = coords
    d.setField(field)
    d.makeMap(m, which)
    mp, sh = (d.smap, d.sshift) if which == 0 else (d.gmap, d.gshift)
    ref_map, ref_shift = GOLD[f"map_w{which}_f{field}"], GOLD[f"shift_w{which}_f{field}"]
    assert (ref_map[:, 0] < 0).any() and (ref_map[:, 0] >= 0).any()     # off-grid and on-grid traces covered
    on = ref_map[:, 0] >= 0
    assert np.array_equal(mp[:, 0] >= 0, on)
    assert np.array_equal(mp[on], ref_map[on])
    assert np.array_equal(sh[on], ref_shift[on])


@pytest.mark.parametrize("pair", [tuple(int(x) for x in p) for p in GOLD["rev_pairs"]])
def test_revolve_schedule_matches_reference(pair):
    nt, nc = pair
    ref = GOLD[f"rev_{nt}_{nc}"]
    n = ref.shape[1]
    a, c, k = (np.zeros(n + 8, np.int32) for _ in range(3))
    cnt = C.c_int()
    ip = C.POINTER(C.c_int)
    abi.check(abi.lib.rsgpu_revolve_trace(nt, nc, n + 8, a.ctypes.data_as(ip), c.ctypes.data_as(ip),
                                          k.ctypes.data_as(ip), C.byref(cnt)))
    assert cnt.value == n
    assert np.array_equal(np.stack([a[:n], c[:n], k[:n]]), ref)
    assert abi.lib.rsgpu_revolve_numforw(nt, nc) == int(GOLD[f"rev_numforw_{nt}_{nc}"][0])


# ---------------------------------------------------------------- oracle vs the reference library, live
needs_ref = pytest.mark.skipif(not api.ref_available(), reason="reference library oracle/_ref not built here")


def _live_case(seed, elastic, fs, sf, rf):
    s = SHOT
    vp = synth.layered_vp(s["nx"], s["nz"], s["dx"], 1600, 3200, 4, 0.08, 40, seed)
    rho = synth.gardner(vp)
    vs = (vp / 1.9).astype(np.float32) if elastic else None
    prec = abi.F32_EXACT
    m = (ModelElastic2D if elastic else ModelAcoustic2D)(s["nx"], s["nz"], s["lpml"], s["dx"], s["dx"], 0.0, 0.0, fs)
    m.createModel()
    m.Vp[:], m.R[:] = vp, rho
    if elastic:
        m.Vs[:] = vs
    rng = np.random.default_rng(seed)
    sc = np.array([[rng.uniform(50, 350), rng.uniform(5, 250)]])
    gc = synth.surface_line(9, rng.uniform(0, 20), 41.0, rng.uniform(0, 30)).astype(np.float32).astype(np.float64)
    wav = synth.ricker(s["nt"], s["dt"], 18.0)[None, :]
    src, rec = Data2D(1, s["nt"], s["dt"], 0.0, prec), Data2D(len(gc), s["nt"], s["dt"], 0.0, prec)
    src.scoords[:], rec.gcoords[:] = sc, gc
    src.setField(sf)
    rec.setField(rf)
    src.makeMap(m, 0)
    rec.makeMap(m, 1)
    tab = np.zeros(12 * s["lpml"], np.float32)
    abi.check(abi.lib.rsgpu_pml_tables(s["lpml"], s["dt"], prec, tab.ctypes.data))
    pb = problem(fs, vp, rho, vs)
    return pb, m, src, rec, tab, sc, gc, wav


@needs_ref
@pytest.mark.parametrize("seed,elastic,fs,sf,rf", [(101, False, 0, abi.PRESSURE, abi.VZ),
                                                   (102, False, 1, abi.VX, abi.PRESSURE),
                                                   (103, True, 1, abi.PRESSURE, abi.PRESSURE),
                                                   (104, True, 0, abi.VZ, abi.VX)])
def test_oracle_with_library_preprocessing_matches_reference_live(seed, elastic, fs, sf, rf):
    """Oracle fed by this library's host preprocessing vs the reference run end to end."""
    pb, m, src, rec, tab, sc, gc, wav = _live_case(seed, elastic, fs, sf, rf)
    args = (pb, m.padded(), tab, src.smap, src.sshift, wav, sf, rec.gmap, rec.gshift, rf)
    if elastic:
        out, ref = api.orc_modelling_e2d(*args), api.ref_modelling_e2d(pb, sc, wav, sf, gc, rf)
    else:
        out, ref = api.orc_modelling_a2d(*args), api.ref_modelling_a2d(pb, sc, wav, sf, gc, rf)
    assert np.abs(ref).max() > 0
    assert np.array_equal(out, ref), f"max abs diff {np.abs(out - ref).max()}"


# ---------------------------------------------------------------- acoustic 3D
def _a3d_key(case):
    """'a3d_fs<fs>_s<src field>_r<rec field>' -> (fs, src field, rec field)."""
    _, f, s_, r = case.split("_")
    return int(f[2:]), int(s_[1:]), int(r[1:])


def _a3d_problem(fs):
    nx, ny, nz, L, nt, dx = (GOLD["a3d_grid"][k] for k in range(6))
    return api.Problem3D(int(nx), int(ny), int(nz), dx, dx, dx, int(L), 8, fs, 1e-3, int(nt), GOLD["a3d_vp"],
                         GOLD["a3d_rho"])


@pytest.mark.parametrize("case", [str(c) for c in GOLD["a3d_cases"]])
def test_oracle_3d_shot_gather_matches_reference(case):
    fs, sf, rf = _a3d_key(case)
    pb = _a3d_problem(fs)
    g = lambda k: GOLD[f"{case}_{k}"]  # noqa: E731
    out = api.orc_modelling_a3d(pb, list(g("models")), GOLD["a3d_tab"], g("smap"), g("sshift"), GOLD["a3d_wav"], sf,
                                g("gmap"), g("gshift"), rf)
    ref = g("traces")
    assert np.abs(ref).max() > 0
    assert np.array_equal(out, ref), f"max abs diff {np.abs(out - ref).max()}"


@pytest.mark.parametrize("case", [str(c) for c in GOLD["a3d_cases"]])
def test_3d_host_preprocessing_matches_reference(case):
    from rockseis_b200.rockseis import Data3D, ModelAcoustic3D
    fs, sf, rf = _a3d_key(case)
    nx, ny, nz, L, nt, dx = (GOLD["a3d_grid"][k] for k in range(6))
    m = ModelAcoustic3D(int(nx), int(ny), int(nz), int(L), dx, dx, dx, 0.0, 0.0, 0.0, fs)
    m.createModel()
    m.Vp[:], m.R[:] = GOLD["a3d_vp"], GOLD["a3d_rho"]
    for got, ref in zip(m.padded(), GOLD[f"{case}_models"]):
        assert np.array_equal(got, ref)
    for which, coords, field, key in ((0, GOLD["a3d_sc"], sf, "s"), (1, GOLD["a3d_gc"], rf, "g")):
        d = Data3D(len(coords), int(nt), 1e-3, 0.0)
        (d.scoords if which == 0 else d.gcoords)[:] = coords
        d.setField(field)
        d.makeMap(m, which)
        mp, sh = (d.smap, d.sshift) if which == 0 else (d.gmap, d.gshift)
        assert np.array_equal(mp, GOLD[f"{case}_{key}map"])
        assert np.array_equal(sh, GOLD[f"{case}_{key}shift"])


def test_oracle_3d_rtm_image_matches_reference():
    case = "a3d_fs0_s0_r0"
    pb = _a3d_problem(0)
    g = lambda k: GOLD[f"{case}_{k}"]  # noqa: E731
    img = api.orc_rtm_a3d(pb, list(g("models")), GOLD["a3d_tab"], g("smap"), g("sshift"), GOLD["a3d_wav"], g("gmap"),
                          g("gshift"), g("traces"), 3, 1, 3)
    ref = GOLD["a3d_rtm_image"]
    assert np.abs(ref).max() > 0
    assert np.array_equal(img, ref), f"max abs diff {np.abs(img - ref).max()}"


def test_oracle_3d_fwi_gradient_matches_reference():
    case = "a3d_fs0_s0_r0"
    pb = _a3d_problem(0)
    g = lambda k: GOLD[f"{case}_{k}"]  # noqa: E731
    r = api.orc_fwi_a3d(pb, list(g("models")), GOLD["a3d_tab"], g("smap"), g("sshift"), GOLD["a3d_wav"], g("gmap"),
                        g("gshift"), GOLD["a3d_fwi_obs"])
    for k in ("vpgrad", "rhograd", "wavgrad", "datamod", "datares"):
        ref = GOLD[f"a3d_fwi_{k}"]
        assert np.abs(ref).max() > 0, k
        assert np.array_equal(r[k], ref), f"{k}: max abs diff {np.abs(r[k] - ref).max()}"
    assert r["misfit"] == float(GOLD["a3d_fwi_misfit"])


def test_oracle_3d_correlation_misfit_matches_reference():
    # FwiAcoustic3D's CORRELATION residuals carry no percentile clip
    case = "a3d_fs0_s0_r0"
    pb = _a3d_problem(0)
    g = lambda k: GOLD[f"{case}_{k}"]  # noqa: E731
    r = api.orc_fwi_a3d(pb, list(g("models")), GOLD["a3d_tab"], g("smap"), g("sshift"), GOLD["a3d_wav"], g("gmap"),
                        g("gshift"), GOLD["a3d_fwi_obs"], misfit=1)
    for k in ("vpgrad", "rhograd", "wavgrad", "datamod", "datares"):
        ref = GOLD[f"a3d_fwi_corr_{k}"]
        assert np.abs(ref).max() > 0, k
        assert np.array_equal(r[k], ref), f"{k}: max abs diff {np.abs(r[k] - ref).max()}"
    assert r["misfit"] == float(GOLD["a3d_fwi_corr_misfit"])


def test_oracle_elastic_fwi_gradient_matches_reference():
    # FwiElastic2D::run_optimal with P, Ux and Uz data (DIFFERENCE misfit)
    g = lambda k: GOLD[f"e2dfwi_{k}"]  # noqa: E731
    pb = problem(0, g("vp"), g("rho"), g("vs"))
    r = api.orc_fwi_e2d(pb, list(g("models")), g("tab"), g("smap"), g("sshift"), g("wav"), abi.PRESSURE,
                        [g("gmap"), g("gmap_vx"), g("gmap_vz")], [g("gshift"), g("gshift_vx"), g("gshift_vz")],
                        list(g("obs")))
    for k in ("vpgrad", "vsgrad", "rhograd", "wavgrad", "datamod", "datares"):
        ref = g(f"out_{k}")
        assert np.abs(ref).max() > 0, k
        assert np.array_equal(r[k], ref), f"{k}: max abs diff {np.abs(r[k] - ref).max()}"
    assert r["misfit"] == float(g("out_misfit"))


def test_oracle_elastic_correlation_misfit_matches_reference():
    g = lambda k: GOLD[f"e2dfwi_{k}"]  # noqa: E731
    pb = problem(0, g("vp"), g("rho"), g("vs"))
    r = api.orc_fwi_e2d(pb, list(g("models")), g("tab"), g("smap"), g("sshift"), g("wav"), abi.PRESSURE,
                        [g("gmap"), g("gmap_vx"), g("gmap_vz")], [g("gshift"), g("gshift_vx"), g("gshift_vz")],
                        list(g("obs")), misfit=1)
    for k in ("vpgrad", "vsgrad", "rhograd", "wavgrad", "datamod", "datares"):
        ref = g(f"corr_{k}")
        assert np.abs(ref).max() > 0, k
        assert np.array_equal(r[k], ref), f"{k}: max abs diff {np.abs(r[k] - ref).max()}"
    assert r["misfit"] == float(g("corr_misfit")) and r["misfit"] < 0


INTERP_AXES = ((800, 0.0, 1e-3), (333, 0.0103, 2.37e-3), (120, -0.05, 7e-3))


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_oracle_interp_matches_reference(mode):
    n1, o1, d1 = GOLD["interp_axis_in"]
    for a, (n2, o2, d2) in enumerate(INTERP_AXES):
        got = api.orc_interp(mode, GOLD["interp_in"], np.float32(o1), np.float32(d1), n2, np.float32(o2),
                             np.float32(d2))
        ref = GOLD[f"interp_m{mode}_a{a}"]
        assert np.abs(ref).max() > 0
        assert np.array_equal(got, ref), (mode, a, np.abs(got - ref).max())


@pytest.mark.parametrize("fs", [0, 1])
def test_stagger_elastic3d_matches_reference(fs):
    """ModelElastic3D::staggerModels restated on the host (rsgpu_stagger_model),
    against the reference library itself (skipped where it is not built)."""
    from oracle import api
    from rockseis_b200.rockseis import ModelElastic3D
    if not api.ref_available():
        pytest.skip("reference library not built")
    import ctypes as C
    rng = np.random.default_rng(7)
    nx, ny, nz, l = 9, 7, 6, 3
    vp = rng.uniform(1500, 3000, (nz, ny, nx)).astype(np.float32)
    vs = (vp / rng.uniform(1.6, 2.1, vp.shape)).astype(np.float32)
    rho = rng.uniform(1000, 2500, vp.shape).astype(np.float32)
    m = ModelElastic3D(nx, ny, nz, l, 10.0, 10.0, 10.0, 0.0, 0.0, 0.0, fs)
    m.createModel()
    m.Vp[:], m.Vs[:], m.R[:] = vp, vs, rho
    g = api.RefGrid(nx, ny, nz, l, 8, fs, 10.0, 10.0, 10.0, 0.0, 0.0, 0.0, 1e-3, 10)
    ref = [np.zeros((nz + 2 * l, ny + 2 * l, nx + 2 * l), np.float32) for _ in range(8)]
    api.ref().ref_stagger_e3d_f(C.byref(g), vp.ctypes.data, vs.ctypes.data, rho.ctypes.data,
                                *[a.ctypes.data for a in ref])
    for name, got, r in zip(m.names, m.padded(), ref):
        assert np.array_equal(got, r), name


# ---------------------------------------------------------------- FULL snapshots (Fwi/RtmAcoustic2D::run)
def _snapfull():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "snapfull.npz"))


@needs_ref
def test_snapfull_fixture_matches_reference_live():
    from tests.cases import fwi_case
    g = _snapfull()
    c = fwi_case()
    assert np.array_equal(c.obs.astype(np.float32), g["obs"]) and np.array_equal(c.pb.vp, g["vp"])
    r = api.ref_fwi_a2d_full(c.pb, g["scoords"], g["wav"], g["gcoords"], g["obs"], 7)
    for k in ("vpgrad", "rhograd", "wavgrad"):
        assert np.array_equal(r[k], g[f"fwi_s7_{k}"]), k
    for k in ("datamod", "datares", "misfit"):
        assert np.array_equal(r[k], g[f"fwi_{k}"]), k
    img = api.ref_rtm_a2d_full(c.pb, g["scoords"], g["wav"], g["gcoords"], g["obs"], 4, nhx=3)
    assert np.array_equal(img, g["rtm_s4_h3"])


def test_snapshot_enddiff_and_count():
    """Snapshot2D (lib/snap.cpp:334-337): snapnt = (nt-1)/snapinc + 1 snapshots and
    enddiff = (nt-1) mod snapinc for the time steps in use; the last adjoint time
    that correlates is nt-1, the snapshot it reads is the one saved at nt-1-enddiff."""
    for nt in (2, 3, 300, 1001, 2000):
        for si in (1, 2, 3, 7, 64, nt - 1):
            if si < 1:
                continue
            snapnt = (nt - 1) // si + 1
            dt = np.float32(6e-4)
            enddiff = int(np.rint(np.float32((nt - 1) * dt - (snapnt - 1) * (dt * np.float32(si))) / dt))
            assert enddiff == (nt - 1) % si, (nt, si)


# ---------------------------------------------------------------- FULL snapshots, elastic 2D (FwiElastic2D::run)
def _e2d_full():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "e2d_full.npz"))


@needs_ref
def test_e2d_full_fixture_matches_reference_live():
    """tests/golden/e2d_full.npz (make_golden_e2d_full.py) is what the reference's
    FwiElastic2D::run returns on the elastic FWI case: the checker for a GPU FULL
    elastic gradient."""
    from tests.cases import ElasticFwiCase
    g = _e2d_full()
    c = ElasticFwiCase()
    obs3 = [o.astype(np.float32) for o in c.obs]
    assert np.array_equal(np.stack(obs3), g["obs"])
    r = api.ref_fwi_e2d(c.pb, c.src.scoords, c.src.data.astype(np.float32), c.sfield, c.recs[0].gcoords, obs3, 0,
                        full_snapinc=3)
    for k in ("vpgrad", "vsgrad", "rhograd", "wavgrad"):
        assert np.array_equal(r[k], g[f"s3_{k}"]), k
    for k in ("datamod", "datares", "misfit"):
        assert np.array_equal(r[k], g[k]), k


def test_e2d_full_fixture_is_complete():
    g = _e2d_full()
    for si in (1, 3, 5):
        for k in ("vpgrad", "vsgrad", "rhograd", "wavgrad"):
            assert np.all(np.isfinite(g[f"s{si}_{k}"])), (si, k)
    # coarser snapshots change the gradient: the adjoint correlates with older states
    assert not np.array_equal(g["s1_vpgrad"], g["s3_vpgrad"])

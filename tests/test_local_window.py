"""Aperture windows of the batched drivers: Model::getLocalsize2d/3d and the
edge-clamped copy of Model*::getLocal (lib/model.cpp:272-470, 1443-1509,
2369-2450), restated in rockseis_b200.rockseis.  The window sizes are pinned to the
reference's own getLocalsize2d/3d: against golden cases it computed
(tests/golden/localsize.json, tests/golden/make_golden_localsize.py) and, where
oracle/_ref is built, against the live library on further seeded cases.  The
reference reads its models from .rss files inside getLocal, so the copy itself is
checked against cases worked by hand."""
import json
import os

import numpy as np
import pytest

from rockseis_b200.rockseis import SMAP, GMAP, Data2D, Data3D, ModelAcoustic2D, ModelAcoustic3D

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "localsize.json")


def _ours(c):
    s, g = np.array(c["s"]), np.array(c["g"])
    if c["dim"] == 2:
        m = ModelAcoustic2D(400, 100, 10, c["dx"], c["dx"], c["ox"], 0.0, 0)
        d = Data2D(len(s), 1, 1e-3, 0.0)
        d.scoords[:] = s[:, [0, 2]]
        d.gcoords[:] = g[:, [0, 2]]
        return list(m.getLocalsize2d(d, c["ap"], c["map"]))
    m = ModelAcoustic3D(400, 300, 100, 10, c["dx"], c["dy"], c["dx"], c["ox"], c["oy"], 0.0, 0)
    d = Data3D(len(s), 1, 1e-3, 0.0)
    d.scoords[:] = s
    d.gcoords[:] = g
    (sx, nx), (sy, ny) = m.getLocalsize3d(d, c["ap"], c["apy"], c["map"])
    return [sx, nx, sy, ny]


def test_windows_equal_the_reference_golden_cases():
    with open(GOLDEN) as f:
        cases = json.load(f)
    assert len(cases) >= 60
    for c in cases:
        assert _ours(c) == c["want"], c


def test_windows_equal_the_live_reference():
    from oracle import api
    if not api.ref_available():
        pytest.skip("reference library oracle/_ref not built")
    import importlib.util
    spec = importlib.util.spec_from_file_location("mk", os.path.join(os.path.dirname(GOLDEN), "make_golden_localsize.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    for c in mk.cases(seed=99, n=200):
        s, g = np.array(c["s"]), np.array(c["g"])
        if c["dim"] == 2:
            grid = api.RefGrid(400, 1, 100, 10, 8, 0, c["dx"], 1.0, c["dx"], c["ox"], 0.0, 0.0, 1e-3, 10)
            want = list(api.ref_localsize2d(grid, s[:, [0, 2]], g[:, [0, 2]], c["ap"], c["map"]))
        else:
            grid = api.RefGrid(400, 300, 100, 10, 8, 0, c["dx"], c["dy"], c["dx"], c["ox"], c["oy"], 0.0, 1e-3, 10)
            (sx, nx), (sy, ny) = api.ref_localsize3d(grid, s, g, c["ap"], c["apy"], c["map"])
            want = [sx, nx, sy, ny]
        assert _ours(c) == want, c


def model2d(nx=100, nz=20):
    m = ModelAcoustic2D(nx, nz, 10, 10.0, 10.0, 0.0, 0.0, 0)
    m.createModel()
    m.Vp[:] = np.arange(nx, dtype=np.float32)[None, :] + 1000 * np.arange(nz, dtype=np.float32)[:, None]
    m.R[:] = 2000.0
    return m


def shot2d(sx, gxs):
    d = Data2D(len(gxs), 10, 1e-3, 0.0)
    d.scoords[:] = [[sx, 10.0]] * len(gxs)
    d.gcoords[:] = [[g, 0.0] for g in gxs]
    return d


def test_positive_aperture_centres_an_odd_window_on_the_source():
    m = model2d()
    d = shot2d(503.7, [100.0, 900.0])
    # size = rint(200/10) + 1 = 21 ; start = rint(50.37) - 10 = 40
    assert m.getLocalsize2d(d, 200.0, SMAP) == (40, 21)
    loc = m.getLocal(d, 200.0, SMAP)
    assert (loc.nx, loc.nz, loc.ox) == (21, 20, 400.0)
    assert np.array_equal(loc.Vp[0], np.arange(40, 61, dtype=np.float32))


def test_even_size_is_made_odd_and_edges_are_clamped():
    m = model2d()
    d = shot2d(15.0, [0.0])
    # size = rint(190/10) + 1 = 20 -> 21 ; start = rint(1.5) - 10 = -8 (copy clamps to column 0)
    assert m.getLocalsize2d(d, 190.0, SMAP) == (-8, 21)
    loc = m.getLocal(d, 190.0, SMAP)
    assert np.array_equal(loc.Vp[3, :10], np.full(10, 3000.0, np.float32) + np.array([0] * 9 + [1], np.float32))
    assert loc.ox == -80.0


def test_zero_aperture_uses_the_largest_offset():
    m = model2d()
    d = shot2d(500.0, [380.0, 650.0])
    # size = 2*rint(150/10) + 1 = 31 ; start = rint(50) - 15 = 35
    assert m.getLocalsize2d(d, 0.0, SMAP) == (35, 31)
    # receiver side: min over receivers = 380 -> start = 38 - 15
    assert m.getLocalsize2d(d, 0.0, GMAP) == (23, 31)


def test_negative_aperture_spans_sources_and_receivers_plus_margin():
    m = model2d()
    d = shot2d(500.0, [380.0, 650.0])
    # size = rint((650-380 + 2*50)/10) + 2 = 39 ; start = rint(38) - rint(5) - 1 = 32
    assert m.getLocalsize2d(d, -50.0, SMAP) == (32, 39)


def test_3d_window_per_axis():
    m = ModelAcoustic3D(60, 50, 10, 5, 12.5, 12.5, 12.5, 0.0, 0.0, 0.0, 0)
    m.createModel()
    m.Vp[:] = np.arange(60, dtype=np.float32)[None, None, :] + 100 * np.arange(50, dtype=np.float32)[None, :, None]
    m.R[:] = 1.0
    d = Data3D(1, 10, 1e-3, 0.0)
    d.scoords[:] = [[300.0, 200.0, 20.0]]
    d.gcoords[:] = [[300.0, 200.0, 0.0]]
    (sx, nxw), (sy, nyw) = m.getLocalsize3d(d, 250.0, 100.0, SMAP)
    assert (sx, nxw, sy, nyw) == (14, 21, 12, 9)
    loc = m.getLocal(d, 250.0, 100.0, SMAP)
    assert loc.Vp.shape == (10, 9, 21)
    assert loc.Vp[0, 0, 0] == 14 + 100 * 12
    assert (loc.ox, loc.oy) == (175.0, 150.0)

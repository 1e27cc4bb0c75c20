"""The fused z-marching step against the per-tile half-step kernels (both through the C ABI).

The fused step (rsgpu_config.launch_mode 3, the library's choice for forward
propagation) computes the same per-point arithmetic as the per-tile velocity and
stress kernels (launch_mode 2), which the other GPU tests pin to the reference.
Every trace and every wavefield after any number of steps must therefore be bit
for bit the same in all three arithmetics -- across uneven shot windows in one
batch, strips and row bands of every size, free surface, reduced stencil orders,
odd step counts and runs split at arbitrary steps.
"""
import numpy as np
import pytest

from rockseis_b200 import abi, synth
from rockseis_b200.rockseis import Data2D, ModelAcoustic2D, ModelElastic2D, Plan

pytestmark = pytest.mark.gpu

FIELDS = {abi.ACOUSTIC2D: (abi.PRESSURE, abi.VX, abi.VZ),
          abi.ELASTIC2D: (abi.VX, abi.VZ, abi.SXX, abi.SZZ, abi.SXZ)}


def batch(physics, prec, fs=0, nt=90, windows=((230, 150), (171, 121), (300, 97)), sfield=abi.PRESSURE,
          rfield=abi.VX, dx=10.0, lpml=12, seed=3):
    rng = np.random.default_rng(seed)
    models, srcs, recs = [], [], []
    for k, (nx, nz) in enumerate(windows):
        vp = synth.layered_vp(nx, nz, dx, 1500, 3500, 4, 0.05, 100, seed + k)
        cls = ModelAcoustic2D if physics == abi.ACOUSTIC2D else ModelElastic2D
        m = cls(nx, nz, lpml, dx, dx, 0.0, 0.0, fs, prec)
        m.createModel()
        m.Vp[:] = vp
        m.R[:] = synth.gardner(vp)
        if physics == abi.ELASTIC2D:
            m.Vs[:] = vp / 1.8
        s = Data2D(2, nt, 1e-3, 0.0, prec)
        s.scoords[:] = [[rng.uniform(20, (nx - 3) * dx), rng.uniform(5, 40)], [0.5 * nx * dx + 3.3, 0.4 * nz * dx]]
        s.data[:] = synth.ricker(nt, 1e-3, 15.0, abi.real_dtype(prec))[None, :] * np.array([[1.0], [0.5]])
        s.setField(sfield)
        s.makeMap(m, 0)
        r = Data2D(nx // 3, nt, 1e-3, 0.0, prec)
        r.gcoords[:] = synth.surface_line(nx // 3, 3.1, 3 * dx, 7.3)
        r.setField(rfield)
        r.makeMap(m, 1)
        models.append(m)
        srcs.append(s)
        recs.append(r)
    return models, srcs, recs


def run_plan(physics, prec, mode, splits, zchunk=0, order=8, **kw):
    models, srcs, recs = batch(physics, prec, **kw)
    p = Plan(models, srcs, recs, order, prec, launch_mode=mode, zchunk=zchunk)
    assert p.info()[0] == (3 if mode == 3 else 2)
    it = 0
    for n in splits:
        p.run(it, n)
        it += n
    traces = [p.read_traces(i) for i in range(len(models))]
    fields = [[p.read_field(i, f, (m.getNz_pml(), m.getNx_pml())) for f in FIELDS[physics]]
              for i, m in enumerate(models)]
    p.close()
    return traces, fields


def assert_same(a, b):
    ta, fa = a
    tb, fb = b
    for x, y in zip(ta, tb):
        assert np.abs(y).max() > 0
        assert np.array_equal(x, y), f"traces differ: max {np.abs(x - y).max()}"
    for sa, sb in zip(fa, fb):
        for x, y in zip(sa, sb):
            assert np.array_equal(x, y), f"wavefields differ: max {np.abs(x - y).max()}"


@pytest.mark.parametrize("prec", [abi.F32_EXACT, abi.F32_FAST, abi.F64])
@pytest.mark.parametrize("physics", [abi.ACOUSTIC2D, abi.ELASTIC2D])
def test_fused_equals_tiles(require_gpu, physics, prec):
    ref = run_plan(physics, prec, 2, [90])
    assert_same(run_plan(physics, prec, 3, [90]), ref)


@pytest.mark.parametrize("physics", [abi.ACOUSTIC2D, abi.ELASTIC2D])
@pytest.mark.parametrize("splits", [[1, 2, 3, 33, 51], [37, 53], [64, 26], [89, 1]])
def test_fused_split_runs(require_gpu, physics, splits):
    ref = run_plan(physics, abi.F32_EXACT, 2, [90])
    assert_same(run_plan(physics, abi.F32_EXACT, 3, splits), ref)


@pytest.mark.parametrize("zchunk", [8, 24, 40, 200])
def test_fused_row_bands(require_gpu, zchunk):
    ref = run_plan(abi.ELASTIC2D, abi.F32_EXACT, 2, [70], nt=70)
    assert_same(run_plan(abi.ELASTIC2D, abi.F32_EXACT, 3, [70], zchunk=zchunk, nt=70), ref)


@pytest.mark.parametrize("order", [2, 5, 8])
@pytest.mark.parametrize("fs", [0, 1])
def test_fused_orders_free_surface(require_gpu, order, fs):
    for physics in (abi.ACOUSTIC2D, abi.ELASTIC2D):
        ref = run_plan(physics, abi.F32_EXACT, 2, [60], order=order, fs=fs, nt=60)
        assert_same(run_plan(physics, abi.F32_EXACT, 3, [60], order=order, fs=fs, nt=60), ref)


@pytest.mark.parametrize("sfield,rfield", [(abi.VX, abi.PRESSURE), (abi.VZ, abi.VZ), (abi.PRESSURE, abi.PRESSURE)])
def test_fused_source_receiver_fields(require_gpu, sfield, rfield):
    for physics in (abi.ACOUSTIC2D, abi.ELASTIC2D):
        ref = run_plan(physics, abi.F32_EXACT, 2, [80], sfield=sfield, rfield=rfield, nt=80)
        assert_same(run_plan(physics, abi.F32_EXACT, 3, [80], sfield=sfield, rfield=rfield, nt=80), ref)


def test_fused_small_and_narrow_windows(require_gpu):
    w = ((20, 18), (113, 17), (9, 140))
    ref = run_plan(abi.ELASTIC2D, abi.F32_EXACT, 2, [50], windows=w, nt=50, lpml=5)
    assert_same(run_plan(abi.ELASTIC2D, abi.F32_EXACT, 3, [50], windows=w, nt=50, lpml=5), ref)

"""The column-marching elastic half-steps (rsgpu_config.launch_mode 4) against the
per-tile kernels (launch_mode 2), both FAST arithmetic through the C ABI.

The marching kernels evaluate every derivative in the per-tile FAST kernels'
summation order (x taps in dx_quad's order, z taps in dz_stream_f32's row order)
and every C-PML update operation by operation, so every trace and every wavefield
after any number of steps must be bit for bit the same: across uneven shot windows
in one batch, strips and row bands of every size (band edges inside and outside
the C-PML strips), windows narrower than one strip, free surface, reduced stencil
orders, all source and receiver fields, and runs split at arbitrary steps.
"""
import numpy as np
import pytest

from test_gpu_fused import batch, FIELDS
from rockseis_b200 import abi
from rockseis_b200.rockseis import Plan

pytestmark = pytest.mark.gpu

E2 = abi.ELASTIC2D
FAST = abi.F32_FAST


def run_plan(mode, splits, zchunk=0, order=8, **kw):
    models, srcs, recs = batch(E2, FAST, **kw)
    p = Plan(models, srcs, recs, order, FAST, launch_mode=mode, zchunk=zchunk)
    info = p.info()
    assert info[0] == (4 if mode == 4 else 2)
    if mode == 4:
        assert info[1] > 0 and info[2] % 8 == 0
    it = 0
    for n in splits:
        p.run(it, n)
        it += n
    traces = [p.read_traces(i) for i in range(len(models))]
    fields = [[p.read_field(i, f, (m.getNz_pml(), m.getNx_pml())) for f in FIELDS[E2]] for i, m in enumerate(models)]
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


def test_march_equals_tiles(require_gpu):
    assert_same(run_plan(4, [90]), run_plan(2, [90]))


@pytest.mark.parametrize("splits", [[1, 2, 3, 33, 51], [64, 26]])
def test_march_split_runs(require_gpu, splits):
    assert_same(run_plan(4, splits), run_plan(2, [90]))


@pytest.mark.parametrize("zchunk", [8, 24, 40, 200])
def test_march_row_bands(require_gpu, zchunk):
    ref = run_plan(2, [70], nt=70)
    assert_same(run_plan(4, [70], zchunk=zchunk, nt=70), ref)


@pytest.mark.parametrize("order", [2, 5, 8])
@pytest.mark.parametrize("fs", [0, 1])
def test_march_orders_free_surface(require_gpu, order, fs):
    ref = run_plan(2, [60], order=order, fs=fs, nt=60)
    assert_same(run_plan(4, [60], order=order, fs=fs, nt=60), ref)


@pytest.mark.parametrize("sfield,rfield", [(abi.VX, abi.PRESSURE), (abi.VZ, abi.VZ), (abi.PRESSURE, abi.PRESSURE)])
def test_march_source_receiver_fields(require_gpu, sfield, rfield):
    ref = run_plan(2, [80], sfield=sfield, rfield=rfield, nt=80)
    assert_same(run_plan(4, [80], sfield=sfield, rfield=rfield, nt=80), ref)


def test_march_small_narrow_and_wide_windows(require_gpu):
    w = ((20, 18), (113, 17), (9, 140), (301, 44))
    ref = run_plan(2, [50], windows=w, nt=50, lpml=5)
    assert_same(run_plan(4, [50], windows=w, nt=50, lpml=5), ref)


def test_march_mode_falls_back_outside_its_scope(require_gpu):
    """Launch mode 4 covers FAST elastic forward propagation only; the exact
    arithmetics (and acoustic plans) keep the per-tile kernels."""
    models, srcs, recs = batch(E2, abi.F32_EXACT)
    p = Plan(models, srcs, recs, 8, abi.F32_EXACT, launch_mode=4)
    assert p.info()[0] == 2
    p.close()

"""GPU parity of the 2D forward propagators (through the C ABI) against the oracle.

EXACT mode must reproduce the reference's float arithmetic bit for bit
(np.array_equal against the CPU restatement, which is itself pinned bit-exact
against the reference).  FAST mode (FMA, pre-scaled coefficients) is held to the
plain-FP32 parity bar: relative L2 <= 1e-5 on the shot gather.
"""
import numpy as np
import pytest

from rockseis_b200 import abi
from rockseis_b200.rockseis import ModellingAcoustic2D, ModellingElastic2D, Plan, modelling_batch
from tests.cases import Case2D, rel_l2

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-5


def run_gpu(case, precision=None, tile=-1):
    prec = case.precision if precision is None else precision
    case.rec.data[:] = 0
    cls = ModellingAcoustic2D if case.physics == abi.ACOUSTIC2D else ModellingElastic2D
    mod = cls(case.model, case.src, case.order, 1, precision=prec)
    mod.tile = tile
    if case.rec.field == abi.PRESSURE:
        mod.setRecP(case.rec)
    elif case.rec.field == abi.VX:
        mod.setRecVx(case.rec)
    else:
        mod.setRecVz(case.rec)
    assert mod.run() == 1
    return case.rec.data.copy()


@pytest.mark.parametrize("fs", [0, 1])
@pytest.mark.parametrize("tile", list(range(10)))
def test_acoustic2d_exact_bitwise(require_gpu, fs, tile):
    c = Case2D(abi.ACOUSTIC2D, fs=fs)
    gpu = run_gpu(c, tile=tile)
    ref = c.oracle_traces()
    assert np.abs(ref).max() > 0
    assert np.array_equal(gpu, ref), f"max abs diff {np.abs(gpu - ref).max()}"


@pytest.mark.parametrize("sfield,rfield", [(abi.PRESSURE, abi.PRESSURE), (abi.PRESSURE, abi.VX),
                                           (abi.VX, abi.PRESSURE), (abi.VZ, abi.VZ)])
@pytest.mark.parametrize("fs", [0, 1])
def test_elastic2d_exact_bitwise(require_gpu, sfield, rfield, fs):
    c = Case2D(abi.ELASTIC2D, fs=fs, sfield=sfield, rfield=rfield, nt=250)
    gpu = run_gpu(c)
    ref = c.oracle_traces()
    assert np.abs(ref).max() > 0
    assert np.array_equal(gpu, ref), f"max abs diff {np.abs(gpu - ref).max()}"


@pytest.mark.parametrize("physics", [abi.ACOUSTIC2D, abi.ELASTIC2D])
def test_fast_mode_within_fp32_tolerance(require_gpu, physics):
    c = Case2D(physics, nt=300)
    gpu = run_gpu(c, precision=abi.F32_FAST)
    ref = c.oracle_traces()
    assert rel_l2(gpu, ref) <= FAST_TOL


@pytest.mark.parametrize("order", [2, 4, 6])
def test_low_orders_and_vz_source(require_gpu, order):
    c = Case2D(abi.ACOUSTIC2D, order=order, sfield=abi.VZ, rfield=abi.VX, nt=200)
    gpu = run_gpu(c)
    assert np.array_equal(gpu, c.oracle_traces())


def test_states_after_steps_bitwise(require_gpu):
    """Every wavefield (not only the traces) equals the oracle after n steps."""
    c = Case2D(abi.ELASTIC2D, nt=120, fs=1)
    p = Plan([c.model], [c.src], [c.rec], c.order)
    p.run(0, 120)
    _, st = c.oracle_traces(nsteps=120, want_state=True)
    shape = st.shape[1:]
    for k, f in enumerate((abi.VX, abi.VZ, abi.SXX, abi.SZZ, abi.SXZ)):
        assert np.array_equal(p.read_field(0, f, shape), st[k])
    p.close()


def test_batched_uneven_windows_bitwise(require_gpu):
    """Shots with different window sizes advance in one launch; each equals its solo run."""
    cases = [Case2D(abi.ELASTIC2D, nx=nx, nz=nz, nt=150, scoord=(sx, 31.0), seed=s)
             for nx, nz, sx, s in [(81, 61, 400.3, 1), (97, 45, 150.0, 2), (64, 70, 333.3, 3)]]
    for c in cases:
        c.rec.data[:] = 0
    modelling_batch([c.model for c in cases], [c.src for c in cases], [c.rec for c in cases], 8)
    for c in cases:
        assert np.array_equal(c.rec.data, c.oracle_traces())


def test_offgrid_receivers_are_skipped(require_gpu):
    c = Case2D(abi.ACOUSTIC2D, nt=100, rx0=-300.0, rdx=100.0, nrec=12)
    assert (c.rec.gmap[:, 0] < 0).any()
    gpu = run_gpu(c)
    ref = c.oracle_traces()
    assert np.array_equal(gpu, ref)
    assert np.all(gpu[c.rec.gmap[:, 0] < 0] == 0)


def test_graph_replay_matches_direct_launches(require_gpu):
    """Steps replayed from the captured CUDA graph equal steps launched one by one."""
    c = Case2D(abi.ACOUSTIC2D, nt=100)
    p = Plan([c.model], [c.src], [c.rec], c.order)
    p.run(0, 64)
    p.run(64, 36)
    a = p.read_traces(0)
    p.reset()
    for it in range(100):
        p.run(it, 1)
    b = p.read_traces(0)
    assert np.array_equal(a, b)
    assert np.array_equal(a, c.oracle_traces())
    p.close()

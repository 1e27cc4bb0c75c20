"""Elastic 3D propagation on the GPU (through the C ABI) against the reference itself.

The checker is the unmodified reference library (oracle/_ref/librsref.so):
ModellingElastic3D<float>::run for shot gathers and WavesElastic3D's
forwardstepVelocity / forwardstepStress / insertSource for whole wavefields
(lib/waves.cpp:2465-3257, 4104-4400, lib/modelling.cpp:727-850).  EXACT
arithmetic must reproduce both bit for bit -- all nine fields, every source and
receiver type, free surface on and off, reduced stencil orders; FAST arithmetic
(FMA) is held to relative L2 <= 1e-5 on the gather.
"""
import numpy as np
import pytest

from oracle import api
from rockseis_b200 import abi, synth
from rockseis_b200.rockseis import Data3D, ModelElastic3D, ModellingElastic3D, Plan
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-5
E3_FIELDS = (abi.VX, abi.VY, abi.VZ, abi.SXX, abi.SYY, abi.SZZ, abi.SYZ, abi.SXZ, abi.SXY)


@pytest.fixture(scope="module", autouse=True)
def need_reference():
    if not api.ref_available():
        pytest.skip("reference library oracle/_ref not built")


class Case3D:
    def __init__(self, nx=23, ny=19, nz=21, lpml=6, dx=10.0, dt=1e-3, nt=60, order=8, fs=0, seed=5,
                 sfield=abi.PRESSURE, rfield=abi.VX, precision=abi.F32_EXACT, nrec=9):
        rng = np.random.default_rng(seed)
        vp = 2000.0 + 1000.0 * np.linspace(0, 1, nz)[:, None, None] * np.ones((1, ny, nx))
        vp = (vp * (1 + 0.05 * rng.standard_normal((nz, ny, nx)).clip(-2, 2))).astype(np.float32)
        vs = (vp / rng.uniform(1.7, 2.0, vp.shape)).astype(np.float32)
        rho = synth.gardner(vp)
        self.vp, self.vs, self.rho = vp, vs, rho
        self.nt, self.dt, self.order, self.precision = nt, dt, order, precision
        m = ModelElastic3D(nx, ny, nz, lpml, dx, dx, dx, 0.0, 0.0, 0.0, fs, precision)
        m.createModel()
        m.Vp[:], m.Vs[:], m.R[:] = vp, vs, rho
        self.model = m
        self.scoords = np.array([[0.47 * nx * dx + 1.3, 0.52 * ny * dx - 2.1, 0.4 * nz * dx + 0.7]])
        self.gcoords = np.stack([np.linspace(15.3, (nx - 3) * dx, nrec), np.linspace(20.9, (ny - 4) * dx, nrec),
                                 np.full(nrec, 12.6)], 1)
        src = Data3D(1, nt, dt, 0.0, precision)
        src.scoords[:] = self.scoords
        src.data[:] = synth.ricker(nt, dt, 25.0, abi.real_dtype(precision))[None, :]
        src.setField(sfield)
        src.makeMap(m, 0)
        rec = Data3D(nrec, nt, dt, 0.0, precision)
        rec.gcoords[:] = self.gcoords
        rec.setField(rfield)
        rec.makeMap(m, 1)
        self.src, self.rec = src, rec
        self.sfield, self.rfield = sfield, rfield
        self.pb = api.Problem3D(nx, ny, nz, dx, dx, dx, lpml, order, fs, dt, nt, vp, rho, vs)

    def gpu_traces(self, precision=None):
        prec = self.precision if precision is None else precision
        self.rec.data[:] = 0
        mod = ModellingElastic3D(self.model, self.src, self.order, 1, precision=prec)
        {abi.PRESSURE: mod.setRecP, abi.VX: mod.setRecVx, abi.VY: mod.setRecVy, abi.VZ: mod.setRecVz}[self.rfield](self.rec)
        assert mod.run() == 1
        return self.rec.data.copy()

    def ref_traces(self):
        return api.ref_modelling_e3d(self.pb, self.scoords, self.src.data.astype(np.float32), self.sfield,
                                     self.gcoords, self.rfield)


@pytest.mark.parametrize("sfield,rfield", [(abi.PRESSURE, abi.PRESSURE), (abi.PRESSURE, abi.VX), (abi.VY, abi.VY),
                                           (abi.VZ, abi.VZ), (abi.VX, abi.PRESSURE)])
@pytest.mark.parametrize("fs", [0, 1])
def test_elastic3d_gather_exact_equals_reference(require_gpu, sfield, rfield, fs):
    c = Case3D(sfield=sfield, rfield=rfield, fs=fs)
    gpu, ref = c.gpu_traces(), c.ref_traces()
    assert np.abs(ref).max() > 0
    assert np.array_equal(gpu, ref), f"max abs diff {np.abs(gpu - ref).max()}"


@pytest.mark.parametrize("order", [3, 8])
def test_elastic3d_wavefields_exact_equal_reference(require_gpu, order):
    c = Case3D(order=order, nt=40, fs=1)
    p = Plan([c.model], [c.src], [c.rec], c.order, abi.F32_EXACT)
    p.run(0, 40)
    shape = (c.model.getNz_pml(), c.model.getNy_pml(), c.model.getNx_pml())
    ref = api.ref_steps_e3d(c.pb, c.scoords, c.src.data.astype(np.float32), c.sfield, 40)
    for k, f in enumerate(E3_FIELDS):
        got = p.read_field(0, f, shape)
        assert np.abs(ref[k]).max() > 0, k
        assert np.array_equal(got, ref[k]), f"field {f}: max abs diff {np.abs(got - ref[k]).max()}"
    p.close()


def test_elastic3d_fast_within_fp32(require_gpu):
    c = Case3D(nt=80, rfield=abi.VZ)
    ref = c.ref_traces()
    assert rel_l2(c.gpu_traces(abi.F32_FAST), ref) <= FAST_TOL


def test_elastic3d_pressure_needs_factor(require_gpu):
    """The C ABI refuses elastic 3D pressure receivers without the recording divisor."""
    import ctypes as C
    from rockseis_b200.rockseis import make_config, make_shot
    c = Case3D(rfield=abi.PRESSURE)
    cfg = make_config(c.model, c.order, c.nt, c.dt, abi.F32_EXACT)
    keep: list = []
    shot = make_shot(c.model, c.src, c.rec, keep)
    shot.rec_factor = None
    st = abi.lib.rsgpu_modelling(C.byref(cfg), 1, C.byref(shot))
    assert st == abi.ERR_ARG

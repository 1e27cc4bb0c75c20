"""GPU parity of the 3D acoustic propagator (through the C ABI) against the oracle.

Exact arithmetic must reproduce the oracle (itself pinned bit-exact against the
reference's ModellingAcoustic3D::run) bit for bit, for every source/receiver
field, with and without a free surface, at reduced orders, across z-chunk
boundaries of the z-marching kernels, and for shots with different windows
batched in one plan.  FAST mode is held to relative L2 <= 1e-5.
"""
import numpy as np
import pytest

from oracle import api
from rockseis_b200 import abi, synth
from rockseis_b200.rockseis import Data3D, ModelAcoustic3D, ModellingAcoustic3D, modelling_batch
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu


class Case3D:
    def __init__(self, nx=41, ny=37, nz=33, lpml=8, dx=10.0, dt=1e-3, nt=120, order=8, fs=0, seed=5,
                 sfield=abi.PRESSURE, rfield=abi.PRESSURE, scoord=(203.3, 171.9, 142.2), precision=abi.F32_EXACT):
        self.nt, self.dt, self.order, self.precision = nt, dt, order, precision
        vp = np.stack([synth.layered_vp(nx, nz, dx, 1500, 3000, 4, 0.05, 60, seed + k) for k in range(ny)], 1)
        vp = np.ascontiguousarray(vp.astype(abi.real_dtype(precision)))
        rho = synth.gardner(vp)
        m = ModelAcoustic3D(nx, ny, nz, lpml, dx, dx, dx, 0.0, 0.0, 0.0, fs, precision)
        m.createModel()
        m.Vp[:], m.R[:] = vp, rho
        self.model = m
        src = Data3D(1, nt, dt, 0.0, precision)
        src.scoords[:] = [scoord]
        src.data[:] = synth.ricker(nt, dt, 25.0, abi.real_dtype(precision))[None, :]
        src.setField(sfield)
        src.makeMap(m, 0)
        n = 9
        gc = np.stack([np.linspace(15.0, (nx - 2) * dx, n), np.linspace(11.0, (ny - 2) * dx, n), np.full(n, 12.6)], 1)
        rec = Data3D(n, nt, dt, 0.0, precision)
        rec.gcoords[:] = gc
        rec.setField(rfield)
        rec.makeMap(m, 1)
        self.src, self.rec = src, rec
        self.pb = api.Problem3D(nx, ny, nz, dx, dx, dx, lpml, order, fs, dt, nt, vp, rho)
        self.tab = np.zeros(12 * lpml, np.float32)
        abi.check(abi.lib.rsgpu_pml_tables(lpml, dt, abi.F32_EXACT, self.tab.ctypes.data))

    def oracle(self):
        s, r = self.src, self.rec
        return api.orc_modelling_a3d(self.pb, [a.astype(np.float32) for a in self.model.padded()], self.tab, s.smap,
                                     s.sshift, s.data.astype(np.float32), s.field, r.gmap, r.gshift, r.field)

    def gpu(self, precision=None, zchunk=0):
        self.rec.data[:] = 0
        mod = ModellingAcoustic3D(self.model, self.src, self.order, 1,
                                  precision=self.precision if precision is None else precision)
        mod.zchunk = zchunk
        {abi.PRESSURE: mod.setRecP, abi.VX: mod.setRecVx, abi.VY: mod.setRecVy, abi.VZ: mod.setRecVz}[self.rec.field](
            self.rec)
        assert mod.run() == 1
        return self.rec.data.copy()


@pytest.mark.parametrize("fs", [0, 1])
@pytest.mark.parametrize("sfield,rfield", [(abi.PRESSURE, abi.PRESSURE), (abi.PRESSURE, abi.VZ),
                                           (abi.VX, abi.PRESSURE), (abi.VY, abi.VY)])
def test_acoustic3d_exact_bitwise(require_gpu, fs, sfield, rfield):
    c = Case3D(fs=fs, sfield=sfield, rfield=rfield)
    ref = c.oracle()
    got = c.gpu()
    assert np.abs(ref).max() > 0
    assert np.array_equal(got, ref), f"max abs diff {np.abs(got - ref).max()}"


@pytest.mark.parametrize("order", [2, 4, 8])
@pytest.mark.parametrize("zchunk", [7, 16, 0])
def test_acoustic3d_orders_and_z_chunks_bitwise(require_gpu, order, zchunk):
    c = Case3D(order=order, nt=80)
    ref = c.oracle()
    got = c.gpu(zchunk=zchunk)
    assert np.array_equal(got, ref), f"max abs diff {np.abs(got - ref).max()}"


def test_acoustic3d_batched_windows_bitwise(require_gpu):
    cases = [Case3D(nx=41, ny=37, nz=33, seed=5), Case3D(nx=29, ny=45, nz=38, seed=9, scoord=(120.4, 300.8, 97.0))]
    refs = [c.oracle() for c in cases]
    for c in cases:
        c.rec.data[:] = 0
    modelling_batch([c.model for c in cases], [c.src for c in cases], [c.rec for c in cases], 8)
    for c, ref in zip(cases, refs):
        assert np.array_equal(c.rec.data, ref), f"max abs diff {np.abs(c.rec.data - ref).max()}"


def test_acoustic3d_fast_within_fp32_tolerance(require_gpu):
    c = Case3D()
    ref = c.oracle()
    got = c.gpu(precision=abi.F32_FAST)
    assert rel_l2(got, ref) <= 1e-5


# ---------------------------------------------------------------- RtmAcoustic3D::run_optimal
def rtm_inputs(c):
    """Data to migrate: the oracle's pressure gather of the case's shot."""
    return c.oracle().astype(np.float32)


def oracle_rtm3d(c, data, nhx, nhy, nhz):
    s, r = c.src, c.rec
    return api.orc_rtm_a3d(c.pb, [a.astype(np.float32) for a in c.model.padded()], c.tab, s.smap, s.sshift,
                           s.data.astype(np.float32), r.gmap, r.gshift, data, nhx, nhy, nhz)


def gpu_rtm3d(c, data, nhx, nhy, nhz, ncheck=5, precision=None, ckpt=abi.CKPT_NATIVE, accum=abi.ACCUM_REFERENCE):
    from rockseis_b200.rockseis import Image3D, RtmAcoustic3D
    prec = c.precision if precision is None else precision
    c.rec.data = np.ascontiguousarray(data.astype(abi.real_dtype(prec)))
    img = Image3D("pimage", c.model, nhx, nhy, nhz, prec)
    r = RtmAcoustic3D(c.model, img, c.src, c.rec, c.order, 1, precision=prec)
    r.setNcheck(ncheck)
    r.setCheckpointPrecision(ckpt)
    r.setAccumulation(accum)
    assert r.run_optimal() == 1
    return img.getImagedata()


@pytest.mark.parametrize("lags,ncheck", [((1, 1, 1), 5), ((3, 1, 3), 9), ((1, 3, 1), 120)])
def test_rtm3d_exact_bitwise(require_gpu, lags, ncheck):
    c = Case3D(nx=29, ny=27, nz=25)
    data = rtm_inputs(c)
    ref = oracle_rtm3d(c, data, *lags)
    got = gpu_rtm3d(c, data, *lags, ncheck=ncheck)
    assert np.abs(ref).max() > 0
    assert np.array_equal(got, ref), f"max abs diff {np.abs(got - ref).max()}"


def test_rtm3d_batched_windows_bitwise(require_gpu):
    from rockseis_b200.rockseis import Image3D, RtmAcoustic3D, rtm_image_batch
    cases = [Case3D(nx=29, ny=27, nz=25, seed=5), Case3D(nx=23, ny=31, nz=27, seed=9, scoord=(120.4, 200.8, 97.0))]
    jobs, refs = [], []
    for c in cases:
        data = rtm_inputs(c)
        refs.append(oracle_rtm3d(c, data, 1, 1, 1))
        c.rec.data = np.ascontiguousarray(data)
        r = RtmAcoustic3D(c.model, Image3D("pimage", c.model, 1, 1, 1), c.src, c.rec, c.order, 1)
        r.setNcheck(6)
        jobs.append(r)
    rtm_image_batch(jobs)
    for r, ref in zip(jobs, refs):
        assert np.array_equal(r.pimage.getImagedata(), ref)


def test_rtm3d_fast_fp16_checkpoints_within_tolerance(require_gpu):
    c = Case3D(nx=29, ny=27, nz=25)
    data = rtm_inputs(c)
    ref = oracle_rtm3d(c, data, 1, 1, 1)
    got = gpu_rtm3d(c, data, 1, 1, 1, ncheck=8, precision=abi.F32_FAST, ckpt=abi.CKPT_F16, accum=abi.ACCUM_F64)
    err = rel_l2(got, ref)
    print(f"3D RTM image, FMA + FP16 checkpoints + FP64 accumulation vs exact: {err:.3g}")
    assert err <= 1e-3


# ---------------------------------------------------------------- FwiAcoustic3D::run_optimal
def fwi3d_case(**kw):
    c = Case3D(nx=27, ny=25, nz=23, nt=110, **kw)
    # observed data: the oracle's gather in a model with a slow block
    vt = c.pb.vp.copy()
    vt[8:14, 7:13, 9:16] *= 0.92
    from rockseis_b200.rockseis import ModelAcoustic3D
    m = c.model
    mt = ModelAcoustic3D(m.nx, m.ny, m.nz, m.lpml, m.dx, m.dy, m.dz, 0.0, 0.0, 0.0, m.fs)
    mt.createModel()
    mt.Vp[:], mt.R[:] = vt, c.pb.rho
    pbt = api.Problem3D(m.nx, m.ny, m.nz, m.dx, m.dy, m.dz, m.lpml, c.order, m.fs, c.dt, c.nt, vt, c.pb.rho)
    s, r = c.src, c.rec
    c.obs = api.orc_modelling_a3d(pbt, mt.padded(), c.tab, s.smap, s.sshift, s.data.astype(np.float32), 0, r.gmap,
                                  r.gshift, 0)
    return c


def oracle_fwi3d(c, misfit=0):
    s, r = c.src, c.rec
    return api.orc_fwi_a3d(c.pb, [a.astype(np.float32) for a in c.model.padded()], c.tab, s.smap, s.sshift,
                           s.data.astype(np.float32), r.gmap, r.gshift, c.obs, misfit)


def gpu_fwi3d(c, ncheck=6, precision=None, ckpt=abi.CKPT_NATIVE, accum=abi.ACCUM_REFERENCE, misfit=0):
    from rockseis_b200.rockseis import Data3D, FwiAcoustic3D, Image3D
    prec = c.precision if precision is None else precision
    c.rec.data = np.ascontiguousarray(c.obs.astype(abi.real_dtype(prec)))
    f = FwiAcoustic3D(c.model, c.src, c.rec, c.order, 1, precision=prec)
    f.setNcheck(ncheck)
    f.setCheckpointPrecision(ckpt)
    f.setAccumulation(accum)
    f.setMisfit_type(misfit)
    f.setVpgrad(Image3D("vp", c.model, 1, 1, 1, prec))
    f.setRhograd(Image3D("rho", c.model, 1, 1, 1, prec))
    f.setWavgrad(Data3D(c.src.ntrace, c.nt, c.dt, 0.0, prec))
    f.setDatamodP(Data3D(c.rec.ntrace, c.nt, c.dt, 0.0, prec))
    f.setDataresP(Data3D(c.rec.ntrace, c.nt, c.dt, 0.0, prec))
    assert f.run_optimal() == 1
    return dict(vpgrad=f.vpgrad.getImagedata()[0, 0, 0], rhograd=f.rhograd.getImagedata()[0, 0, 0],
                wavgrad=f.wavgrad.data, datamod=f.datamodP.data, datares=f.dataresP.data, misfit=f.getMisfit())


@pytest.mark.parametrize("ncheck", [4, 110])
def test_fwi3d_exact_bitwise(require_gpu, ncheck):
    c = fwi3d_case()
    ref = oracle_fwi3d(c)
    got = gpu_fwi3d(c, ncheck=ncheck)
    for k in ("vpgrad", "rhograd", "wavgrad", "datamod", "datares"):
        assert np.abs(ref[k]).max() > 0, k
        assert np.array_equal(got[k], ref[k]), f"{k}: max abs diff {np.abs(got[k] - ref[k]).max()}"
    assert got["misfit"] == ref["misfit"]


def test_fwi3d_fast_fp16_checkpoints_close_to_exact(require_gpu):
    c = fwi3d_case()
    ref = oracle_fwi3d(c)
    got = gpu_fwi3d(c, ncheck=8, precision=abi.F32_FAST, ckpt=abi.CKPT_F16, accum=abi.ACCUM_F64)
    err = {k: rel_l2(got[k], ref[k]) for k in ("vpgrad", "rhograd", "wavgrad")}
    print(f"3D FWI gradient, FMA + FP16 checkpoints + FP64 accumulation vs exact: {err}")
    assert max(err.values()) <= 1e-3, err


def test_fwi3d_correlation_misfit_exact_bitwise(require_gpu):
    c = fwi3d_case()
    ref = oracle_fwi3d(c, misfit=abi.MISFIT_CORRELATION)
    got = gpu_fwi3d(c, ncheck=5, misfit=abi.MISFIT_CORRELATION)
    for k in ("vpgrad", "rhograd", "wavgrad", "datamod", "datares"):
        assert np.abs(ref[k]).max() > 0, k
        assert np.array_equal(got[k], ref[k]), f"{k}: max abs diff {np.abs(got[k] - ref[k]).max()}"
    assert got["misfit"] == ref["misfit"] and got["misfit"] < 0


@pytest.mark.parametrize("misfit", [2, 3])
def test_fwi3d_adaptive_misfit_bitwise(require_gpu, misfit):
    # FwiAcoustic3D with ADAPTIVE_GAUSS / ADAPTIVE_LINEAR: no residual clip in 3D
    import os
    c = fwi3d_case()
    if api.ref_available():
        ref = api.ref_fwi_a3d(c.pb, c.src.scoords, c.src.data.astype(np.float32), c.rec.gcoords,
                              c.obs.astype(np.float32), 5, misfit=misfit)
    else:
        g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "adaptive.npz"))
        assert np.array_equal(c.obs.astype(np.float32), g["a3d_obs"])
        name = {2: "gauss", 3: "linear"}[misfit]
        ref = {k: g[f"a3d_{name}_{k}"] for k in ("vpgrad", "rhograd", "wavgrad", "datares", "misfit")}
        ref["datamod"] = g["a3d_datamod"]
    got = gpu_fwi3d(c, ncheck=5, misfit=misfit)
    for k in ("vpgrad", "rhograd", "wavgrad", "datamod", "datares"):
        assert np.abs(ref[k]).max() > 0, k
        assert np.array_equal(got[k], ref[k]), f"{k}: max abs diff {np.abs(got[k] - ref[k]).max()}"
    assert got["misfit"] == float(ref["misfit"])


@pytest.mark.parametrize("snapinc,lags", [(4, (1, 1, 1)), (3, (3, 1, 3)), (1, (1, 3, 1))])
def test_rtm3d_full_snapshots_bitwise(require_gpu, snapinc, lags):
    # RtmAcoustic3D::run: the P interior every snapinc steps, correlated at the adjoint
    # times shifted by enddiff (nt = 120: enddiff 3, 2, 0)
    import os
    from rockseis_b200.rockseis import Image3D, RtmAcoustic3D
    c = Case3D(nx=29, ny=27, nz=25)
    data = rtm_inputs(c)
    if api.ref_available():
        ref = api.ref_rtm_a3d(c.pb, c.src.scoords, c.src.data.astype(np.float32), c.rec.gcoords, data, 0, *lags,
                              full_snapinc=snapinc)
    elif (snapinc, lags) == (4, (1, 1, 1)):
        g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "snapfull.npz"))
        assert np.array_equal(data, g["rtm3d_data"])
        ref = g["rtm3d_s4"]
    else:
        pytest.skip("reference library not built")
    c.rec.data = np.ascontiguousarray(data)
    img = Image3D("pimage", c.model, *lags)
    r = RtmAcoustic3D(c.model, img, c.src, c.rec, c.order, snapinc)
    assert r.run() == 1
    got = img.getImagedata()
    assert np.abs(ref).max() > 0
    assert np.array_equal(got, ref), f"max abs diff {np.abs(got - ref).max()}"

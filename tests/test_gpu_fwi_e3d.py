"""GPU parity of the elastic 3D FWI gradient (FwiElastic3D::run_optimal).

The checker is the unmodified reference library (oracle/_ref/librsref.so) running
FwiElastic3D<float>::run_optimal (lib/fwi.cpp:6770-6990) in core.  With exact
arithmetic and lossless checkpoints every output -- vp/vs/rho gradients, wavelet
gradient, modelled data and residuals of the Ux, Uy and Uz sets, misfit -- must
equal the reference bit for bit, for any Revolve snapshot count, with and without
the free surface, for every source type and for a batch of shots with different
windows.  FMA arithmetic with 16-bit checkpoints and FP64 accumulation is held to
bounds against the FP64 GPU gradient.
"""
import numpy as np
import pytest

from oracle import api
from rockseis_b200 import abi, synth
from rockseis_b200.rockseis import Data3D, FwiElastic3D, Image3D, ModelElastic3D, fwi_gradient_batch
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu

AMP = 1e8   # source scale that keeps the gradients' products clear of float subnormals


@pytest.fixture(scope="module", autouse=True)
def need_reference():
    if not api.ref_available():
        pytest.skip("reference library oracle/_ref not built")


class Fwi3DCase:
    """Starting model, source, Ux/Uy/Uz receiver sets, and observed data modelled
    by the reference in a model with a slow block."""

    def __init__(self, nx=22, ny=18, nz=20, lpml=6, dx=10.0, dt=1e-3, nt=70, fs=0, seed=11, sfield=abi.PRESSURE,
                 scoord=(104.3, 91.7, 62.2), nrec=8, precision=abi.F32_EXACT, amp=AMP):
        rng = np.random.default_rng(seed)
        self.nt, self.dt, self.precision, self.sfield = nt, dt, precision, sfield
        t = abi.real_dtype(precision)
        vp = 2000.0 + 900.0 * np.linspace(0, 1, nz)[:, None, None] * np.ones((1, ny, nx))
        vp = (vp * (1 + 0.03 * rng.standard_normal((nz, ny, nx)).clip(-2, 2))).astype(np.float32)
        vs = (vp / rng.uniform(1.7, 2.0, vp.shape)).astype(np.float32)
        rho = synth.gardner(vp)
        vt = vp.copy()
        vt[nz // 2: nz // 2 + 5, ny // 3: ny // 3 + 6, nx // 3: nx // 3 + 7] *= 0.92
        self.vp, self.vs, self.rho = vp, vs, rho
        m = ModelElastic3D(nx, ny, nz, lpml, dx, dx, dx, 0.0, 0.0, 0.0, fs, precision)
        m.createModel()
        m.Vp[:], m.Vs[:], m.R[:] = vp, vs, rho
        self.model = m
        self.scoords = np.array([scoord])
        src = Data3D(1, nt, dt, 0.0, precision)
        src.scoords[:] = self.scoords
        src.data[:] = amp * synth.ricker(nt, dt, 25.0, t)[None, :]
        src.setField(sfield)
        src.makeMap(m, 0)
        self.src = src
        self.gcoords = np.stack([np.linspace(-12.0, (nx - 2) * dx, nrec), np.linspace(15.5, (ny - 3) * dx, nrec),
                                 np.full(nrec, 14.2)], 1)         # the first receiver lies off the grid
        self.recs = []
        for f in (abi.VX, abi.VY, abi.VZ):
            r = Data3D(nrec, nt, dt, 0.0, precision)
            r.gcoords[:] = self.gcoords
            r.setField(f)
            r.makeMap(m, 1)
            self.recs.append(r)
        self.pb = api.Problem3D(nx, ny, nz, dx, dx, dx, lpml, 8, fs, dt, nt, vp, rho, vs)
        pbt = api.Problem3D(nx, ny, nz, dx, dx, dx, lpml, 8, fs, dt, nt, vt, rho, vs)
        wav32 = (amp * synth.ricker(nt, dt, 25.0)[None, :]).astype(np.float32)
        self.obs = [api.ref_modelling_e3d(pbt, self.scoords, wav32, sfield, self.gcoords, f).astype(t)
                    for f in (abi.VX, abi.VY, abi.VZ)]

    def reference(self, ncheck):
        return api.ref_fwi_e3d(self.pb, self.scoords, self.src.data.astype(np.float32), self.sfield, self.gcoords,
                               [o.astype(np.float32) for o in self.obs], ncheck)


def make_job(c, precision=None, ncheck=7, ckpt=abi.CKPT_NATIVE, accum=abi.ACCUM_REFERENCE):
    prec = c.precision if precision is None else precision
    for r, o in zip(c.recs, c.obs):
        r.data = np.ascontiguousarray(o.astype(abi.real_dtype(prec)))
    f = FwiElastic3D(c.model, c.src, c.recs[0], c.recs[1], c.recs[2], 8, 1, precision=prec)
    f.setNcheck(ncheck)
    f.setCheckpointPrecision(ckpt)
    f.setAccumulation(accum)
    f.setVpgrad(Image3D("vp", c.model, 1, 1, 1, prec))
    f.setVsgrad(Image3D("vs", c.model, 1, 1, 1, prec))
    f.setRhograd(Image3D("rho", c.model, 1, 1, 1, prec))
    f.setWavgrad(Data3D(c.src.ntrace, c.nt, c.dt, 0.0, prec))
    n = c.recs[0].ntrace
    mk = lambda: Data3D(n, c.nt, c.dt, 0.0, prec)  # noqa: E731
    f.setDatamodUx(mk()); f.setDatamodUy(mk()); f.setDatamodUz(mk())
    f.setDataresUx(mk()); f.setDataresUy(mk()); f.setDataresUz(mk())
    return f


def outputs(f):
    return dict(vpgrad=f.vpgrad.getImagedata()[0, 0, 0], vsgrad=f.vsgrad.getImagedata()[0, 0, 0],
                rhograd=f.rhograd.getImagedata()[0, 0, 0], wavgrad=f.wavgrad.data,
                datamod=np.stack([f.datamodUx.data, f.datamodUy.data, f.datamodUz.data]),
                datares=np.stack([f.dataresUx.data, f.dataresUy.data, f.dataresUz.data]), misfit=f.getMisfit())


def assert_same(got, ref):
    for k in ("vpgrad", "vsgrad", "rhograd", "wavgrad", "datamod", "datares"):
        assert np.abs(ref[k]).max() > 0, k
        assert np.array_equal(got[k], ref[k]), f"{k}: max abs diff {np.abs(got[k] - ref[k]).max()}"
    assert got["misfit"] == ref["misfit"]


@pytest.mark.parametrize("ncheck", [3, 8, 70])
def test_elastic3d_fwi_exact_equals_reference(require_gpu, ncheck):
    c = Fwi3DCase()
    ref = c.reference(ncheck)
    f = make_job(c, ncheck=ncheck)
    assert f.run_optimal() == 1
    assert_same(outputs(f), ref)


@pytest.mark.parametrize("fs,sfield", [(1, abi.PRESSURE), (0, abi.VX), (1, abi.VY), (0, abi.VZ)])
def test_elastic3d_fwi_free_surface_and_source_fields(require_gpu, fs, sfield):
    c = Fwi3DCase(fs=fs, sfield=sfield, nt=50)
    ref = c.reference(6)
    f = make_job(c, ncheck=6)
    f.run_optimal()
    assert_same(outputs(f), ref)


def test_elastic3d_fwi_batched_equals_reference(require_gpu):
    cases = [Fwi3DCase(seed=3), Fwi3DCase(nx=26, ny=15, nz=19, seed=4, scoord=(131.0, 70.4, 44.9))]
    refs = [c.reference(5) for c in cases]
    jobs = [make_job(c, ncheck=5) for c in cases]
    fwi_gradient_batch(jobs)
    for f, ref in zip(jobs, refs):
        assert_same(outputs(f), ref)


# FP16 keeps 11 significant bits: the north-star bound of 1e-3 holds.  BF16 keeps 8
# (rounding up to 2^-9 relative per stored value), so a restored wavefield carries
# about 1e-3 relative error into the gradient by itself; it is held to 3e-3.
@pytest.mark.parametrize("ckpt,tol", [(abi.CKPT_F16, 1e-3), (abi.CKPT_BF16, 3e-3)])
def test_elastic3d_fwi_16bit_checkpoints_fp64_accumulation(require_gpu, ckpt, tol):
    c64 = Fwi3DCase(precision=abi.F64)
    f64 = make_job(c64, ncheck=10, accum=abi.ACCUM_F64)
    f64.run_optimal()
    ref64 = outputs(f64)
    exact = Fwi3DCase().reference(10)
    c = Fwi3DCase()
    f = make_job(c, precision=abi.F32_FAST, ncheck=10, ckpt=ckpt, accum=abi.ACCUM_F64)
    f.run_optimal()
    got = outputs(f)
    for k in ("vpgrad", "vsgrad", "rhograd"):
        base, err = rel_l2(exact[k], ref64[k]), rel_l2(got[k], ref64[k])
        print(f"{k}: FMA + 16-bit checkpoints ({ckpt}) {err:.3g}, reference float {base:.3g} (vs FP64)")
        assert err <= tol, k
    assert abs(got["misfit"] - ref64["misfit"]) <= 1e-3 * abs(ref64["misfit"])


def test_elastic3d_fwi_lossless_fast_within_fp32(require_gpu):
    # FMA arithmetic, lossless checkpoints: as close to FP64 as the reference's float
    c64 = Fwi3DCase(precision=abi.F64)
    f64 = make_job(c64, ncheck=10, accum=abi.ACCUM_F64)
    f64.run_optimal()
    ref64 = outputs(f64)
    exact = Fwi3DCase().reference(10)
    f = make_job(Fwi3DCase(), precision=abi.F32_FAST, ncheck=10, accum=abi.ACCUM_F64)
    f.run_optimal()
    got = outputs(f)
    for k in ("vpgrad", "vsgrad", "rhograd"):
        base, err = rel_l2(exact[k], ref64[k]), rel_l2(got[k], ref64[k])
        print(f"{k}: FMA, lossless checkpoints {err:.3g}, reference float {base:.3g} (vs FP64)")
        assert err <= max(2.0 * base, 1e-5), k


def test_elastic3d_fwi_16bit_checkpoints_of_subnormal_tails(require_gpu):
    # unit source amplitude: C-PML memory blocks whose largest value is subnormal are
    # checkpointed; their scale must stay finite (the gradient stays finite and close)
    c = Fwi3DCase(amp=1.0)
    lossless = make_job(c, precision=abi.F32_FAST, ncheck=6, accum=abi.ACCUM_F64)
    lossless.run_optimal()
    ref = outputs(lossless)
    for ckpt in (abi.CKPT_F16, abi.CKPT_BF16):
        f = make_job(Fwi3DCase(amp=1.0), precision=abi.F32_FAST, ncheck=6, ckpt=ckpt, accum=abi.ACCUM_F64)
        f.run_optimal()
        got = outputs(f)
        for k in ("vpgrad", "vsgrad", "rhograd"):
            assert np.isfinite(got[k]).all(), (ckpt, k)
            assert rel_l2(got[k], ref[k]) < 5e-3, (ckpt, k, rel_l2(got[k], ref[k]))

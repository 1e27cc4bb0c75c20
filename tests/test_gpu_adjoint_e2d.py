"""GPU parity of the elastic 2D FWI gradient (FwiElastic2D::run_optimal).

The adjoint propagation uses the adjoint elastic kernels (backwardstepVelocity /
backwardstepStress, lib/waves.cpp:1738-2080); with exact arithmetic and lossless
checkpoints every output -- vp/vs/rho gradients, wavelet gradient, modelled data
and residuals of the P, Ux and Uz sets, misfit -- must equal the oracle (pinned
bit-exact against the reference) bit for bit, for any Revolve snapshot count.
"""
import numpy as np
import pytest

from rockseis_b200 import abi
from rockseis_b200.rockseis import Data2D, FwiElastic2D, Image2D, fwi_gradient_batch
from tests.cases import ElasticFwiCase, rel_l2

pytestmark = pytest.mark.gpu


def make_job(c, precision=None, ncheck=7, ckpt=abi.CKPT_NATIVE, accum=abi.ACCUM_REFERENCE):
    prec = c.precision if precision is None else precision
    for r, o in zip(c.recs, c.obs):
        r.data = np.ascontiguousarray(o.astype(abi.real_dtype(prec)))
    f = FwiElastic2D(c.model, c.src, c.recs[0], c.recs[1], c.recs[2], 8, 1, precision=prec)
    f.setNcheck(ncheck)
    f.setCheckpointPrecision(ckpt)
    f.setAccumulation(accum)
    f.setVpgrad(Image2D("vp", c.model, 1, 1, prec))
    f.setVsgrad(Image2D("vs", c.model, 1, 1, prec))
    f.setRhograd(Image2D("rho", c.model, 1, 1, prec))
    f.setWavgrad(Data2D(c.src.ntrace, c.nt, c.dt, 0.0, prec))
    n = c.recs[0].ntrace
    mk = lambda: Data2D(n, c.nt, c.dt, 0.0, prec)  # noqa: E731
    f.setDatamodP(mk()); f.setDatamodUx(mk()); f.setDatamodUz(mk())
    f.setDataresP(mk()); f.setDataresUx(mk()); f.setDataresUz(mk())
    return f


def outputs(f):
    return dict(vpgrad=f.vpgrad.getImagedata()[0, 0], vsgrad=f.vsgrad.getImagedata()[0, 0],
                rhograd=f.rhograd.getImagedata()[0, 0], wavgrad=f.wavgrad.data,
                datamod=np.stack([f.datamodP.data, f.datamodUx.data, f.datamodUz.data]),
                datares=np.stack([f.dataresP.data, f.dataresUx.data, f.dataresUz.data]), misfit=f.getMisfit())


def assert_same(got, ref):
    for k in ("vpgrad", "vsgrad", "rhograd", "wavgrad", "datamod", "datares"):
        assert np.abs(ref[k]).max() > 0, k
        assert np.array_equal(got[k], ref[k]), f"{k}: max abs diff {np.abs(got[k] - ref[k]).max()}"
    assert got["misfit"] == ref["misfit"]


@pytest.mark.parametrize("ncheck", [3, 7, 250])
def test_elastic_fwi_exact_bitwise(require_gpu, ncheck):
    c = ElasticFwiCase()
    ref = c.oracle()
    f = make_job(c, ncheck=ncheck)
    assert f.run_optimal() == 1
    assert_same(outputs(f), ref)


@pytest.mark.parametrize("fs,sfield", [(1, abi.PRESSURE), (0, abi.VX), (1, abi.VZ)])
def test_elastic_fwi_free_surface_and_source_fields(require_gpu, fs, sfield):
    c = ElasticFwiCase(fs=fs, sfield=sfield, nrec=22, rx0=-14.0)    # first receiver off the grid
    ref = c.oracle()
    f = make_job(c, ncheck=9)
    f.run_optimal()
    assert_same(outputs(f), ref)


def test_elastic_fwi_batched_bitwise(require_gpu):
    cases = [ElasticFwiCase(seed=7), ElasticFwiCase(nx=70, nz=41, seed=8, scoord=(150.2, 21.9))]
    refs = [c.oracle() for c in cases]
    jobs = [make_job(c, ncheck=5) for c in cases]
    fwi_gradient_batch(jobs)
    for f, ref in zip(jobs, refs):
        assert_same(outputs(f), ref)


def test_elastic_fwi_fast_mode_as_accurate_as_reference_float(require_gpu):
    c64 = ElasticFwiCase(precision=abi.F64)
    f64 = make_job(c64, ncheck=10, accum=abi.ACCUM_F64)
    f64.run_optimal()
    ref64 = outputs(f64)
    exact = ElasticFwiCase().oracle()
    c = ElasticFwiCase()
    f = make_job(c, precision=abi.F32_FAST, ncheck=10, ckpt=abi.CKPT_F16, accum=abi.ACCUM_F64)
    f.run_optimal()
    got = outputs(f)
    for k in ("vpgrad", "vsgrad", "rhograd"):
        base, err = rel_l2(exact[k], ref64[k]), rel_l2(got[k], ref64[k])
        print(f"{k}: FMA+FP16 checkpoints {err:.3g}, reference float {base:.3g} (vs FP64)")
        assert err <= max(1.25 * base + 1e-5, 1e-3), k


@pytest.mark.parametrize("ncheck", [4, 9])
def test_elastic_fwi_correlation_misfit_exact_bitwise(require_gpu, ncheck):
    # CORRELATION misfit of P, Ux and Uz with the reference's x/z and P residual clips
    c = ElasticFwiCase()
    ref = c.oracle(misfit=abi.MISFIT_CORRELATION)
    f = make_job(c, ncheck=ncheck)
    f.setMisfit_type(abi.MISFIT_CORRELATION)
    assert f.run_optimal() == 1
    got = outputs(f)
    assert_same(got, ref)
    assert got["misfit"] < 0
    assert (ref["datares"][0] == 0).mean() >= 0.03 and (ref["datares"][1] == 0).any()


# ---------------------------------------------------------------- ADAPTIVE misfits (FwiElastic2D)
def adaptive_reference(c, misfit, ncheck=7):
    """FwiElastic2D::run_optimal with an ADAPTIVE misfit: the reference library where
    oracle/_ref is built, else the committed outputs (tests/golden/make_golden_adaptive.py)."""
    import os
    from oracle import api
    obs3 = [o.astype(np.float32) for o in c.obs]
    if api.ref_available():
        return api.ref_fwi_e2d(c.pb, c.src.scoords, c.src.data.astype(np.float32), c.sfield, c.recs[0].gcoords, obs3,
                               ncheck, misfit=misfit)
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "adaptive.npz"))
    assert ncheck == 7 and np.array_equal(np.stack(obs3), g["e2d_obs"])
    name = {2: "gauss", 3: "linear", 4: "single"}[misfit]
    out = {k: g[f"e2d_{name}_{k}"] for k in ("vpgrad", "vsgrad", "rhograd", "wavgrad", "datares")}
    out["datamod"] = g["e2d_datamod"]
    out["misfit"] = float(g[f"e2d_{name}_misfit"])
    return out


@pytest.mark.parametrize("misfit", [abi.MISFIT_ADAPTIVE_GAUSS, abi.MISFIT_ADAPTIVE_LINEAR,
                                    abi.MISFIT_ADAPTIVE_SINGLE])
def test_elastic_fwi_adaptive_misfit_bitwise(require_gpu, misfit):
    # Ux and Uz shaped separately and clipped together (GAUSS, LINEAR) or joined end to
    # end under one filter (SINGLE); the P residual is zero
    c = ElasticFwiCase()
    ref = adaptive_reference(c, misfit)
    f = make_job(c, ncheck=7)
    f.setMisfit_type(misfit)
    assert f.run_optimal() == 1
    got = outputs(f)
    for k in ("vpgrad", "vsgrad", "rhograd", "wavgrad", "datamod", "datares"):
        assert np.abs(ref[k]).max() > 0, k
        assert np.array_equal(got[k], ref[k]), f"{k}: max abs diff {np.abs(got[k] - ref[k]).max()}"
    assert got["misfit"] == ref["misfit"]
    assert not np.any(got["datares"][0])

"""Parity at the benchmark configurations' full sizes, against the reference itself.

tests/golden/fullsize.json holds SHA-256 digests of the reference's own outputs
(oracle/_ref/librsref.so: ModellingAcoustic2D/ModellingElastic2D::run,
FwiAcoustic2D::run_optimal, in float) on the full-size inputs of
rockseis_b200.workloads, made by tests/golden/make_golden_fullsize.py:

  C1  acoustic 2D, 501 x 301, nt 2000, the whole gather;
  C2  elastic 2D, 801 x 401, nt 4000, shot 0 of 16 (400 Vx traces);
  C3  acoustic 2D FWI gradient, 601 x 201, nt 3000, shot 0 of 64: its observed
      data (modelled in the true model), then the vp / rho / wavelet gradients,
      modelled data, residuals and misfit of run_optimal with 50 snapshots.

EXACT arithmetic must reproduce each digest, i.e. equal the reference bit for
bit at full size.  FAST arithmetic (FMA) is held to relative L2 <= 1e-5 against
that result, FAST with FP16 checkpoints to <= 1e-3 on the gradients, and the FMA
result's error against the FP64 GPU propagator must not exceed twice the
reference float's own.
"""
import json
import os

import numpy as np
import pytest

from rockseis_b200 import abi, synth, workloads as W
from rockseis_b200.rockseis import (Data2D, FwiAcoustic2D, Image2D, ModelAcoustic2D, ModelElastic2D,
                                    ModellingAcoustic2D, ModellingElastic2D)
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "fullsize.json")))
FAST_TOL = 1e-5
CKPT16_TOL = 1e-3


def same_as_reference(name, a):
    a = np.ascontiguousarray(a)
    g = GOLD[name]
    assert list(a.shape) == g["shape"] and str(a.dtype) == g["dtype"], name
    return W.digest(a) == g["sha256"]


def _data(n, nt, dt, prec, coords, field, model, which, wav=None):
    d = Data2D(n, nt, dt, 0.0, prec)
    if which == 0:
        d.scoords[:] = coords
        d.data[:] = wav
    else:
        d.gcoords[:] = coords
    d.setField(field)
    d.makeMap(model, which)
    return d


def c1_gather(prec):
    c = W.C1
    vp, rho, src, wav, rec = W.acoustic2d_c1()
    m = ModelAcoustic2D(c["nx"], c["nz"], c["lpml"], c["dx"], c["dx"], 0.0, 0.0, 0, prec)
    m.createModel()
    m.Vp[:], m.R[:] = vp, rho
    s = _data(1, c["nt"], c["dt"], prec, src, abi.PRESSURE, m, 0, wav)
    r = _data(len(rec), c["nt"], c["dt"], prec, rec, abi.PRESSURE, m, 1)
    mod = ModellingAcoustic2D(m, s, c["order"], 1, precision=prec)
    mod.setRecP(r)
    assert mod.run() == 1
    return r.data.copy()


def c2_gather(prec, shot=0):
    c = W.C2
    vp, vs, rho, sx, wav, rec = W.elastic2d_c2()
    m = ModelElastic2D(c["nx"], c["nz"], c["lpml"], c["dx"], c["dx"], 0.0, 0.0, 0, prec)
    m.createModel()
    m.Vp[:], m.Vs[:], m.R[:] = vp, vs, rho
    s = _data(1, c["nt"], c["dt"], prec, [[sx[shot], c["sz"]]], abi.PRESSURE, m, 0, wav[None, :])
    r = _data(len(rec), c["nt"], c["dt"], prec, rec, abi.VX, m, 1)
    mod = ModellingElastic2D(m, s, c["order"], 1, precision=prec)
    mod.setRecVx(r)
    assert mod.run() == 1
    return r.data.copy()


def c3_model(prec, true_model):
    c = W.C3
    vt, vs, sx, wav, rec = W.fwi_c3()
    v = vt if true_model else vs
    m = ModelAcoustic2D(c["nx"], c["nz"], c["lpml"], c["dx"], c["dx"], 0.0, 0.0, 0, prec)
    m.createModel()
    m.Vp[:] = v
    m.R[:] = synth.gardner(v)
    s = _data(1, c["nt"], c["dt"], prec, [[sx[0], c["sz"]]], abi.PRESSURE, m, 0, wav[None, :])
    return m, s, rec


def c3_observed(prec):
    c = W.C3
    m, s, rec = c3_model(prec, True)
    r = _data(len(rec), c["nt"], c["dt"], prec, rec, abi.PRESSURE, m, 1)
    mod = ModellingAcoustic2D(m, s, c["order"], 1, precision=prec)
    mod.setRecP(r)
    assert mod.run() == 1
    return r.data.copy()


def c3_gradient(prec, obs, ckpt=abi.CKPT_NATIVE, accum=abi.ACCUM_REFERENCE):
    c = W.C3
    m, s, rec = c3_model(prec, False)
    o = _data(len(rec), c["nt"], c["dt"], prec, rec, abi.PRESSURE, m, 1)
    o.data[:] = obs
    f = FwiAcoustic2D(m, s, o, c["order"], 1, precision=prec)
    f.setNcheck(c["ncheck"])
    f.setCheckpointPrecision(ckpt)
    f.setAccumulation(accum)
    f.setVpgrad(Image2D("vpgrad", m, 1, 1, prec))
    f.setRhograd(Image2D("rhograd", m, 1, 1, prec))
    f.setWavgrad(Data2D(1, c["nt"], c["dt"], 0.0, prec))
    f.setDatamodP(Data2D(len(rec), c["nt"], c["dt"], 0.0, prec))
    f.setDataresP(Data2D(len(rec), c["nt"], c["dt"], 0.0, prec))
    assert f.run_optimal() == 1
    return dict(vpgrad=f.vpgrad.getImagedata()[0, 0].copy(), rhograd=f.rhograd.getImagedata()[0, 0].copy(),
                wavgrad=f.wavgrad.data.copy(), datamod=f.datamodP.data.copy(), datares=f.dataresP.data.copy(),
                misfit=np.array([f.getMisfit()]))


@pytest.fixture(scope="module")
def c2_exact(require_gpu):
    return c2_gather(abi.F32_EXACT)


def test_c1_exact_equals_reference_and_fast_within_fp32(require_gpu):
    ex = c1_gather(abi.F32_EXACT)
    assert np.abs(ex).max() > 0
    assert same_as_reference("c1_traces", ex)
    fa = c1_gather(abi.F32_FAST)
    assert rel_l2(fa, ex) <= FAST_TOL


def test_c2_shot0_exact_equals_reference(c2_exact):
    assert np.abs(c2_exact).max() > 0
    assert same_as_reference("c2_traces", c2_exact)


def test_c2_shot0_fast_within_fp32_and_fp64(c2_exact):
    fa = c2_gather(abi.F32_FAST)
    assert rel_l2(fa, c2_exact) <= FAST_TOL
    f64 = c2_gather(abi.F64)
    e_ref, e_fast = rel_l2(c2_exact, f64), rel_l2(fa, f64)
    print(f"C2 shot 0 rel-L2 vs FP64 GPU: reference float {e_ref:.3g}, FMA {e_fast:.3g}")
    assert e_fast <= 2 * max(e_ref, 1e-7)


@pytest.fixture(scope="module")
def c3_obs(require_gpu):
    return c3_observed(abi.F32_EXACT)


def test_c3_observed_data_equals_reference(c3_obs):
    assert same_as_reference("c3_obs", c3_obs)


def test_c3_shot0_gradient_exact_equals_reference(c3_obs):
    g = c3_gradient(abi.F32_EXACT, c3_obs)
    for k in ("vpgrad", "rhograd", "wavgrad", "datamod", "datares", "misfit"):
        assert np.abs(g[k]).max() > 0, k
        assert same_as_reference(f"c3_{k}", g[k]), k


def test_c3_shot0_gradient_fast_and_fp16_checkpoints(c3_obs):
    ex = c3_gradient(abi.F32_EXACT, c3_obs)
    g64 = c3_gradient(abi.F64, c3_obs.astype(np.float64), accum=abi.ACCUM_F64)
    fa = c3_gradient(abi.F32_FAST, c3_obs, accum=abi.ACCUM_F64)
    f16 = c3_gradient(abi.F32_FAST, c3_obs, ckpt=abi.CKPT_F16, accum=abi.ACCUM_F64)
    for k in ("vpgrad", "rhograd"):
        e_ref, e_fast, e16 = rel_l2(ex[k], g64[k]), rel_l2(fa[k], g64[k]), rel_l2(f16[k], g64[k])
        print(f"C3 shot 0 {k} rel-L2 vs FP64 GPU: reference float {e_ref:.3g}, FMA {e_fast:.3g}, "
              f"FMA + FP16 checkpoints {e16:.3g}")
        assert e_fast <= 2 * max(e_ref, 1e-7), k
        assert rel_l2(f16[k], ex[k]) <= CKPT16_TOL, k

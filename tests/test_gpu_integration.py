"""The reference classes driven through the GPU binding (integration/rockseis_gpu.cpp).

oracle/_ref/librsref_gpu.so is the reference library built by integration/Makefile
with ModellingAcoustic2D<float>::run, ModellingElastic2D<float>::run and
FwiAcoustic2D<float>::run_optimal specialised to call librsgpu.  The harness
builds the reference objects (Model, Data2D, Geometry2D, Fwi*) exactly as for the
stock library and calls the same public methods; every output must equal the
stock reference's CPU result bit for bit.  The stock library runs in a separate
process so the two builds' identical C++ symbols never meet in one address space.
"""
import os
import pickle
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from oracle import api
from rockseis_b200 import abi, synth
from tests.cases import Case2D, fwi_case

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def need_builds():
    if not (api.ref_available() and api.ref_gpu_available()):
        pytest.skip("reference builds oracle/_ref/librsref.so and librsref_gpu.so not present")


def stock(fn: str, *args, **kw):
    """api.<fn>(*args, **kw) on the stock reference library, in a fresh process."""
    with tempfile.TemporaryDirectory() as d:
        inp, out = os.path.join(d, "in.pkl"), os.path.join(d, "out.pkl")
        with open(inp, "wb") as f:
            pickle.dump((fn, args, kw), f)
        code = ("import pickle, sys; sys.path.insert(0, %r); from oracle import api; "
                "fn, a, k = pickle.load(open(%r, 'rb')); pickle.dump(getattr(api, fn)(*a, **k), open(%r, 'wb'))"
                % (ROOT, inp, out))
        subprocess.run([sys.executable, "-c", code], check=True, timeout=600)
        with open(out, "rb") as f:
            return pickle.load(f)


@pytest.mark.parametrize("sfield,rfield", [(abi.PRESSURE, abi.PRESSURE), (abi.PRESSURE, abi.VX), (abi.VZ, abi.VZ)])
def test_modelling_acoustic2d_through_binding(require_gpu, sfield, rfield):
    c = Case2D(abi.ACOUSTIC2D, nt=300, sfield=sfield, rfield=rfield)
    args = (c.pb, c.src.scoords, c.src.data.astype(np.float32), sfield, c.rec.gcoords, rfield)
    want = stock("ref_modelling_a2d", *args)
    got = api.ref_modelling_a2d(*args, lib=api.ref_gpu())
    assert np.abs(want).max() > 0
    assert np.array_equal(got, want), f"max abs diff {np.abs(got - want).max()}"


@pytest.mark.parametrize("sfield,rfield", [(abi.PRESSURE, abi.VX), (abi.VX, abi.PRESSURE)])
def test_modelling_elastic2d_through_binding(require_gpu, sfield, rfield):
    c = Case2D(abi.ELASTIC2D, nt=250, sfield=sfield, rfield=rfield)
    args = (c.pb, c.src.scoords, c.src.data.astype(np.float32), sfield, c.rec.gcoords, rfield)
    want = stock("ref_modelling_e2d", *args)
    got = api.ref_modelling_e2d(*args, lib=api.ref_gpu())
    assert np.abs(want).max() > 0
    assert np.array_equal(got, want), f"max abs diff {np.abs(got - want).max()}"


@pytest.mark.parametrize("ncheck,ilum", [(5, False), (300, True)])
def test_fwi_acoustic2d_through_binding(require_gpu, ncheck, ilum):
    c = fwi_case()
    args = (c.pb, c.src.scoords, c.src.data.astype(np.float32), c.rec.gcoords, c.obs.astype(np.float32), ncheck)
    want = stock("ref_fwi_a2d", *args, srcilum=ilum)
    got = api.ref_fwi_a2d(*args, srcilum=ilum, lib=api.ref_gpu())
    keys = ("vpgrad", "rhograd", "wavgrad", "datamod", "datares") + (("srcilum",) if ilum else ())
    for k in keys:
        assert np.abs(want[k]).max() > 0, k
        assert np.array_equal(got[k], want[k]), f"{k}: max abs diff {np.abs(got[k] - want[k]).max()}"
    assert got["misfit"] == want["misfit"]

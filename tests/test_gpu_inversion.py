"""InversionAcoustic2D.runGrad on the GPU: gathers from a recorded-data file, local
model windows, batched gradients stacked into the global images on the device.  The
stacked gradient must equal, bit for bit, the reference's procedure written out on
the host: every gather's gradient computed on its own, then added into the global
images window by window in gather order in the element type (Image2D::stackImage,
lib/image.cpp:348-438); also after an injected failure and retry."""
import numpy as np
import pytest

from rockseis_b200 import abi, synth
from rockseis_b200.inversion import InversionAcoustic2D
from rockseis_b200.rockseis import Data2D, ModelAcoustic2D, fwi_gradient_batch

pytestmark = pytest.mark.gpu

NX, NZ, DX, NT, DT = 121, 61, 10.0, 240, 1e-3


def setup(tmp_path):
    vp = synth.layered_vp(NX, NZ, DX, 1800, 3000, 3, 0.05, 60, 11).astype(np.float32)
    g = ModelAcoustic2D(NX, NZ, 10, DX, DX, 0.0, 0.0, 0)
    g.createModel()
    g.Vp[:], g.R[:] = vp, synth.gardner(vp)
    w = Data2D(1, NT, DT, 0.0)
    w.data[0] = synth.ricker(NT, DT, 20.0, np.float32)
    rng = np.random.default_rng(4)
    rows = [(s, gx) for s in (150.3, 930.7, 420.1, 700.5) for gx in np.arange(60.0, 1150.0, 90.0)]
    d = Data2D(len(rows), NT, DT, 0.0)
    d.scoords[:] = [[s, 15.0] for s, _ in rows]
    d.gcoords[:] = [[gx, 5.0] for _, gx in rows]
    d.data[:] = (rng.standard_normal(d.data.shape) * 1e-3).astype(np.float32)
    path = tmp_path / "precord.rss"
    d.setFile(str(path))
    d.write()
    inv = InversionAcoustic2D(g, w, str(path), order=8, apertx=300.0, ncheck=20)
    return inv


def host_stack(inv):
    """Each gather alone, then stacked on the host in gather order (float32 adds)."""
    from rockseis_b200.rockseis import Sort
    s = Sort()
    s.createShotmap(inv.precord)
    vp = np.zeros((NZ, NX), np.float32)
    rho = np.zeros_like(vp)
    mis = {}
    for k in range(s.getNensemb()):
        j = inv.job(s.get2DGather(k))
        fwi_gradient_batch([j])
        ix, iz = inv.window_origin(j.model)
        gv, gr = j.vpgrad.getImagedata()[0, 0], j.rhograd.getImagedata()[0, 0]
        nz, nx = gv.shape
        vp[iz:iz + nz, ix:ix + nx] = vp[iz:iz + nz, ix:ix + nx] + gv
        rho[iz:iz + nz, ix:ix + nx] = rho[iz:iz + nz, ix:ix + nx] + gr
        mis[k] = float(j.misfit)
    return vp, rho, mis


def test_rungrad_stack_equals_gatherwise_stack(require_gpu, tmp_path):
    inv = setup(tmp_path)
    inv.setPmodelledfile(tmp_path / "pmod.rss")
    r = inv.runGrad(batch=3)
    vp, rho, mis = host_stack(inv)
    assert np.abs(vp).max() > 0 and len(mis) == 4 and r["batches"] == 2
    assert np.array_equal(r["vpgrad"], vp), np.abs(r["vpgrad"] - vp).max()
    assert np.array_equal(r["rhograd"], rho)
    assert r["misfits"] == mis
    # the modelled gathers went to their traces' places in the output file
    out = Data2D.fromFile(str(tmp_path / "pmod.rss"))
    assert out.ntrace == 4 * 13 and np.abs(out.data).max() > 0


def test_rungrad_after_an_injected_failure(require_gpu, tmp_path):
    inv = setup(tmp_path)
    calls = {"n": 0}

    def flaky(jobs, vpgrad, rhograd):
        calls["n"] += 1
        if calls["n"] == 1:
            raise abi.RsgpuError(abi.ERR_CUDA, "injected failure of the first batch")
        inv.run_batch(jobs, vpgrad, rhograd)
    r = inv.runGrad(batch=4, runner=flaky)
    vp, rho, _ = host_stack(inv)
    assert r["failed"] == [] and calls["n"] == 1 + 4          # then the four gathers one by one
    assert np.array_equal(r["vpgrad"], vp) and np.array_equal(r["rhograd"], rho)

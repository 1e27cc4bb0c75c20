"""The no-allocation modelling entry point against the regular one.

rsgpu_modelling_a2d_noalloc serves callers that may not allocate device memory
(their memory belongs to another allocator or a fixed budget, or they cannot
take the device-wide synchronisation of cudaMalloc/cudaFree): they pass device
buffers they own for the model, wavelet and traces, and the library works in a
static per-device scratch array.  This test owns its buffers through torch; the
entry point itself allocates nothing.  Two calls in a row must both reproduce
rsgpu_modelling bit for bit (exact arithmetic), which also shows that a call
clears what the previous call left in the shared scratch array.

The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from rockseis_b200 import abi
from rockseis_b200.rockseis import ModellingAcoustic2D, make_config
from tests.cases import Case2D

pytestmark = pytest.mark.gpu


def test_noalloc_matches_regular_entry_point_twice(require_gpu):
    import torch

    c = Case2D(abi.ACOUSTIC2D, nt=200, sfield=abi.PRESSURE, rfield=abi.PRESSURE)
    mod = ModellingAcoustic2D(c.model, c.src, c.order, 1)
    mod.setRecP(c.rec)
    assert mod.run() == 1
    expected = c.rec.data.copy()
    assert np.abs(expected).max() > 0

    dev = torch.device("cuda", 0)
    models = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in c.model.padded()]
    wav = torch.from_numpy(np.ascontiguousarray(c.src.data)).to(dev)
    smap, sshift = np.ascontiguousarray(c.src.smap), np.ascontiguousarray(c.src.sshift)
    gmap, gshift = np.ascontiguousarray(c.rec.gmap), np.ascontiguousarray(c.rec.gshift)
    cfg = make_config(c.model, c.order, c.nt, c.dt, abi.F32_EXACT)
    torch.cuda.synchronize()

    for call in range(2):
        out = torch.zeros((c.rec.ntrace, c.nt), dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        s = abi.Shot()
        s.nx, s.ny, s.nz = c.model.nx, 1, c.model.nz
        for k, m in enumerate(models):
            s.model[k] = m.data_ptr()
        s.nsrc, s.smap, s.sshift, s.wavelet, s.src_field = c.src.ntrace, smap.ctypes.data, sshift.ctypes.data, \
            wav.data_ptr(), abi.PRESSURE
        s.nrec, s.gmap, s.gshift, s.rec_field = c.rec.ntrace, gmap.ctypes.data, gshift.ctypes.data, abi.PRESSURE
        s.rec_out = out.data_ptr()
        abi.check(abi.lib.rsgpu_modelling_a2d_noalloc(C.byref(cfg), C.byref(s), None))
        got = out.cpu().numpy()
        assert np.array_equal(got, expected), f"call {call}: max diff {np.abs(got - expected).max()}"


def test_noalloc_rejects_grids_beyond_its_scratch(require_gpu):
    c = Case2D(abi.ACOUSTIC2D, nx=81, nz=61, nt=10)
    cfg = make_config(c.model, c.order, c.nt, c.dt, abi.F32_EXACT)
    s = abi.Shot()
    s.nx, s.ny, s.nz = 4000, 1, 3000          # ~12 M padded cells x 6 arrays > 32 MiB
    for k in range(3):
        s.model[k] = 1                          # never dereferenced: the size check comes first
    st = abi.lib.rsgpu_modelling_a2d_noalloc(C.byref(cfg), C.byref(s), None)
    assert st == abi.ERR_ARG
    assert b"scratch" in abi.lib.rsgpu_last_error()

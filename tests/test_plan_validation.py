"""Plan creation rejects malformed batches with RSGPU_ERR_ARG (or UNSUPPORTED)
before touching a device, so these run on the CPU: empty and negative sizes,
grids narrower than the stencil, missing arrays, unknown fields and physics,
and the gradient drivers' own option checks."""
import ctypes as C

import numpy as np

import pytest

from rockseis_b200 import abi
from rockseis_b200.rockseis import make_config, make_shot
from tests.cases import Case2D


def _batch(physics=abi.ACOUSTIC2D):
    c = Case2D(physics, nt=20)
    keep: list = []
    cfg = make_config(c.model, c.order, c.nt, c.dt, abi.F32_EXACT)
    shots = (abi.Shot * 2)(make_shot(c.model, c.src, c.rec, keep), make_shot(c.model, c.src, c.rec, keep))
    return cfg, shots, keep


def _create(cfg, shots, n=None):
    h = C.c_void_p()
    st = abi.lib.rsgpu_plan_create(C.byref(cfg), len(shots) if n is None else n, shots, C.byref(h))
    if h.value:                                  # a valid batch on a machine with a GPU
        abi.lib.rsgpu_plan_destroy(h)
    return st


@pytest.mark.parametrize("mutate,status", [
    (lambda cfg, s: None, None),                                           # valid: fails only for want of a GPU
    (lambda cfg, s: setattr(cfg, "nt", 0), abi.ERR_ARG),
    (lambda cfg, s: setattr(cfg, "dt", 0.0), abi.ERR_ARG),
    (lambda cfg, s: setattr(cfg, "lpml", 0), abi.ERR_ARG),
    (lambda cfg, s: setattr(cfg, "physics", 7), abi.ERR_ARG),
    (lambda cfg, s: setattr(cfg, "precision", 5), abi.ERR_ARG),
    (lambda cfg, s: setattr(cfg, "physics", abi.ELASTIC3D), abi.ERR_ARG),     # a 2D batch lacks the 3D arrays
    (lambda cfg, s: setattr(s[1], "nx", 0), abi.ERR_ARG),                  # empty window
    (lambda cfg, s: (setattr(cfg, "lpml", 1), setattr(s[0], "nx", 2), setattr(s[0], "nz", 2)), abi.ERR_ARG),
    (lambda cfg, s: s[0].model.__setitem__(1, None), abi.ERR_ARG),         # missing parameter array
    (lambda cfg, s: setattr(s[0], "nrec", -1), abi.ERR_ARG),
    (lambda cfg, s: setattr(s[1], "gmap", None), abi.ERR_ARG),
    (lambda cfg, s: setattr(s[0], "src_field", 2), abi.ERR_ARG),          # VY has no 2D meaning
    (lambda cfg, s: setattr(s[0], "rec_field", 9), abi.ERR_ARG),
])
def test_plan_create_rejects_malformed_batches(mutate, status):
    cfg, shots, keep = _batch()
    mutate(cfg, shots)
    st = _create(cfg, shots)
    if status is None:
        # every check passed: the plan exists on a GPU machine, otherwise there is no device
        assert st in (abi.OK, abi.ERR_NODEVICE)
    else:
        assert st == status, abi.lib.rsgpu_last_error()
        assert abi.lib.rsgpu_last_error()


def test_plan_create_rejects_empty_batch():
    cfg, shots, keep = _batch()
    assert _create(cfg, shots, n=0) == abi.ERR_ARG


def test_gradient_driver_option_checks():
    c = Case2D(abi.ACOUSTIC2D, nt=20)
    keep: list = []
    cfg = make_config(c.model, c.order, c.nt, c.dt, abi.F32_EXACT)
    a = abi.AdjointShot()
    a.shot = make_shot(c.model, c.src, c.rec, keep)
    for field, value, status in (("misfit", 7, abi.ERR_UNSUPPORTED), ("ckpt_precision", 9, abi.ERR_ARG),
                                 ("accum", 5, abi.ERR_ARG), ("snapmethod", 7, abi.ERR_ARG)):
        o = abi.AdjointOpts()
        o.ncheck, o.nhx, o.nhz, o.nhy = 5, 1, 1, 1
        setattr(o, field, value)
        st = abi.lib.rsgpu_fwi_gradient(C.byref(cfg), C.byref(o), 1, C.byref(a))
        assert st == status, (field, abi.lib.rsgpu_last_error())
    o = abi.AdjointOpts()
    o.ncheck, o.nhx, o.nhz, o.nhy = 5, 2, 1, 1                               # RTM lags must be odd
    assert abi.lib.rsgpu_rtm_image(C.byref(cfg), C.byref(o), 1, C.byref(a)) == abi.ERR_ARG


def test_source_illumination_only_for_acoustic_2d_fwi():
    """FwiAcoustic2D alone has setSrcilum: elastic and 3D gradients and RTM refuse it."""
    c = Case2D(abi.ACOUSTIC2D, nt=20)
    keep: list = []
    cfg = make_config(c.model, c.order, c.nt, c.dt, abi.F32_EXACT)
    a = abi.AdjointShot()
    a.shot = make_shot(c.model, c.src, c.rec, keep)
    ilum = np.zeros((c.model.nz, c.model.nx), np.float32)
    a.srcilum = ilum.ctypes.data
    a.data = a.vp = a.rho = a.vs = ilum.ctypes.data
    o = abi.AdjointOpts()
    o.ncheck, o.nhx, o.nhz = 4, 1, 1
    st = abi.lib.rsgpu_rtm_image(C.byref(cfg), C.byref(o), 1, C.byref(a))
    assert st == abi.ERR_ARG
    assert b"illumination" in abi.lib.rsgpu_last_error()

"""The C ABI library without a GPU: it loads, exports what include/rsgpu.h declares,
validates arguments, and refuses compute calls loudly when no device is present
(there is no CPU fallback)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from rockseis_b200 import abi
from rockseis_b200.rockseis import ModellingAcoustic2D
from tests.cases import Case2D

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(rsgpu_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_the_entry_points():
    names = declared_entry_points()
    for must in ("rsgpu_modelling", "rsgpu_plan_create", "rsgpu_plan_run", "rsgpu_pml_tables",
                 "rsgpu_stagger_model", "rsgpu_make_map", "rsgpu_revolve_trace", "rsgpu_modelling_a2d_noalloc"):
        assert must in names


@pytest.mark.parametrize("name", declared_entry_points())
def test_library_exports_declared_symbol(name):
    lib = C.CDLL(abi.LIB_PATH)
    assert hasattr(lib, name), f"{name} declared in include/ but not exported by librsgpu.so"


def test_abi_version_and_error_text():
    assert abi.lib.rsgpu_abi_version() >= 1
    st = abi.lib.rsgpu_plan_create(None, 1, None, None)
    assert st == abi.ERR_ARG
    assert b"null" in abi.lib.rsgpu_last_error()


def test_host_preprocessing_rejects_bad_arguments():
    out = np.zeros(12, np.float32)
    assert abi.lib.rsgpu_pml_tables(0, 1e-3, abi.F32_EXACT, out.ctypes.data) == abi.ERR_ARG
    assert abi.lib.rsgpu_pml_tables(1, 1e-3, 99, out.ctypes.data) == abi.ERR_ARG


@pytest.mark.skipif(abi.lib.rsgpu_device_count() > 0, reason="a CUDA device is present")
def test_compute_without_device_fails_loudly():
    c = Case2D(abi.ACOUSTIC2D, nt=20)
    mod = ModellingAcoustic2D(c.model, c.src, c.order, 1)
    mod.setRecP(c.rec)
    with pytest.raises(abi.RsgpuError) as e:
        mod.run()
    assert e.value.status == abi.ERR_NODEVICE
    assert not c.rec.data.any()


def test_failure_self_test_without_device_fails_loudly():
    assert abi.lib.rsgpu_selftest_bounded_wait() == abi.ERR_NODEVICE

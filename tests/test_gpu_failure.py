"""Failure detection on the GPU without a fault: a kernel waits on a barrier that
nothing completes; its bounded wait gives up after 2 s, the host reads
RSGPU_ERR_TIMEOUT, and the same process then models a shot bit-exactly."""
import time

import numpy as np
import pytest

from rockseis_b200 import abi
from rockseis_b200.rockseis import ModellingAcoustic2D
from tests.cases import Case2D

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_device_stays_usable(require_gpu):
    t0 = time.perf_counter()
    st = abi.lib.rsgpu_selftest_bounded_wait()
    dt = time.perf_counter() - t0
    assert st == abi.ERR_TIMEOUT, abi.lib.rsgpu_last_error()
    assert b"time limit" in abi.lib.rsgpu_last_error()
    assert 1.5 < dt < 30.0
    c = Case2D(abi.ACOUSTIC2D, nt=120)
    c.rec.data[:] = 0
    mod = ModellingAcoustic2D(c.model, c.src, c.order, 1)
    mod.setRecP(c.rec)
    assert mod.run() == 1
    assert np.array_equal(c.rec.data, c.oracle_traces())

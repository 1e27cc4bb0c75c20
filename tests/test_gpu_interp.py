"""GPU trace resampling (rsgpu_interp_traces, the reference's Interp<T>::interp)
against the reference's own outputs: LINEAR and BSPLINE bit for bit, SINC to the
last bit of float (sin is evaluated by CUDA instead of the host libm)."""
import numpy as np
import pytest

from rockseis_b200 import abi
from rockseis_b200.rockseis import Data2D, Interp
from tests.test_oracle_pin import GOLD, INTERP_AXES

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [abi.INTERP_LINEAR, abi.INTERP_BSPLINE, abi.INTERP_SINC])
def test_interp_matches_reference(require_gpu, mode):
    n1, o1, d1 = GOLD["interp_axis_in"]
    data = GOLD["interp_in"]
    frm = Data2D(data.shape[0], int(n1), d1, o1)
    frm.data[:] = data
    frm.gcoords[:] = np.arange(2 * data.shape[0]).reshape(-1, 2)
    for a, (n2, o2, d2) in enumerate(INTERP_AXES):
        to = Data2D(data.shape[0], n2, d2, o2)
        Interp(mode).interp(frm, to)
        ref = GOLD[f"interp_m{mode}_a{a}"]
        assert np.array_equal(to.gcoords, frm.gcoords)
        if mode == abi.INTERP_SINC:
            ulp = np.spacing(np.abs(ref).astype(np.float32))
            assert np.all(np.abs(to.data - ref) <= 2 * ulp + 1e-30), (a, np.abs(to.data - ref).max())
        else:
            assert np.array_equal(to.data, ref), (mode, a, np.abs(to.data - ref).max())


def test_interp_fp64_and_empty(require_gpu):
    frm = Data2D(3, 50, 1e-3, 0.0, abi.F64)
    frm.data[:] = np.sin(np.arange(150).reshape(3, 50) * 0.1)
    to = Data2D(3, 90, 5e-4, 0.0, abi.F64)
    Interp(abi.INTERP_LINEAR).interp(frm, to)
    # linear interpolation of the midpoints
    assert np.allclose(to.data[:, 1:89:2], 0.5 * (frm.data[:, :44] + frm.data[:, 1:45]), atol=1e-12)
    empty = Data2D(0, 10, 1e-3, 0.0)
    Interp(abi.INTERP_SINC).interp(Data2D(0, 10, 1e-3, 0.0), empty)

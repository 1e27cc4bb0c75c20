"""Golden outputs of the reference's acoustic FWI gradient with the ADAPTIVE_GAUSS and
ADAPTIVE_LINEAR misfits (FwiAcoustic2D::computeMisfit / computeResiduals,
lib/fwi.cpp:646-751, 851-1026; FwiAcoustic3D, lib/fwi.cpp:1541-1631, 1725-1842),
through oracle/_ref/librsref.so.

Run from the repository root after the reference library is built:
    python tests/golden/make_golden_adaptive.py
Writes tests/golden/adaptive.npz: for the acoustic 2D FWI case of tests/cases.py
(fwi_case(): 81 x 61 cells, nt = 300, 30 receivers) run_optimal with 7 Revolve
snapshots, and for the small acoustic 3D FWI case (fwi3d_case()) with 5, every
output (gradients, wavelet gradient, modelled data, residuals, misfit) of both
misfits, and for the elastic 2D case (ElasticFwiCase(), P/Ux/Uz data, 7 snapshots)
the same with ADAPTIVE_SINGLE added (FwiElastic2D, lib/fwi.cpp:3002-3196,
3428-3753); the observed data of each case are kept so that a test can check that
it rebuilds the same problem.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import api  # noqa: E402
from tests.cases import ElasticFwiCase, fwi_case  # noqa: E402
from tests.test_gpu_modelling_3d import fwi3d_case  # noqa: E402

MISFITS = {"gauss": 2, "linear": 3}


def keep(out, case, name, r):
    """Outputs of one run; the modelled data, the same for every misfit, are kept once."""
    for k, v in r.items():
        if k == "datamod":
            if f"{case}_datamod" in out:
                assert np.array_equal(out[f"{case}_datamod"], v)
            out[f"{case}_datamod"] = np.asarray(v)
        else:
            out[f"{case}_{name}_{k}"] = np.asarray(v)


def main():
    if not api.ref_available():
        raise SystemExit("oracle/_ref/librsref.so is not built")
    out = {}
    c = fwi_case()
    out["a2d_obs"] = c.obs.astype(np.float32)
    for name, m in MISFITS.items():
        r = api.ref_fwi_a2d(c.pb, c.src.scoords, c.src.data.astype(np.float32), c.rec.gcoords,
                            c.obs.astype(np.float32), 7, misfit=m)
        keep(out, "a2d", name, r)
    c3 = fwi3d_case()
    out["a3d_obs"] = c3.obs.astype(np.float32)
    for name, m in MISFITS.items():
        r = api.ref_fwi_a3d(c3.pb, c3.src.scoords, c3.src.data.astype(np.float32), c3.rec.gcoords,
                            c3.obs.astype(np.float32), 5, misfit=m)
        keep(out, "a3d", name, r)
    ce = ElasticFwiCase()
    obs3 = [o.astype(np.float32) for o in ce.obs]
    out["e2d_obs"] = np.stack(obs3)
    for name, m in dict(MISFITS, single=4).items():
        r = api.ref_fwi_e2d(ce.pb, ce.src.scoords, ce.src.data.astype(np.float32), ce.sfield, ce.recs[0].gcoords, obs3,
                            7, misfit=m)
        keep(out, "e2d", name, r)
    path = os.path.join(ROOT, "tests", "golden", "adaptive.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()

"""Golden outputs of the reference's FULL-snapshot elastic 2D gradient,
FwiElastic2D::run (lib/fwi.cpp:3774-3934), through oracle/_ref/librsref.so.

Run from the repository root after the reference library is built:
    python tests/golden/make_golden_e2d_full.py
Writes tests/golden/e2d_full.npz for the elastic FWI case of tests/cases.py
(ElasticFwiCase(): P, Ux and Uz observed data):
  * the case's observed data (so that a test can check that it rebuilds the same
    problem);
  * the modelled data, residuals and misfit (the same for every snapinc: the
    script asserts it);
  * the vp, vs and rho gradients and the wavelet gradient for snapinc 1, 3 and 5.
The driver saves Vx and Vz before each forward step whose index is a multiple of
snapinc and, in the adjoint loop, correlates every step with the snapshot read
last (Snapshot2D::readSnap, lib/snap.cpp) through the pointer form of crossCorr
(lib/fwi.cpp:2411-2590).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import api  # noqa: E402
from tests.cases import ElasticFwiCase  # noqa: E402

SNAPINC = (1, 3, 5)


def main():
    if not api.ref_available():
        raise SystemExit("oracle/_ref/librsref.so is not built")
    c = ElasticFwiCase()
    wav = c.src.data.astype(np.float32)
    obs3 = [o.astype(np.float32) for o in c.obs]
    out = dict(obs=np.stack(obs3))
    runs = {si: api.ref_fwi_e2d(c.pb, c.src.scoords, wav, c.sfield, c.recs[0].gcoords, obs3, 0, full_snapinc=si)
            for si in SNAPINC}
    for k in ("datamod", "datares", "misfit"):
        for si in SNAPINC[1:]:
            assert np.array_equal(runs[si][k], runs[SNAPINC[0]][k]), k
        out[k] = np.asarray(runs[SNAPINC[0]][k])
    for si in SNAPINC:
        for k in ("vpgrad", "vsgrad", "rhograd", "wavgrad"):
            assert np.all(np.isfinite(runs[si][k])), (si, k)
            out[f"s{si}_{k}"] = runs[si][k]
    assert np.abs(out["s1_vpgrad"]).max() > 0
    path = os.path.join(ROOT, "tests", "golden", "e2d_full.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()

"""Golden outputs of the reference's FULL-snapshot drivers, FwiAcoustic2D::run
(lib/fwi.cpp:1030-1156) and RtmAcoustic2D::run (lib/rtm.cpp:222-326), through
oracle/_ref/librsref.so.

Run from the repository root after the reference library is built:
    python tests/golden/make_golden_snapfull.py
Writes tests/golden/snapfull.npz for the acoustic FWI case of tests/cases.py
(fwi_case(): 81 x 61 cells, nt = 300, one source, 30 receivers):
  * the case's inputs (vp, rho, wavelet, observed data, coordinates), so that a
    test can check that it rebuilds the same problem;
  * the modelled data, residuals and misfit (the same for every snapinc, and
    with noreverse, which leaves the gradients, the wavelet gradient and the
    residuals at zero: the script asserts both);
  * the gradients for snapinc 3 and 7 (enddiff 2 and 5: the correlated times
    are shifted against the saved ones);
  * the RTM image for snapinc 4 with three x lags, from full snapshots
    (RtmAcoustic2D::run) and from edge lines (RtmAcoustic2D::run_edge,
    lib/rtm.cpp:328-421);
  * the 3D RTM image (RtmAcoustic3D::run, lib/rtm.cpp:640-733) of the small 3D
    case of tests/test_gpu_modelling_3d.py (29 x 27 x 25, nt = 120) for snapinc 4,
    with the data it migrates.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import api  # noqa: E402
from tests.cases import fwi_case  # noqa: E402

FWI_SNAPINC = (3, 7)
RTM_SNAPINC, RTM_NHX = 4, 3


def main():
    if not api.ref_available():
        raise SystemExit("oracle/_ref/librsref.so is not built")
    c = fwi_case()
    wav = c.src.data.astype(np.float32)
    obs = c.obs.astype(np.float32)
    out = dict(vp=c.pb.vp, rho=c.pb.rho, wav=wav, obs=obs, scoords=c.src.scoords, gcoords=c.rec.gcoords)
    runs = {si: api.ref_fwi_a2d_full(c.pb, c.src.scoords, wav, c.rec.gcoords, obs, si) for si in FWI_SNAPINC}
    runs["noreverse"] = api.ref_fwi_a2d_full(c.pb, c.src.scoords, wav, c.rec.gcoords, obs, 3, noreverse=1)
    # the forward pass, hence datamod, datares and the misfit, do not depend on snapinc
    for k in ("datamod", "datares", "misfit"):
        for si in FWI_SNAPINC[1:]:
            assert np.array_equal(runs[si][k], runs[FWI_SNAPINC[0]][k]), k
    for k in ("datamod", "misfit"):
        assert np.array_equal(runs["noreverse"][k], runs[FWI_SNAPINC[0]][k]), k
    for k in ("datamod", "datares", "misfit"):
        out[f"fwi_{k}"] = np.asarray(runs[FWI_SNAPINC[0]][k])
    for si in FWI_SNAPINC:
        for k in ("vpgrad", "rhograd", "wavgrad"):
            out[f"fwi_s{si}_{k}"] = runs[si][k]
    for k in ("vpgrad", "rhograd", "wavgrad", "datares"):
        assert not np.any(runs["noreverse"][k]), k
    out[f"rtm_s{RTM_SNAPINC}_h{RTM_NHX}"] = api.ref_rtm_a2d_full(c.pb, c.src.scoords, wav, c.rec.gcoords, obs,
                                                                 RTM_SNAPINC, nhx=RTM_NHX)
    out[f"rtm_edge_s{RTM_SNAPINC}_h{RTM_NHX}"] = api.ref_rtm_a2d_full(c.pb, c.src.scoords, wav, c.rec.gcoords, obs,
                                                                      RTM_SNAPINC, nhx=RTM_NHX, edges=True)
    from tests.test_gpu_modelling_3d import Case3D, rtm_inputs
    c3 = Case3D(nx=29, ny=27, nz=25)
    data3 = rtm_inputs(c3)
    out["rtm3d_data"] = data3
    out["rtm3d_s4"] = api.ref_rtm_a3d(c3.pb, c3.src.scoords, c3.src.data.astype(np.float32), c3.rec.gcoords, data3,
                                      0, full_snapinc=4)
    path = os.path.join(ROOT, "tests", "golden", "snapfull.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()

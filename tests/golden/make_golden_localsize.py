"""Golden aperture windows from the reference's Model::getLocalsize2d/3d
(lib/model.cpp:272-470), through oracle/_ref/librsref.so.

Run from the repository root after the reference library is built:
    python tests/golden/make_golden_localsize.py
Writes tests/golden/localsize.json: seeded cases covering positive, zero and
negative apertures, SMAP and GMAP, several origins and spacings, single and
multi-trace gathers, and windows that run over the model edges (the windows are
not clipped: the getLocal copy clamps them).
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import api  # noqa: E402


def cases(seed=17, n=60):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        dim = 2 if k % 2 == 0 else 3
        ntr = int(rng.integers(1, 9))
        dx, dy = float(rng.choice([5.0, 10.0, 12.5, 7.3])), float(rng.choice([5.0, 10.0, 12.5]))
        ox, oy = float(rng.choice([0.0, -120.0, 37.5])), float(rng.choice([0.0, 55.0]))
        ext = 4000.0
        sxyz = rng.uniform(-100.0, ext, (ntr, 3))
        if k % 3 == 0:
            sxyz[:] = sxyz[0]          # one source for the whole gather
        gxyz = rng.uniform(-100.0, ext, (ntr, 3))
        ap = float(rng.choice([0.0, 850.0, 1999.0, -300.0, 2500.5]))
        apy = float(rng.choice([0.0, 400.0, -150.0]))
        smap = int(k % 4 < 2)
        out.append(dict(dim=dim, dx=dx, dy=dy, ox=ox, oy=oy, s=sxyz.tolist(), g=gxyz.tolist(), ap=ap, apy=apy,
                        map=0 if smap else 1))
    return out


def main():
    res = []
    for c in cases():
        s, g = np.array(c["s"]), np.array(c["g"])
        if c["dim"] == 2:
            grid = api.RefGrid(400, 1, 100, 10, 8, 0, c["dx"], 1.0, c["dx"], c["ox"], 0.0, 0.0, 1e-3, 10)
            c["want"] = list(api.ref_localsize2d(grid, s[:, [0, 2]], g[:, [0, 2]], c["ap"], c["map"]))
        else:
            grid = api.RefGrid(400, 300, 100, 10, 8, 0, c["dx"], c["dy"], c["dx"], c["ox"], c["oy"], 0.0, 1e-3, 10)
            (sx, nx), (sy, ny) = api.ref_localsize3d(grid, s, g, c["ap"], c["apy"], c["map"])
            c["want"] = [sx, nx, sy, ny]
        res.append(c)
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "localsize.json"), "w") as f:
        json.dump(res, f)
    print(f"{len(res)} cases")


if __name__ == "__main__":
    main()

"""Digests of the reference's own outputs at the benchmark configurations' full sizes.

Run where the reference library is built (oracle/_ref/librsref.so, from the
unmodified reference sources by `make -C oracle ref`):

    python tests/golden/make_golden_fullsize.py

It runs, each in its own process and each through the reference's public
drivers in float:
  c1   ModellingAcoustic2D::run        501 x 301, nt 2000, P source, 251 P receivers
  c2   ModellingElastic2D::run         shot 0 of the 16: 801 x 401, nt 4000,
                                       explosive source, 400 Vx receivers
  c3   ModellingAcoustic2D::run in the true model (the observed data of shot 0),
       then FwiAcoustic2D::run_optimal in the starting model with 50 snapshots
                                       601 x 201, nt 3000, 601 receivers
and writes fullsize.json (SHA-256 of every output array's bytes, plus its
shape, norm and extreme) and fullsize.npz (a regular sample of every output,
see sample(), for diagnosing a mismatch).  The inputs come
from rockseis_b200.workloads, which the GPU tests use as well.  About ten
minutes of CPU on four cores.
"""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

PRESSURE, VX = 0, 1


def _summary(a):
    from rockseis_b200.workloads import digest
    a = np.ascontiguousarray(a)
    return {"sha256": digest(a), "shape": list(a.shape), "dtype": str(a.dtype),
            "l2": float(np.linalg.norm(a.astype(np.float64))), "absmax": float(np.abs(a).max())}


def job_c1():
    from oracle import api
    from rockseis_b200 import workloads as W
    c = W.C1
    vp, rho, src, wav, rec = W.acoustic2d_c1()
    pb = api.Problem2D(c["nx"], c["nz"], c["dx"], c["dx"], c["lpml"], c["order"], 0, c["dt"], c["nt"], vp, rho)
    t0 = time.perf_counter()
    d = api.ref_modelling_a2d(pb, src, wav, PRESSURE, rec, PRESSURE)
    return {"c1_traces": d}, time.perf_counter() - t0


def job_c2():
    from oracle import api
    from rockseis_b200 import workloads as W
    c = W.C2
    vp, vs, rho, sx, wav, rec = W.elastic2d_c2()
    pb = api.Problem2D(c["nx"], c["nz"], c["dx"], c["dx"], c["lpml"], c["order"], 0, c["dt"], c["nt"], vp, rho, vs)
    t0 = time.perf_counter()
    d = api.ref_modelling_e2d(pb, np.array([[sx[0], c["sz"]]]), wav[None, :], PRESSURE, rec, VX)
    return {"c2_traces": d}, time.perf_counter() - t0


def job_c3():
    from oracle import api
    from rockseis_b200 import synth, workloads as W
    c = W.C3
    vt, vs, sx, wav, rec = W.fwi_c3()
    src = np.array([[sx[0], c["sz"]]])
    t0 = time.perf_counter()
    pt = api.Problem2D(c["nx"], c["nz"], c["dx"], c["dx"], c["lpml"], c["order"], 0, c["dt"], c["nt"], vt,
                       synth.gardner(vt))
    obs = api.ref_modelling_a2d(pt, src, wav[None, :], PRESSURE, rec, PRESSURE)
    ps = api.Problem2D(c["nx"], c["nz"], c["dx"], c["dx"], c["lpml"], c["order"], 0, c["dt"], c["nt"], vs,
                       synth.gardner(vs))
    g = api.ref_fwi_a2d(ps, src, wav[None, :], rec, obs, c["ncheck"])
    out = {"c3_obs": obs, "c3_vpgrad": g["vpgrad"], "c3_rhograd": g["rhograd"], "c3_wavgrad": g["wavgrad"],
           "c3_datamod": g["datamod"], "c3_datares": g["datares"], "c3_misfit": np.array([g["misfit"]])}
    return out, time.perf_counter() - t0


def sample(name, a):
    """The slice of an output kept in fullsize.npz: every 16th trace at every 8th
    sample of a gather, every 4th point of a gradient in each direction."""
    if a.ndim == 2 and name.endswith(("traces", "obs", "datamod", "datares")):
        return np.ascontiguousarray(a[::16, ::8])
    if a.ndim == 2 and name.endswith("grad") and a.shape[0] > 1:
        return np.ascontiguousarray(a[::4, ::4])
    return a


def input_digests():
    """Digests of the workload inputs the outputs were computed from (the CPU test
    suite checks that rockseis_b200.workloads still produces them)."""
    from rockseis_b200 import workloads as W
    out = {}
    for name, arrays in (("c1", W.acoustic2d_c1()), ("c2", W.elastic2d_c2()), ("c3", W.fwi_c3())):
        for k, a in enumerate(arrays):
            out[f"{name}_input{k}"] = W.digest(np.asarray(a))
    return out


def _run(name):
    return name, *globals()[f"job_{name}"]()


def main():
    from oracle import api
    if not api.ref_available():
        raise SystemExit("oracle/_ref/librsref.so is not built (make -C oracle ref)")
    with mp.get_context("spawn").Pool(3) as pool:
        results = pool.map(_run, ["c2", "c3", "c1"])
    summary, keep = {}, {}
    for name, arrays, secs in results:
        summary[f"{name}_reference_seconds"] = round(secs, 1)
        for k, a in arrays.items():
            summary[k] = _summary(a)
            keep[k] = sample(k, a)
    summary["inputs"] = input_digests()
    with open(os.path.join(HERE, "fullsize.json"), "w") as f:
        json.dump(summary, f, indent=1, sort_keys=True)
    np.savez_compressed(os.path.join(HERE, "fullsize.npz"), **keep)
    print(json.dumps({k: v for k, v in summary.items() if k.endswith("seconds")}))


if __name__ == "__main__":
    main()

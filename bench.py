"""Benchmark of the finite-difference hot path (one JSON line on stdout).

Workload: 2D elastic forward modelling, 16 shots at uneven spacing batched in
one plan: 801 x 401 grid, dx = dz = 5 m, 30-cell C-PML (padded 861 x 461),
order 8 (16-tap staggered stencil), nt = 4000, dt = 0.5 ms, explosive source at
z = 10 m, 400 Vx receivers every 10 m at the surface.  Seeded synthetic model
(layered vp <= 4450 m/s, vp/vs 1.7-2.0, Gardner density, random lenses).

A "step" is one complete forward modelling of the batch (all nt time steps of
all shots).  Metric: Gpts/s = padded grid points x time steps / second, summed
over shots (and over ranks with --gpus N: every rank models its own 16 shots,
weak scaling, no data-path collective).

  value   device-resident plan (models uploaded once), CUDA-event timed.
  e2e     rsgpu_modelling through the C ABI from pinned host buffers: upload of
          models, maps and wavelets, the run, and the read-back of the traces.
  roofline  dominant half-step kernel: algorithmic bytes per launch / its
          CUDA-event duration inside the timed region (events recorded in the
          captured graph), against the measured HBM copy bandwidth.
  cpu_baseline  the reference's own ModellingElastic2D::run (oracle/_ref,
          compiled from the reference sources) on all host cores, one shot per
          process, first 100 time steps of the same shot (bounded sample).

--impl reference times that CPU reference alone (same metric and config).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from rockseis_b200 import workloads as W  # noqa: E402

NX, NZ, DX, LPML, ORDER, DT, NT, NSHOTS, NREC = (W.C2[k] for k in ("nx", "nz", "dx", "lpml", "order", "dt", "nt",
                                                                    "nshots", "nrec"))
CPU_SAMPLE_STEPS = 100          # the reference arm: time steps of one bench step
CPU_BASELINE_STEPS = 400        # the cpu_baseline object of our own line (10 % of nt)


def workload_inputs():
    """The elastic 2D workload (rockseis_b200.workloads.elastic2d_c2)."""
    return W.elastic2d_c2()


def config_dict(ngpus, precision_name, nt=NT):
    return {"workload": f"elastic2d_forward_16shots_801x401_nt{nt}", "nx": NX, "nz": NZ, "dx": DX, "lpml": LPML,
            "order": ORDER, "nt": nt, "dt": DT, "shots_per_gpu": NSHOTS, "receivers": NREC,
            "padded_points_per_shot": (NX + 2 * LPML) * (NZ + 2 * LPML), "arithmetic": precision_name,
            "l2": "working set 254 MB per GPU > 126 MB L2 (no flush needed)", "parallelism": f"shots x{ngpus}"}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    def __init__(self, index=0):
        self.index, self.proc, self.lines = index, None, []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- CPU reference
def _ref_sample(args):
    """One process: the reference's ModellingElastic2D::run on one shot, bounded nt."""
    shot, nsteps = args
    sys.path.insert(0, ROOT)
    import ctypes as C
    from oracle import api
    vp, vs, rho, sx, wav, gc = workload_inputs()
    pb = api.Problem2D(NX, NZ, DX, DX, LPML, ORDER, 0, DT, nsteps, vp, rho, vs)
    t0 = time.perf_counter()
    api.ref_modelling_e2d(pb, np.array([[sx[shot], 10.0]]), wav[None, :nsteps], 0, gc, 1)
    dt = time.perf_counter() - t0
    return dt


def cpu_reference(nsteps=CPU_SAMPLE_STEPS, procs=None):
    """Aggregate Gpts/s of the reference CPU path on all host cores (P concurrent processes)."""
    import multiprocessing as mp
    from oracle import api
    if not api.ref_available():
        return None
    procs = procs or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        times = pool.map(_ref_sample, [(i % NSHOTS, nsteps) for i in range(procs)])
    wall = time.perf_counter() - t0
    pts = (NX + 2 * LPML) * (NZ + 2 * LPML) * nsteps * procs
    return {"value": pts / max(times) / 1e9, "unit": "Gpts/s", "cores": procs, "kind": "reference",
            "sample": f"{procs} processes x 1 shot x first {nsteps} of {NT} steps, full 861x461 padded grid",
            "max_process_s": round(max(times), 3), "wall_s": round(wall, 3)}


def c1_config(ngpus, precision_name):
    c = W.C1
    return {"workload": "acoustic2d_forward_1shot_501x301_nt2000", "nx": c["nx"], "nz": c["nz"], "dx": c["dx"],
            "lpml": c["lpml"], "order": c["order"], "nt": c["nt"], "dt": c["dt"], "shots_per_gpu": 1,
            "receivers": c["nrec"], "padded_points_per_shot": (c["nx"] + 2 * c["lpml"]) * (c["nz"] + 2 * c["lpml"]),
            "arithmetic": precision_name, "vp_clip": c["vclip"],
            "l2": "working set 6.6 MB: L2-resident; timed steps repeat the same shot without a flush",
            "parallelism": f"shots x{ngpus}"}


def _c1_ref_sample(nsteps):
    sys.path.insert(0, ROOT)
    from oracle import api
    c = W.C1
    vp, rho, src, wav, rec = W.acoustic2d_c1(nsteps)
    pb = api.Problem2D(c["nx"], c["nz"], c["dx"], c["dx"], c["lpml"], c["order"], 0, c["dt"], nsteps, vp, rho)
    t0 = time.perf_counter()
    api.ref_modelling_a2d(pb, src, wav, 0, rec, 0)
    return time.perf_counter() - t0


def cpu_c1_reference(nsteps=500):
    """The reference's ModellingAcoustic2D::run on the one shot (one process: the
    reference parallelises only over shots), first nsteps of 2000."""
    import multiprocessing as mp
    from oracle import api
    if not api.ref_available():
        return None
    with mp.get_context("spawn").Pool(1) as pool:
        t = pool.map(_c1_ref_sample, [nsteps])[0]
    c = W.C1
    pts = (c["nx"] + 2 * c["lpml"]) * (c["nz"] + 2 * c["lpml"]) * nsteps
    return {"value": round(pts / t / 1e9, 5), "unit": "Gpts/s", "cores": 1, "kind": "reference",
            "sample": f"1 process (one shot) x first {nsteps} of {c['nt']} steps, full 541x341 padded grid",
            "process_s": round(t, 3)}


# ---------------------------------------------------------------- GPU arm
def _pin(models, srcs, recs):
    """Move the batch's host arrays into pinned memory (the end-to-end measurement)."""
    import torch
    for m in models:
        pinned_pads = []
        for a in m.padded():
            t = torch.empty(a.shape, dtype=torch.float32).pin_memory()
            t.numpy()[:] = a
            pinned_pads.append(t)
        m._pinned = pinned_pads
        m._padded = dict(zip(m.names, [t.numpy() for t in pinned_pads]))
    for r in recs:
        t = torch.zeros(r.data.shape, dtype=torch.float32).pin_memory()
        r._pinned = t
        r.data = t.numpy()
    for s_ in srcs:
        t = torch.empty(s_.data.shape, dtype=torch.float32).pin_memory()
        t.numpy()[:] = s_.data
        s_._pinned = t
        s_.data = t.numpy()


def build_batch(precision, vp, vs, rho, sx, wav, gc, nt=NT, pinned=False, shots=None):
    """The elastic 2D batch: one model window per shot (the whole model), explosive
    source at z = 10 m, Vx receivers at the surface."""
    from rockseis_b200 import abi
    from rockseis_b200.rockseis import Data2D, ModelElastic2D
    models, srcs, recs = [], [], []
    for i in (range(NSHOTS) if shots is None else shots):
        m = ModelElastic2D(NX, NZ, LPML, DX, DX, 0.0, 0.0, 0, precision)
        m.createModel()
        m.Vp[:], m.Vs[:], m.R[:] = vp, vs, rho
        s = Data2D(1, nt, DT, 0.0, precision)
        s.scoords[:] = [[sx[i], W.C2["sz"]]]
        s.data[:] = wav[None, :nt]
        s.setField(abi.PRESSURE)
        s.makeMap(m, 0)
        r = Data2D(NREC, nt, DT, 0.0, precision)
        r.gcoords[:] = gc
        r.setField(abi.VX)
        r.makeMap(m, 1)
        models.append(m)
        srcs.append(s)
        recs.append(r)
    if pinned:
        _pin(models, srcs, recs)
    return models, srcs, recs


def build_c1(precision, nt=None, pinned=False):
    """The acoustic 2D shot of rockseis_b200.workloads.acoustic2d_c1."""
    from rockseis_b200 import abi
    from rockseis_b200.rockseis import Data2D, ModelAcoustic2D
    c = W.C1
    nt = nt or c["nt"]
    vp, rho, src, wav, rec = W.acoustic2d_c1(nt)
    m = ModelAcoustic2D(c["nx"], c["nz"], c["lpml"], c["dx"], c["dx"], 0.0, 0.0, 0, precision)
    m.createModel()
    m.Vp[:], m.R[:] = vp, rho
    s = Data2D(1, nt, c["dt"], 0.0, precision)
    s.scoords[:] = src
    s.data[:] = wav
    s.setField(abi.PRESSURE)
    s.makeMap(m, 0)
    r = Data2D(len(rec), nt, c["dt"], 0.0, precision)
    r.gcoords[:] = rec
    r.setField(abi.PRESSURE)
    r.makeMap(m, 1)
    models, srcs, recs = [m], [s], [r]
    if pinned:
        _pin(models, srcs, recs)
    return models, srcs, recs


def algorithmic_bytes(models, physics="elastic2d"):
    """Algorithmic bytes per launch over the batch (fp32) and the padded points.

    elastic, fused step: read Vx,Vz,Sxx,Szz,Sxz,Rx,Rz,L,L2M,M; write the 5 fields
      -> 60 B per padded point, plus 8 C-PML memory arrays (4 in the x strips, 4 in
      the z strips), each read and written once: 32 B per strip point;
    elastic, per-tile half-steps: velocity 36 B, stress 44 B, 16 B per strip point each;
    acoustic, fused: read P,Vx,Vz,Rx,Rz,L, write P,Vx,Vz -> 36 B + 16 B per strip point;
    acoustic, per-tile: velocity 28 B, stress 20 B, 8 B per strip point each.
    Returns (fused, velocity, stress, points)."""
    pts = strip = 0
    for m in models:
        nxp, nzp, L = m.getNx_pml(), m.getNz_pml(), m.lpml
        pts += nxp * nzp
        strip += 2 * L * nzp + 2 * L * nxp
    if physics == "elastic2d":
        return 60 * pts + 32 * strip, 36 * pts + 16 * strip, 44 * pts + 16 * strip, pts
    return 36 * pts + 16 * strip, 28 * pts + 8 * strip, 20 * pts + 8 * strip, pts


def read_traffic(kernel, workload="elastic2d_16shots"):
    """ncu DRAM bytes per launch recorded in profiles/ for the workload, if any."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.txt")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def _shot0_traces(precision, physics, nt):
    """Shot 0 of the workload alone, modelled in `precision` (parity figures)."""
    from rockseis_b200.rockseis import modelling_batch
    if physics == "elastic2d":
        vp, vs, rho, sx, wav, gc = workload_inputs()
        models, srcs, recs = build_batch(precision, vp, vs, rho, sx, wav, gc, nt=nt, shots=[0])
    else:
        models, srcs, recs = build_c1(precision, nt)
    modelling_batch(models, srcs, recs, ORDER, precision)
    return recs[0].data.copy()


def parity_figures(fast0, physics, nt):
    """Errors of the timed FMA result (shot 0), computed outside the timed region:
    against the EXACT GPU run, whose digest is compared with the reference's own
    output at full length (tests/golden/fullsize.json), and against the FP64 GPU
    propagator, beside the reference float's own error against FP64."""
    from rockseis_b200 import abi
    exact = _shot0_traces(abi.F32_EXACT, physics, nt)
    f64 = _shot0_traces(abi.F64, physics, nt)
    key = "c2_traces" if physics == "elastic2d" else "c1_traces"
    equal = None
    full_nt = NT if physics == "elastic2d" else W.C1["nt"]
    if nt == full_nt:
        gold = json.load(open(os.path.join(ROOT, "tests", "golden", "fullsize.json")))[key]
        equal = W.digest(exact) == gold["sha256"]
    return {"shot": 0, "exact_equals_reference": equal,
            "rel_l2_vs_reference": float("%.3g" % rel_l2(fast0, exact)),
            "rel_l2_vs_fp64_gpu": float("%.3g" % rel_l2(fast0, f64)),
            "reference_float_rel_l2_vs_fp64_gpu": float("%.3g" % rel_l2(exact, f64)),
            "how": "FMA traces of the timed run vs the EXACT GPU run (bit-identical to the reference "
                   "when exact_equals_reference) and vs the FP64 GPU propagator"}


def run_gpu(args, rank, world, device, physics="elastic2d"):
    import ctypes as C
    import torch
    from rockseis_b200 import abi
    from rockseis_b200.rockseis import Plan, make_config, make_shot
    precision = abi.F32_FAST if args.precision == "fast" else abi.F32_EXACT
    nt = args.nt if physics == "elastic2d" else min(args.nt, W.C1["nt"])
    if physics == "elastic2d":
        vp, vs, rho, sx, wav, gc = workload_inputs()
        build = lambda pinned: build_batch(precision, vp, vs, rho, sx, wav, gc, nt=nt, pinned=pinned)  # noqa: E731
    else:
        build = lambda pinned: build_c1(precision, nt, pinned=pinned)  # noqa: E731
    models, srcs, recs = build(False)
    torch.cuda.set_device(device)
    plan = Plan(models, srcs, recs, ORDER, precision, args.tile if args.tile >= -1 else -1,
                launch_mode=args.launch_mode, zchunk=args.zchunk)
    mode, items, band = plan.info()
    if mode not in (3, 4):
        # per-tile kernels: the tile shape is the autotuner's pick (cached in JSON), measured before timing
        plan.close()
        from rockseis_b200.autotune import tune_tile
        tile = tune_tile(models, srcs, recs, ORDER, precision) if args.tile == -2 else args.tile
        plan = Plan(models, srcs, recs, ORDER, precision, tile, launch_mode=args.launch_mode)
    plan.enable_timing()
    st = torch.cuda.ExternalStream(plan.stream())
    pts_per_step = sum(m.getNx_pml() * m.getNz_pml() for m in models) * nt

    def one_step():
        plan.reset()
        plan.run(0, nt)

    for _ in range(args.warmup):
        one_step()
    plan.sync()
    dist_barrier(world)
    torch.cuda.synchronize()
    l0 = plan.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(device) as clk:
        e0.record(st)
        for _ in range(args.steps):
            one_step()
        e1.record(st)
        e1.synchronize()
    ms_total = e0.elapsed_time(e1)
    plan.sync()
    launches = plan.launch_count() - l0
    ms_a, ms_b = plan.kernel_times()
    fast0 = plan.read_traces(0)
    plan.close()
    torch.cuda.synchronize()
    dist_barrier(world)
    ms_max = dist_max(ms_total, world)
    ms_step = ms_max / args.steps
    value = pts_per_step * world / (ms_step / 1e3) / 1e9

    # roofline of the dominant kernel (CUDA events recorded inside the replayed graph)
    b_fused, b_vel, b_str, pts = algorithmic_bytes(models, physics)
    peak, peak_kind = measured_peak()
    tag = "elastic2d_16shots" if physics == "elastic2d" else "acoustic2d_1shot"
    if mode == 3:
        dom, ms_dom, b_dom = "zm_step_2d", ms_a, b_fused
        extra = {"launch": "fused z-marching step (velocity + stress + injection + recording of the previous "
                           "step)", "work_items": items, "rows_per_item": band}
    elif mode == 4:
        dom, ms_dom, b_dom = ("e2d_march_stress", ms_b, b_str) if ms_b >= ms_a else ("e2d_march_velocity", ms_a, b_vel)
        extra = {"launch": "column-marching velocity and stress kernels", "ms_velocity": round(ms_a, 5),
                 "ms_stress": round(ms_b, 5), "work_items": items, "rows_per_item": band}
    else:
        dom, ms_dom, b_dom = (("e2d_stress" if physics == "elastic2d" else "a2d_stress"), ms_b, b_str) \
            if ms_b >= ms_a else (("e2d_velocity" if physics == "elastic2d" else "a2d_velocity"), ms_a, b_vel)
        extra = {"launch": "per-tile velocity and stress kernels", "ms_velocity": round(ms_a, 5),
                 "ms_stress": round(ms_b, 5)}
    achieved = b_dom / (ms_dom / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": read_traffic(dom, tag), "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": b_dom, "ms_per_launch": round(ms_dom, 5),
                "bytes_per_point_step": 60 if physics == "elastic2d" else 36,
                "step_frac_of_peak": round((b_fused * nt / (ms_step / 1e3) / 1e9) / peak, 4), **extra}
    parity = parity_figures(fast0, physics, nt) if (rank == 0 and args.precision == "fast") else None
    if args.no_e2e:
        return dict(value=value, ms_step=ms_step, launches=launches, roofline=roofline, e2e=None,
                    clocks=clk.summary(), parity=parity, mode=mode)

    # end to end through the C ABI from pinned host buffers
    models_p, srcs_p, recs_p = build(True)
    cfg = make_config(models_p[0], ORDER, nt, srcs_p[0].dt, precision, -1)
    cfg.launch_mode, cfg.zchunk = int(args.launch_mode), int(args.zchunk)
    keep: list = []
    ns = len(models_p)
    shots = (abi.Shot * ns)(*[make_shot(m, s, r, keep) for m, s, r in zip(models_p, srcs_p, recs_p)])
    h2d = sum(sum(a.nbytes for a in m.padded()) for m in models_p) + sum(s.data.nbytes + s.smap.nbytes +
                                                                        s.sshift.nbytes for s in srcs_p)
    h2d += sum(r.gmap.nbytes + r.gshift.nbytes for r in recs_p)
    d2h = sum(r.data.nbytes for r in recs_p)
    abi.check(abi.lib.rsgpu_modelling(C.byref(cfg), ns, shots))
    dist_barrier(world)
    e2e_steps = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for r in recs_p:
            r.data[:] = 0
        abi.check(abi.lib.rsgpu_modelling(C.byref(cfg), ns, shots))
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e_s = dist_max(e2e_s * 1e3, world) / 1e3
    e2e = {"value": round(pts_per_step * world / e2e_s / 1e9, 3), "unit": "Gpts/s", "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
           "path": "rsgpu_modelling (C ABI): plan create + upload, nt steps, trace read-back, destroy",
           "phases_ms": e2e_phases(cfg, ns, shots, recs_p)}
    return dict(value=value, ms_step=ms_step, launches=launches, roofline=roofline, e2e=e2e, clocks=clk.summary(),
                parity=parity, mode=mode)


def e2e_phases(cfg, ns, shots, recs):
    """The same work as one rsgpu_modelling call, split into its C ABI phases and
    timed on the host: plan creation with the uploads, the nt steps, the trace
    read-back into the host arrays, and the plan's destruction."""
    import ctypes as C
    from rockseis_b200 import abi
    for r in recs:
        r.data[:] = 0
    h = C.c_void_p()
    t0 = time.perf_counter()
    abi.check(abi.lib.rsgpu_plan_create(C.byref(cfg), ns, shots, C.byref(h)))
    abi.check(abi.lib.rsgpu_plan_sync(h))
    t1 = time.perf_counter()
    abi.check(abi.lib.rsgpu_plan_run(h, 0, cfg.nt))
    abi.check(abi.lib.rsgpu_plan_sync(h))
    t2 = time.perf_counter()
    for i, r in enumerate(recs):
        abi.check(abi.lib.rsgpu_plan_read_traces(h, i, r.data.ctypes.data))
    t3 = time.perf_counter()
    abi.lib.rsgpu_plan_destroy(h)
    t4 = time.perf_counter()
    return {"create_upload": round((t1 - t0) * 1e3, 2), "run": round((t2 - t1) * 1e3, 2),
            "read_traces": round((t3 - t2) * 1e3, 2), "destroy": round((t4 - t3) * 1e3, 2)}


# ---------------------------------------------------------------- FWI gradient workload
FWI = dict(nx=601, nz=201, dx=10.0, lpml=20, order=8, nt=3000, dt=1e-3, nshots=64, ncheck=50, f0=10.0, sz=20.0,
           nrec=601, plain_sample=4)


def fwi_problem(precision, nshots, nt=None, start=True, f=FWI):
    """Models, sources and receiver sets of the FWI workload (one Data2D pair per shot)."""
    from rockseis_b200 import abi, synth
    from rockseis_b200.rockseis import Data2D, ModelAcoustic2D
    nt = nt or f["nt"]
    vt, vs = synth.fwi_models(f["nx"], f["nz"], f["dx"])
    m = ModelAcoustic2D(f["nx"], f["nz"], f["lpml"], f["dx"], f["dx"], 0.0, 0.0, 0, precision)
    m.createModel()
    m.Vp[:] = vs if start else vt
    m.R[:] = synth.gardner(m.Vp)
    wav = synth.ricker(nt, f["dt"], f["f0"], abi.real_dtype(precision))
    sx = np.linspace(60.0, (f["nx"] - 1) * f["dx"] - 60.0, f["nshots"])[:nshots]
    gc = synth.surface_line(f["nrec"], 0.0, f["dx"], 0.0)
    srcs, recs = [], []
    for x in sx:
        s_ = Data2D(1, nt, f["dt"], 0.0, precision)
        s_.scoords[:] = [[x, f["sz"]]]
        s_.data[:] = wav[None, :]
        s_.makeMap(m, 0)
        r = Data2D(f["nrec"], nt, f["dt"], 0.0, precision)
        r.gcoords[:] = gc
        r.makeMap(m, 1)
        srcs.append(s_)
        recs.append(r)
    return m, srcs, recs


def fwi_jobs(m, srcs, obs, precision, ckpt, accum, f=FWI, tile=-1):
    from rockseis_b200 import abi
    from rockseis_b200.rockseis import Data2D, FwiAcoustic2D, Image2D
    jobs = []
    for s_, o in zip(srcs, obs):
        j = FwiAcoustic2D(m, s_, o, f["order"], 1, precision=precision)
        j.setNcheck(f["ncheck"])
        j.tile = tile
        j.setCheckpointPrecision(ckpt)
        j.setAccumulation(accum)
        j.setVpgrad(Image2D("vpgrad", m, 1, 1, precision))
        j.setRhograd(Image2D("rhograd", m, 1, 1, precision))
        j.setWavgrad(Data2D(s_.ntrace, s_.nt, s_.dt, 0.0, precision))
        jobs.append(j)
    return jobs


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _fwi_ref_sample(args):
    """One process: the reference's FwiAcoustic2D::run_optimal on one shot, shortened time axis."""
    shot, nt = args
    sys.path.insert(0, ROOT)
    from oracle import api
    from rockseis_b200 import synth
    f = FWI
    vt, vs = synth.fwi_models(f["nx"], f["nz"], f["dx"])
    rho = synth.gardner(vs)
    pb = api.Problem2D(f["nx"], f["nz"], f["dx"], f["dx"], f["lpml"], f["order"], 0, f["dt"], nt, vs, rho)
    sx = np.linspace(60.0, (f["nx"] - 1) * f["dx"] - 60.0, f["nshots"])[shot % f["nshots"]]
    gc = synth.surface_line(f["nrec"], 0.0, f["dx"], 0.0)
    wav = synth.ricker(nt, f["dt"], f["f0"])[None, :]
    obs = np.zeros((f["nrec"], nt), np.float32)
    t0 = time.perf_counter()
    api.ref_fwi_a2d(pb, np.array([[sx, f["sz"]]]), wav, gc, obs, f["ncheck"])
    return time.perf_counter() - t0


def cpu_fwi_reference(nt_sample=300, procs=None, f=FWI):
    """The reference's CPU gradient, one shot per process on all host cores, on the full
    grid with a shortened time axis, extrapolated to nt by the propagation work
    (Revolve forward steps + adjoint steps + correlations)."""
    import multiprocessing as mp
    from oracle import api
    from rockseis_b200 import abi
    if not api.ref_available():
        return None
    procs = procs or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        times = pool.map(_fwi_ref_sample, [(i, nt_sample) for i in range(procs)])

    def work(nt):
        return abi.lib.rsgpu_revolve_numforw(nt, f["ncheck"]) + 1 + 2 * nt
    t_shot = max(times) * work(f["nt"]) / work(nt_sample)
    return {"value": round(procs / t_shot, 5), "unit": "shots/s", "cores": procs, "kind": "reference",
            "sample": f"{procs} processes x 1 shot, full 641x241 padded grid, nt={nt_sample} (ncheck "
                      f"{f['ncheck']}), extrapolated to nt={f['nt']} by Revolve forward + adjoint + "
                      f"correlation steps", "max_process_s": round(max(times), 3)}


def _timed_runs(batch, steps):
    import torch
    st = torch.cuda.ExternalStream(batch.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        batch.run()
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3 / steps


def fwi_config(f=FWI):
    return {"workload": "acoustic2d_fwi_gradient_64shots_601x201_nt3000_ncheck50", "nx": f["nx"], "nz": f["nz"],
            "dx": f["dx"], "lpml": f["lpml"], "order": f["order"], "nt": f["nt"], "dt": f["dt"],
            "shots": f["nshots"], "receivers": f["nrec"], "ncheck": f["ncheck"],
            "l2": "working set > 126 MB L2 (no flush needed)"}


def run_fwi(args, device=0, f=FWI):
    """Shots/s of the checkpointed FWI gradient: all shots batched vs one shot at a time."""
    from rockseis_b200 import abi
    from rockseis_b200.rockseis import AdjointBatch, fwi_gradient_batch, modelling_batch
    ns = min(args.shots or f["nshots"], f["nshots"])
    prec, ckpt, accum = abi.F32_FAST, abi.CKPT_F16, abi.ACCUM_F64
    # observed data: modelled in the true model on the GPU
    mt, srcs, obs = fwi_problem(prec, ns, start=False)
    modelling_batch([mt] * ns, srcs, obs, f["order"], prec)
    m, srcs, _ = fwi_problem(prec, ns)
    # tile shape: autotuned per batch shape (-2) unless --tile names one
    jobs = fwi_jobs(m, srcs, obs, prec, ckpt, accum, tile=getattr(args, "tile", -1))
    batch = AdjointBatch(jobs)
    batch.run()                                   # warm-up (graph capture, first touch)
    with ClockSampler(device) as clk:
        t_batch = _timed_runs(batch, max(1, args.fwi_steps))
    stats = batch.stats()
    batch.read()
    g0 = jobs[0].vpgrad.getImagedata()[0, 0].copy()
    batch.close()
    # one shot at a time, same settings (sample of the shots)
    t_plain = []
    for j in jobs[:f["plain_sample"]]:
        b1 = AdjointBatch([j])
        b1.run()
        t_plain.append(_timed_runs(b1, 1))
        b1.close()
    plain = len(t_plain) / sum(t_plain)
    # accuracy of shot 0 against the FP64 propagator (lossless checkpoints, FP64 accumulation)
    m64, s64, o64 = fwi_problem(abi.F64, 1)
    o64[0].data = obs[0].data.astype(np.float64)
    j64 = fwi_jobs(m64, s64, o64, abi.F64, abi.CKPT_NATIVE, abi.ACCUM_F64)
    b64 = AdjointBatch(j64)
    b64.run()
    b64.read()
    g64 = j64[0].vpgrad.getImagedata()[0, 0]
    b64.close()
    err = rel_l2(g0, g64)
    pts = (f["nx"] + 2 * f["lpml"]) * (f["nz"] + 2 * f["lpml"])
    # end to end: one rsgpu_fwi_gradient call from host buffers (plan creation, upload of
    # models, maps, wavelets and observed data, the gradient, read-back of all outputs)
    e2e = None
    if not args.no_e2e:
        for j in jobs:
            for img in (j.vpgrad, j.rhograd):
                img.getImagedata()[:] = 0
            j.wavgrad.data[:] = 0
        t0 = time.perf_counter()
        fwi_gradient_batch(jobs)
        t_e2e = time.perf_counter() - t0
        h2d = sum(m_.nbytes for m_ in m.padded()) * ns + sum(o.data.nbytes + o.gmap.nbytes + o.gshift.nbytes
                                                                for o in obs)
        h2d += ns * (m.Vp.nbytes + m.R.nbytes) + sum(s_.data.nbytes for s_ in srcs)
        d2h = ns * (2 * m.Vp.nbytes + srcs[0].data.nbytes)
        e2e = {"value": round(ns / t_e2e, 3), "unit": "shots/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "path": "rsgpu_fwi_gradient (C ABI) from host buffers"}
    # whole-gradient roofline with the byte budget of the workload: forward steps 36 B per
    # point (P, Vx, Vz read and written, Rx, Rz, L read), adjoint step with correlation
    # 80 B (the same 36 + forward P 4 + vp, rho 8 + two FP64 gradients read and written
    # 32), plus the checkpoint bytes written and read by the schedule
    peak, peak_kind = measured_peak()
    grad_bytes = ns * pts * (36.0 * stats["fw_steps"] + 80.0 * stats["bw_steps"]) + stats["ckpt_bytes"]
    roof = {"bound": "hbm", "kernel": "whole gradient (forward, adjoint, correlation, checkpoints)",
            "achieved": round(grad_bytes / t_batch / 1e9, 1), "peak": peak, "unit": "GB/s",
            "frac": round(grad_bytes / t_batch / 1e9 / peak, 4), "peak_source": peak_kind,
            "algorithmic_bytes": "36 B per forward point-step, 80 B per adjoint+correlation point-step, "
                                 "checkpoint bytes from the schedule", "traffic": None}
    return {"metric": "FWI gradient shots/s", "shots_per_s_batched": round(ns / t_batch, 3),
            "shots_per_s_plain": round(plain, 3), "batched_over_plain": round((ns / t_batch) / plain, 2),
            "s_per_batch": round(t_batch, 4), "plain_sample_shots": len(t_plain),
            "gradient_rel_l2_vs_fp64": float("%.3g" % err), "arithmetic": "FMA f32, FP16-scaled checkpoints, "
            "FP64 accumulation", "forward_steps": stats["fw_steps"], "adjoint_steps": stats["bw_steps"],
            "checkpoint_bytes": stats["ckpt_bytes"], "gpu_launches": stats["launches"],
            "gpts_per_s_propagation": round(ns * pts * (stats["fw_steps"] + stats["bw_steps"]) / t_batch / 1e9, 3),
            "roofline": roof, "config": fwi_config(), "e2e": e2e, "clocks": clk.summary()}


# ---------------------------------------------------------------- 3D acoustic workload
A3D = dict(nx=400, ny=400, nz=300, dx=12.5, lpml=20, order=8, nt=2500, dt=1e-3, nshots=32, chunk=20, nrec=201,
           f0=12.0, sz=25.0)


def a3d_config(nshots=None, f=A3D):
    ns = f["nshots"] if nshots is None else min(nshots, f["nshots"])
    return {"workload": f"acoustic3d_forward_{ns}shots_400x400x300_windows_nt2500", "nx": f["nx"], "ny": f["ny"],
            "nz": f["nz"], "dx": f["dx"], "lpml": f["lpml"], "order": f["order"], "nt": f["nt"], "dt": f["dt"],
            "shots": ns, "time_steps_per_bench_step": f["chunk"],
            "windows": "per-shot aperture windows (apertures uniform in [1500, 5000] m, seed 6)",
            "l2": "working set tens of GB > 126 MB L2 (no flush needed)"}


def a3d_batch(precision, f=A3D, nshots=None):
    """The windowed shots of the 3D workload (the first nshots of 32): (local models, sources, receivers)."""
    from rockseis_b200 import abi, synth
    from rockseis_b200.rockseis import SMAP, Data3D, ModelAcoustic3D
    vp = synth.dipping_vp_3d(f["nx"], f["ny"], f["nz"], f["dx"], seed=5, vclip=4550.0)
    big = ModelAcoustic3D(f["nx"], f["ny"], f["nz"], f["lpml"], f["dx"], f["dx"], f["dx"], 0.0, 0.0, 0.0, 0, precision)
    big.createModel()
    big.Vp[:] = vp
    big.R[:] = synth.gardner(vp)
    del vp
    rng = np.random.default_rng(6)
    ext = (f["nx"] - 1) * f["dx"], (f["ny"] - 1) * f["dx"]
    gx, gy = np.meshgrid(np.linspace(0.1, 0.9, 8), np.linspace(0.15, 0.85, 4))
    pos = np.stack([gx.ravel() * ext[0], gy.ravel() * ext[1]], 1) + rng.uniform(-150, 150, (f["nshots"], 2))
    apert = rng.uniform(1500.0, 5000.0, (f["nshots"], 2))
    wav = synth.ricker(f["nt"], f["dt"], f["f0"], abi.real_dtype(precision))
    models, srcs, recs = [], [], []
    for k in range(f["nshots"] if nshots is None else min(nshots, f["nshots"])):
        sx, sy = pos[k]
        s_ = Data3D(1, f["nt"], f["dt"], 0.0, precision)
        s_.scoords[:] = [[sx, sy, f["sz"]]]
        xs = np.clip(sx + np.linspace(-1250.0, 1250.0, f["nrec"]), 0.0, ext[0])
        r = Data3D(f["nrec"], f["nt"], f["dt"], 0.0, precision)
        r.gcoords[:] = np.stack([xs, np.full(f["nrec"], sy), np.zeros(f["nrec"])], 1)
        s_.gcoords[:] = [[sx, sy, 0.0]]
        m = big.getLocal(s_, apert[k, 0], apert[k, 1], SMAP)
        s_.data[:] = wav[None, :]
        s_.makeMap(m, 0)
        r.makeMap(m, 1)
        models.append(m)
        srcs.append(s_)
        recs.append(r)
    return models, srcs, recs


def _a3d_ref_sample(args):
    """One process: the reference's ModellingAcoustic3D::run on one mean-size window, few steps."""
    nxw, nyw, nsteps = args
    sys.path.insert(0, ROOT)
    from oracle import api
    from rockseis_b200 import synth
    f = A3D
    vp = synth.dipping_vp_3d(nxw, nyw, f["nz"], f["dx"], seed=5, vclip=4550.0)
    pb = api.Problem3D(nxw, nyw, f["nz"], f["dx"], f["dx"], f["dx"], f["lpml"], f["order"], 0, f["dt"], nsteps, vp,
                       synth.gardner(vp))
    wav = synth.ricker(nsteps, f["dt"], f["f0"])[None, :]
    c = nxw * f["dx"] / 2
    t0 = time.perf_counter()
    api.ref_modelling_a3d(pb, np.array([[c, c, f["sz"]]]), wav, 0, np.array([[c, c, 0.0]]), 0)
    return time.perf_counter() - t0


def cpu_a3d_reference(models, nsteps=6, procs=None, f=A3D):
    """Reference CPU 3D modelling, one mean-size window per process, first nsteps steps."""
    import multiprocessing as mp
    from oracle import api
    if not api.ref_available():
        return None
    procs = procs or min(8, os.cpu_count() or 1)
    nxw = int(round(np.mean([m.nx for m in models])))
    nyw = int(round(np.mean([m.ny for m in models])))
    with mp.get_context("spawn").Pool(procs) as pool:
        times = pool.map(_a3d_ref_sample, [(nxw, nyw, nsteps)] * procs)
    L = f["lpml"]
    pts = (nxw + 2 * L) * (nyw + 2 * L) * (f["nz"] + 2 * L) * nsteps * procs
    return {"value": round(pts / max(times) / 1e9, 5), "unit": "Gpts/s", "cores": procs, "kind": "reference",
            "sample": f"{procs} processes x one {nxw}x{nyw}x{f['nz']} window (the batch's mean), first {nsteps} "
                      f"steps", "max_process_s": round(max(times), 3)}


def a3d_strip_points(models, L):
    """Point-axis pairs in the C-PML strips of the 3D windows: sum over windows of the
    points in the x, the y and the z strips (a corner point counts once per axis).
    Each velocity and each stress half-step reads and writes one 4-byte memory
    variable per pair: 16 B per pair and time step."""
    n = 0
    for m in models:
        nx, ny, nz = m.nx + 2 * L, m.ny + 2 * L, m.nz + 2 * L
        n += 2 * L * ny * nz + nx * 2 * L * nz + nx * ny * 2 * L
    return n


def run_a3d(args, device=0, f=A3D):
    """Gpts/s of the windowed 3D batch: chunks of time steps of all 32 shots."""
    import ctypes as C
    import torch
    from rockseis_b200 import abi
    from rockseis_b200.rockseis import make_config, make_shot
    prec = abi.F32_FAST if args.precision == "fast" else abi.F32_EXACT
    models, srcs, recs = a3d_batch(prec, nshots=args.shots)
    cfg = make_config(models[0], f["order"], f["nt"], f["dt"], prec)
    cfg.zchunk = int(args.zchunk)
    keep: list = []
    shots = (abi.Shot * len(models))(*[make_shot(m, s_, r, keep) for m, s_, r in zip(models, srcs, recs)])
    h = C.c_void_p()
    abi.check(abi.lib.rsgpu_plan_create(C.byref(cfg), len(models), shots, C.byref(h)))
    L = f["lpml"]
    pts = sum((m.nx + 2 * L) * (m.ny + 2 * L) * (m.nz + 2 * L) for m in models)
    win = [(m.nx, m.ny) for m in models]
    del keep, shots
    for m in models:
        m._padded = {}
    st = torch.cuda.ExternalStream(abi.lib.rsgpu_plan_stream(h))
    ch = f["chunk"]
    it = 0
    for _ in range(args.warmup):
        abi.check(abi.lib.rsgpu_plan_run(h, it, ch))
        it += ch
    abi.check(abi.lib.rsgpu_plan_sync(h))
    l0 = abi.lib.rsgpu_plan_launch_count(h)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(device) as clk:
        e0.record(st)
        for _ in range(args.steps):
            abi.check(abi.lib.rsgpu_plan_run(h, it, ch))
            it += ch
        e1.record(st)
        e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    abi.check(abi.lib.rsgpu_plan_sync(h))
    launches = abi.lib.rsgpu_plan_launch_count(h) - l0
    abi.lib.rsgpu_plan_destroy(h)
    value = pts * ch / (ms / 1e3) / 1e9
    # algorithmic bytes per time step: velocity reads P,Vx,Vy,Vz,Rx,Ry,Rz, writes Vx,Vy,Vz (40 B);
    # stress reads Vx,Vy,Vz,P,L, writes P (24 B); 16 B per C-PML strip point-axis pair
    peak, peak_kind = measured_peak()
    strip = a3d_strip_points(models, L)
    achieved = (64.0 * pts + 16.0 * strip) * ch / (ms / 1e3) / 1e9
    return {"metric": "Gpts/s", "value": round(value, 3), "unit": "Gpts/s", "ms_per_step": round(ms, 3),
            "gpu_launches": int(launches), "padded_points_per_step": int(pts),
            "window_sizes": {"min": min(win), "max": max(win)},
            "roofline": {"bound": "hbm", "kernel": "a3d_velocity + a3d_stress (whole step)",
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "algorithmic_bytes_per_point_step": 64, "cpml_bytes_per_strip_point_step": 16,
                         "strip_points": int(strip)},
            "clocks": clk.summary(), "models": models}


# ---------------------------------------------------------------- 3D elastic FWI workload
E3D = dict(W.C5, ncheck=10, nt_bench=200, plain_sample=1)


def e3d_config(nt, ncheck, f=E3D):
    return {"workload": f"elastic3d_fwi_gradient_16shots_256cubed_nt{nt}", "nx": f["nx"], "ny": f["ny"],
            "nz": f["nz"], "dx": f["dx"], "lpml": f["lpml"], "order": f["order"], "dt": f["dt"], "nt": nt,
            "nt_full": f["nt"], "shots": f["nshots"], "receivers": f["nrec_side"] ** 2, "ncheck": ncheck,
            "checkpoints": "BF16, power-of-two scale per field array", "accumulation": "FP64",
            "l2": "working set tens of GB > 126 MB L2 (no flush needed)"}


def e3d_problem(precision, nt, true_model=False, nshots=None, f=E3D):
    """Model, sources and Ux/Uy/Uz receiver sets of the elastic 3D FWI workload."""
    from rockseis_b200 import abi
    from rockseis_b200.rockseis import Data3D, ModelElastic3D
    vp, vs, rho, src, wav, rec = W.elastic3d_c5(nt, true_model)
    m = ModelElastic3D(f["nx"], f["ny"], f["nz"], f["lpml"], f["dx"], f["dx"], f["dx"], 0.0, 0.0, 0.0, 0, precision)
    m.createModel()
    m.Vp[:], m.Vs[:], m.R[:] = vp, vs, rho
    del vp, vs, rho
    t = abi.real_dtype(precision)
    srcs, recsets = [], []
    for xyz in src[: nshots or f["nshots"]]:
        s_ = Data3D(1, nt, f["dt"], 0.0, precision)
        s_.scoords[:] = [xyz]
        s_.data[:] = wav.astype(t)[None, :]
        s_.makeMap(m, 0)
        sets = []
        for fld in (abi.VX, abi.VY, abi.VZ):
            r = Data3D(len(rec), nt, f["dt"], 0.0, precision)
            r.gcoords[:] = rec
            r.setField(fld)
            r.makeMap(m, 1)
            sets.append(r)
        srcs.append(s_)
        recsets.append(sets)
    return m, srcs, recsets


def e3d_jobs(m, srcs, recsets, precision, ckpt, accum, ncheck, f=E3D):
    from rockseis_b200.rockseis import Data3D, FwiElastic3D, Image3D
    jobs = []
    for s_, (rx, ry, rz) in zip(srcs, recsets):
        j = FwiElastic3D(m, s_, rx, ry, rz, f["order"], 1, precision=precision)
        j.setNcheck(ncheck)
        j.setCheckpointPrecision(ckpt)
        j.setAccumulation(accum)
        j.setVpgrad(Image3D("vpgrad", m, 1, 1, 1, precision))
        j.setVsgrad(Image3D("vsgrad", m, 1, 1, 1, precision))
        j.setRhograd(Image3D("rhograd", m, 1, 1, 1, precision))
        j.setWavgrad(Data3D(s_.ntrace, s_.nt, s_.dt, 0.0, precision))
        jobs.append(j)
    return jobs


def _e3d_ref_sample(args):
    """One process: the reference's FwiElastic3D::run_optimal for one shot on the full
    256^3 grid (296^3 padded) with a time axis of nt steps."""
    shot, nt, ncheck = args
    sys.path.insert(0, ROOT)
    from oracle import api
    f = E3D
    vp, vs, rho, src, wav, rec = W.elastic3d_c5(nt)
    pb = api.Problem3D(f["nx"], f["ny"], f["nz"], f["dx"], f["dx"], f["dx"], f["lpml"], f["order"], 0, f["dt"], nt,
                       vp, rho, vs)
    obs = [np.zeros((len(rec), nt), np.float32)] * 3
    t0 = time.perf_counter()
    api.ref_fwi_e3d(pb, src[shot % len(src)][None, :], wav[None, :], 0, rec, obs, ncheck)
    return time.perf_counter() - t0


def cpu_e3d_reference(ncheck_full, nt_target, nt_sample=3, procs=None, f=E3D):
    """The reference's CPU gradient, one full-grid shot per process, nt_sample steps,
    extrapolated to nt_target by the propagation work (Revolve forward steps + adjoint
    steps + correlations) at the GPU run's snapshot count."""
    import multiprocessing as mp
    from oracle import api
    from rockseis_b200 import abi
    if not api.ref_available():
        return None
    procs = procs or max(1, min(4, (os.cpu_count() or 1)))
    with mp.get_context("spawn").Pool(procs) as pool:
        times = pool.map(_e3d_ref_sample, [(i, nt_sample, 2) for i in range(procs)])

    def work(nt, nc):
        return abi.lib.rsgpu_revolve_numforw(nt, nc) + 1 + 2 * nt
    t_shot = max(times) * work(nt_target, ncheck_full) / work(nt_sample, 2)
    return {"value": float("%.4g" % (procs / t_shot)), "unit": "shots/s", "cores": procs, "kind": "reference",
            "sample": f"{procs} processes x 1 shot, full 296^3 padded grid, nt={nt_sample} (ncheck 2), "
                      f"extrapolated to nt={nt_target} with ncheck {ncheck_full} by Revolve forward + adjoint + "
                      f"correlation steps", "max_process_s": round(max(times), 3)}


def e3d_forward_config(nshots, f=E3D):
    return {"workload": f"elastic3d_forward_{nshots}shots_256cubed", "nx": f["nx"], "ny": f["ny"], "nz": f["nz"],
            "dx": f["dx"], "lpml": f["lpml"], "order": f["order"], "dt": f["dt"], "nt": f["nt"], "shots": nshots,
            "time_steps_per_bench_step": 20, "receivers": f["nrec_side"] ** 2,
            "l2": "working set > 126 MB L2 (no flush needed)"}


def run_e3d_forward(args, device=0, f=E3D):
    """Gpts/s of the elastic 3D forward modelling of the C5 shots (Vx receivers):
    bench steps of 20 time steps of the whole batch."""
    import ctypes as C
    import torch
    from rockseis_b200 import abi
    from rockseis_b200.rockseis import make_config, make_shot
    prec = abi.F32_FAST if args.precision == "fast" else abi.F32_EXACT
    ns = args.shots or f["nshots"]
    m, srcs, recsets = e3d_problem(prec, f["nt"], True, ns)
    cfg = make_config(m, f["order"], f["nt"], f["dt"], prec)
    cfg.zchunk = int(args.zchunk)
    keep: list = []
    shots = (abi.Shot * ns)(*[make_shot(m, s_, rs[0], keep) for s_, rs in zip(srcs, recsets)])
    h = C.c_void_p()
    abi.check(abi.lib.rsgpu_plan_create(C.byref(cfg), ns, shots, C.byref(h)))
    del keep, shots
    L = f["lpml"]
    pts = ns * (f["nx"] + 2 * L) * (f["ny"] + 2 * L) * (f["nz"] + 2 * L)
    st = torch.cuda.ExternalStream(abi.lib.rsgpu_plan_stream(h))
    ch, it = 20, 0
    for _ in range(args.warmup):
        abi.check(abi.lib.rsgpu_plan_run(h, it, ch))
        it += ch
    abi.check(abi.lib.rsgpu_plan_sync(h))
    l0 = abi.lib.rsgpu_plan_launch_count(h)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(device) as clk:
        e0.record(st)
        for _ in range(args.steps):
            abi.check(abi.lib.rsgpu_plan_run(h, it, ch))
            it += ch
        e1.record(st)
        e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    launches = abi.lib.rsgpu_plan_launch_count(h) - l0
    abi.lib.rsgpu_plan_destroy(h)
    peak, peak_kind = measured_peak()
    achieved = 140.0 * pts * ch / (ms / 1e3) / 1e9
    return {"metric": "Gpts/s", "value": round(pts * ch / (ms / 1e3) / 1e9, 3), "unit": "Gpts/s",
            "ms_per_step": round(ms, 3), "gpu_launches": int(launches), "padded_points_per_step": int(pts),
            "roofline": {"bound": "hbm", "kernel": "e3d_velocity + e3d_stress + inject_record_e3d (whole step)",
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "algorithmic_bytes_per_point_step": 140, "traffic": None},
            "clocks": clk.summary(), "config": e3d_forward_config(ns)}


def run_e3d(args, device=0, f=E3D):
    """Shots/s of the batched elastic 3D FWI gradient (FMA, BF16 checkpoints, FP64
    accumulation) on a shortened time axis, the one-shot-at-a-time gradient beside it,
    the FP64 error of shot 0, and the forward step's roofline."""
    import ctypes as C
    import torch
    from rockseis_b200 import abi
    from rockseis_b200.rockseis import AdjointBatch, fwi_gradient_batch, make_config, make_shot
    nt = int(args.e3d_nt)
    ns = args.shots or f["nshots"]
    prec, ckpt, accum = abi.F32_FAST, abi.CKPT_BF16, abi.ACCUM_F64
    # observed data: the three components modelled in the true model (batched plans)
    mt, srcs, recsets = e3d_problem(prec, nt, True, ns)
    for k in range(3):
        cfg = make_config(mt, f["order"], nt, f["dt"], prec)
        keep: list = []
        shots = (abi.Shot * ns)(*[make_shot(mt, s_, rs[k], keep) for s_, rs in zip(srcs, recsets)])
        abi.check(abi.lib.rsgpu_modelling(C.byref(cfg), ns, shots))
        del keep, shots
    obs = [[r.data.copy() for r in rs] for rs in recsets]
    del mt
    m, srcs, recsets = e3d_problem(prec, nt, False, ns)
    for rs, o in zip(recsets, obs):
        for r, d in zip(rs, o):
            r.data = d
    # ten Revolve snapshots: what fits next to the two propagators of 16 shots in HBM
    L = f["lpml"]
    pts = (f["nx"] + 2 * L) * (f["ny"] + 2 * L) * (f["nz"] + 2 * L)
    ncheck = f["ncheck"]
    jobs = e3d_jobs(m, srcs, recsets, prec, ckpt, accum, ncheck)
    batch = AdjointBatch(jobs)
    batch.run()                                   # warm-up
    with ClockSampler(device) as clk:
        t_batch = _timed_runs(batch, max(1, args.fwi_steps))
    stats = batch.stats()
    batch.read()
    g0 = jobs[0].vpgrad.getImagedata()[0, 0, 0].copy()
    batch.close()
    torch.cuda.empty_cache()
    t_plain = []
    for j in jobs[: f["plain_sample"]]:
        b1 = AdjointBatch([j])
        b1.run()
        t_plain.append(_timed_runs(b1, 1))
        b1.close()
    plain = len(t_plain) / sum(t_plain)
    # FP64 gradient of shot 0 (lossless checkpoints, FP64 accumulation)
    m64, s64, r64 = e3d_problem(abi.F64, nt, False, 1)
    for r, d in zip(r64[0], obs[0]):
        r.data = d.astype(np.float64)
    j64 = e3d_jobs(m64, s64, r64, abi.F64, abi.CKPT_NATIVE, abi.ACCUM_F64, ncheck)
    b64 = AdjointBatch(j64)
    b64.run()
    b64.read()
    err = rel_l2(g0, j64[0].vpgrad.getImagedata()[0, 0, 0])
    b64.close()
    del m64, j64
    torch.cuda.empty_cache()
    # forward step of the batch alone: CUDA events around chunks of time steps
    cfg = make_config(m, f["order"], nt, f["dt"], prec)
    keep = []
    shots = (abi.Shot * ns)(*[make_shot(m, s_, rs[0], keep) for s_, rs in zip(srcs, recsets)])
    h = C.c_void_p()
    abi.check(abi.lib.rsgpu_plan_create(C.byref(cfg), ns, shots, C.byref(h)))
    st = torch.cuda.ExternalStream(abi.lib.rsgpu_plan_stream(h))
    abi.check(abi.lib.rsgpu_plan_run(h, 0, 5))
    ch = 20
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    abi.check(abi.lib.rsgpu_plan_run(h, 5, ch))
    e1.record(st)
    e1.synchronize()
    fw_ms = e0.elapsed_time(e1) / ch
    abi.lib.rsgpu_plan_destroy(h)
    del keep, shots
    peak, peak_kind = measured_peak()
    # algorithmic bytes per point and forward step: velocity reads 6 stresses, 3
    # velocities, Rx/Ry/Rz and writes 3 velocities (60 B); stress reads 3 velocities,
    # 6 stresses, 5 moduli and writes 6 stresses (80 B)
    achieved = 140.0 * ns * pts / (fw_ms / 1e3) / 1e9
    e2e = None
    if not args.no_e2e:
        for j in jobs:
            for img in (j.vpgrad, j.vsgrad, j.rhograd):
                img.getImagedata()[:] = 0
            j.wavgrad.data[:] = 0
        t0 = time.perf_counter()
        fwi_gradient_batch(jobs)
        t_e2e = time.perf_counter() - t0
        h2d = ns * (sum(a.nbytes for a in m.padded()) + 3 * m.Vp.nbytes +
                    sum(r.data.nbytes + r.gmap.nbytes + r.gshift.nbytes for r in recsets[0]) + srcs[0].data.nbytes)
        d2h = ns * (3 * m.Vp.nbytes + srcs[0].data.nbytes)
        e2e = {"value": float("%.4g" % (ns / t_e2e)), "unit": "shots/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "path": "rsgpu_fwi_gradient (C ABI) from host buffers"}
    work_full = abi.lib.rsgpu_revolve_numforw(f["nt"], ncheck) + 1 + 2 * f["nt"]
    work = stats["fw_steps"] + stats["bw_steps"] + 1
    # whole gradient against the workload's byte budget: 104 B per forward point-step
    # (nine fields read and written, eight parameters read), 188 B per adjoint step with
    # its correlation (104 + nine forward fields 36 + three FP64 gradients read and
    # written 48), plus the checkpoint bytes of the schedule
    grad_bytes = ns * pts * (104.0 * stats["fw_steps"] + 188.0 * stats["bw_steps"]) + stats["ckpt_bytes"]
    roof_grad = {"bound": "hbm", "kernel": "whole gradient (forward, adjoint, correlation, checkpoints)",
                 "achieved": round(grad_bytes / t_batch / 1e9, 1), "peak": peak, "unit": "GB/s",
                 "frac": round(grad_bytes / t_batch / 1e9 / peak, 4), "peak_source": peak_kind,
                 "algorithmic_bytes": "104 B per forward point-step, 188 B per adjoint+correlation point-step, "
                                      "checkpoint bytes from the schedule"}
    return {"shots_per_s_batched": float("%.4g" % (ns / t_batch)), "shots_per_s_plain": float("%.4g" % plain),
            "batched_over_plain": round((ns / t_batch) / plain, 2), "s_per_batch": round(t_batch, 3),
            "shots_per_s_at_full_nt_extrapolated": float("%.4g" % (ns / t_batch * work / work_full)),
            "gradient_rel_l2_vs_fp64": float("%.3g" % err), "ncheck": ncheck,
            "forward_steps": stats["fw_steps"], "adjoint_steps": stats["bw_steps"],
            "checkpoint_bytes": stats["ckpt_bytes"], "gpu_launches": stats["launches"],
            "gpts_per_s_propagation": round(ns * pts * (stats["fw_steps"] + stats["bw_steps"]) / t_batch / 1e9, 3),
            "forward_step_ms": round(fw_ms, 3), "forward_gpts_per_s": round(ns * pts / fw_ms / 1e6, 3),
            "roofline_gradient": roof_grad,
            "roofline": {"bound": "hbm", "kernel": "e3d_velocity + e3d_stress + inject_record_e3d (forward step)",
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "algorithmic_bytes_per_point_step": 140, "traffic": None},
            "config": e3d_config(nt, ncheck), "e2e": e2e, "clocks": clk.summary()}


# ---------------------------------------------------------------- 3D acoustic RTM workload
RTM3 = dict(nt_bench=250, ncheck=10)


def rtm3d_config(nt, nshots=None, f=A3D):
    c = a3d_config(nshots, f)
    c.update(workload=f"acoustic3d_rtm_{c['shots']}shots_400x400x300_windows_nt{nt}", nt=nt, nt_full=f["nt"],
             ncheck=RTM3["ncheck"], checkpoints="FP16, power-of-two scale per array", accumulation="FP64",
             image="zero lag")
    c.pop("time_steps_per_bench_step", None)
    return c


def _rtm3d_ref_sample(args):
    """One process: the reference's RtmAcoustic3D::run_optimal on one mean-size window, nt steps."""
    nxw, nyw, nt = args
    sys.path.insert(0, ROOT)
    from oracle import api
    from rockseis_b200 import synth
    f = A3D
    vp = synth.dipping_vp_3d(nxw, nyw, f["nz"], f["dx"], seed=5, vclip=4550.0)
    pb = api.Problem3D(nxw, nyw, f["nz"], f["dx"], f["dx"], f["dx"], f["lpml"], f["order"], 0, f["dt"], nt, vp,
                       synth.gardner(vp))
    wav = synth.ricker(nt, f["dt"], f["f0"])[None, :]
    c = nxw * f["dx"] / 2
    gc = np.stack([np.linspace(0.0, (nxw - 1) * f["dx"], f["nrec"]), np.full(f["nrec"], c), np.zeros(f["nrec"])], 1)
    data = np.zeros((f["nrec"], nt), np.float32)
    t0 = time.perf_counter()
    api.ref_rtm_a3d(pb, np.array([[c, c, f["sz"]]]), wav, gc, data, 2)
    return time.perf_counter() - t0


def cpu_rtm3d_reference(models, nt_target, ncheck, nt_sample=3, procs=None):
    """The reference's CPU RTM image on the batch's mean window, one per process, nt_sample
    steps, extrapolated to nt_target by Revolve forward steps + adjoint steps + correlations."""
    import multiprocessing as mp
    from oracle import api
    from rockseis_b200 import abi
    if not api.ref_available():
        return None
    procs = procs or min(8, os.cpu_count() or 1)
    nxw = int(round(np.mean([m.nx for m in models])))
    nyw = int(round(np.mean([m.ny for m in models])))
    with mp.get_context("spawn").Pool(procs) as pool:
        times = pool.map(_rtm3d_ref_sample, [(nxw, nyw, nt_sample)] * procs)

    def work(nt, nc):
        return abi.lib.rsgpu_revolve_numforw(nt, nc) + 1 + 2 * nt
    t_img = max(times) * work(nt_target, ncheck) / work(nt_sample, 2)
    return {"value": float("%.4g" % (procs / t_img)), "unit": "images/s", "cores": procs, "kind": "reference",
            "sample": f"{procs} processes x one {nxw}x{nyw}x{A3D['nz']} window (the batch's mean), nt={nt_sample} "
                      f"(ncheck 2), extrapolated to nt={nt_target} with ncheck {ncheck} by Revolve forward + "
                      f"adjoint + correlation steps", "max_process_s": round(max(times), 3)}


def run_rtm3d(args, device=0, f=A3D):
    """Shot images/s of the batched 3D RTM (zero lag) over the windowed C4 shots, on a
    shortened time axis: data modelled on the GPU in the same model, then one
    rsgpu_adjoint batch (FMA arithmetic, FP16 checkpoints, FP64 image accumulation)."""
    from rockseis_b200 import abi
    from rockseis_b200.rockseis import AdjointBatch, Image3D, RtmAcoustic3D, modelling_batch
    nt = int(args.rtm_nt)
    ff = dict(f, nt=nt)
    prec = abi.F32_FAST
    models, srcs, recs = a3d_batch(prec, f=ff, nshots=args.shots)
    ns = len(models)
    modelling_batch(models, srcs, recs, ff["order"], prec)
    jobs = []
    for m, s_, r in zip(models, srcs, recs):
        j = RtmAcoustic3D(m, Image3D("pimage", m, 1, 1, 1, prec), s_, r, ff["order"], 1, precision=prec)
        j.setNcheck(RTM3["ncheck"])
        j.setCheckpointPrecision(abi.CKPT_F16)
        j.setAccumulation(abi.ACCUM_F64)
        jobs.append(j)
    batch = AdjointBatch(jobs, kind=abi.KIND_RTM)
    batch.run()                                   # warm-up
    with ClockSampler(device) as clk:
        t_batch = _timed_runs(batch, max(1, args.fwi_steps))
    stats = batch.stats()
    batch.close()
    L = f["lpml"]
    pts = sum((m.nx + 2 * L) * (m.ny + 2 * L) * (m.nz + 2 * L) for m in models)
    peak, peak_kind = measured_peak()
    # 48 B per forward point-step (four fields read and written, four parameters read),
    # 60 B per adjoint step with the image correlation (48 + forward P 4 + FP32 image
    # read and written 8; FP64 accumulation moves 8 more), checkpoint bytes of the schedule
    img_bytes = pts * (48.0 * stats["fw_steps"] + 60.0 * stats["bw_steps"]) + stats["ckpt_bytes"] + \
        16.0 * a3d_strip_points(models, L) * (stats["fw_steps"] + stats["bw_steps"])
    roof = {"bound": "hbm", "kernel": "whole image (forward, adjoint, correlation, checkpoints)",
            "achieved": round(img_bytes / t_batch / 1e9, 1), "peak": peak, "unit": "GB/s",
            "frac": round(img_bytes / t_batch / 1e9 / peak, 4), "peak_source": peak_kind,
            "algorithmic_bytes": "48 B per forward point-step, 60 B per adjoint+correlation point-step, "
                                 "16 B per C-PML strip point-axis pair and step, checkpoint bytes from the "
                                 "schedule", "traffic": None}
    work_full = abi.lib.rsgpu_revolve_numforw(f["nt"], RTM3["ncheck"]) + 1 + 2 * f["nt"]
    work = stats["fw_steps"] + stats["bw_steps"] + 1
    return {"images_per_s": float("%.4g" % (ns / t_batch)), "s_per_batch": round(t_batch, 3), "shots": ns,
            "images_per_s_at_full_nt_extrapolated": float("%.4g" % (ns / t_batch * work / work_full)),
            "forward_steps": stats["fw_steps"], "adjoint_steps": stats["bw_steps"],
            "checkpoint_bytes": stats["ckpt_bytes"], "gpu_launches": stats["launches"],
            "gpts_per_s_propagation": round(pts * (stats["fw_steps"] + stats["bw_steps"]) / t_batch / 1e9, 3),
            "roofline": roof, "clocks": clk.summary(), "models": models}


# ---------------------------------------------------------------- distributed plumbing
def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def dist_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fast", choices=["fast", "exact"])
    ap.add_argument("--tile", type=int, default=-2,
                    help="2D tile shape index; -2 = autotuned (cached in JSON), -1 = library default")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=None,
                    help="elastic2d: time steps of the reference CPU sample (default 100 for the reference arm, "
                         "400 for our line's cpu_baseline; 4000 = the whole modelling)")
    ap.add_argument("--nt", type=int, default=NT, help="time steps per modelling (profiling runs shorten it)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end C ABI measurement")
    ap.add_argument("--workload", default="elastic2d",
                    choices=["elastic2d", "acoustic2d", "fwi", "acoustic3d", "acoustic3d_rtm", "elastic3d",
                             "elastic3d_fwi"],
                    help="elastic2d: the forward modelling line (with the FWI gradient figures attached); "
                         "acoustic2d: the one-shot acoustic forward; fwi: the FWI gradient line alone")
    ap.add_argument("--launch-mode", type=int, default=0,
                    help="2D: rsgpu_config.launch_mode (0 = library choice: per-tile kernels, 3 = fused step, "
                         "4 = column-marching elastic half-steps)")
    ap.add_argument("--no-fwi", action="store_true", help="leave the FWI gradient figures out of the elastic2d line")
    ap.add_argument("--fwi-steps", type=int, default=2, help="timed gradient batches")
    ap.add_argument("--zchunk", type=int, default=0,
                    help="3D: planes per z-march; 2D fused step: rows per work item (0 = library default)")
    ap.add_argument("--shots", type=int, default=None,
                    help="acoustic3d / elastic3d_fwi: only the first N shots (profiling runs)")
    ap.add_argument("--rtm-nt", type=int, default=RTM3["nt_bench"],
                    help="acoustic3d_rtm: time steps of the timed images (the full workload has 2500)")
    ap.add_argument("--e3d-nt", type=int, default=E3D["nt_bench"],
                    help="elastic3d_fwi: time steps of the timed gradients (the full workload has 2000)")
    args = ap.parse_args()

    if args.impl == "reference" and args.workload == "fwi":
        if int(os.environ.get("RANK", "0")) == 0:
            r = cpu_fwi_reference()
            if r is None:
                print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref not built"}))
                return
            print(json.dumps({"metric": "FWI gradient shots/s", "value": r["value"], "unit": "shots/s",
                              "impl": "reference", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": 1,
                              "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                              "dtype": "f32", "data": "synthetic", "config": fwi_config(), "cpu_baseline": r,
                              "e2e": {"value": r["value"], "unit": "shots/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))
        return

    if args.impl == "reference" and args.workload == "elastic3d_fwi":
        if int(os.environ.get("RANK", "0")) == 0:
            r = cpu_e3d_reference(E3D["ncheck"], args.e3d_nt)
            if r is None:
                print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref not built"}))
                return
            print(json.dumps({"metric": "FWI gradient shots/s", "value": r["value"], "unit": "shots/s",
                              "impl": "reference", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": 1,
                              "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                              "dtype": "f32", "data": "synthetic",
                              "config": e3d_config(args.e3d_nt, E3D["ncheck"]), "cpu_baseline": r,
                              "e2e": {"value": r["value"], "unit": "shots/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))
        return

    if args.impl == "reference" and args.workload == "acoustic3d_rtm":
        if int(os.environ.get("RANK", "0")) == 0:
            from rockseis_b200 import abi
            models, _, _ = a3d_batch(abi.F32_EXACT, f=dict(A3D, nt=args.rtm_nt), nshots=args.shots)
            r = cpu_rtm3d_reference(models, args.rtm_nt, RTM3["ncheck"])
            if r is None:
                print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref not built"}))
                return
            print(json.dumps({"metric": "RTM images/s", "value": r["value"], "unit": "images/s",
                              "impl": "reference", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": 1,
                              "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                              "dtype": "f32", "data": "synthetic", "config": rtm3d_config(args.rtm_nt, args.shots),
                              "cpu_baseline": r, "e2e": {"value": r["value"], "unit": "images/s",
                                                         "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    if args.impl == "reference" and args.workload == "acoustic3d":
        if int(os.environ.get("RANK", "0")) == 0:
            from rockseis_b200 import abi
            models, _, _ = a3d_batch(abi.F32_EXACT)
            r = cpu_a3d_reference(models)
            if r is None:
                print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref not built"}))
                return
            print(json.dumps({"metric": "Gpts/s", "value": r["value"], "unit": "Gpts/s", "impl": "reference",
                              "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": 1, "warmup": 0,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                              "data": "synthetic", "config": a3d_config(), "cpu_baseline": r,
                              "e2e": {"value": r["value"], "unit": "Gpts/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))
        return

    if args.impl == "reference":
        # CPU only: rank 0 times the reference, the other ranks exit without work.
        rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
        if rank == 0:
            per = []
            for _ in range(args.steps):
                r = cpu_reference(args.cpu_steps or CPU_SAMPLE_STEPS)
                if r is None:
                    print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref not built"}))
                    return
                per.append(r["value"])
            val = statistics.median(per)
            line = {"metric": "Gpts/s", "value": round(val, 5), "unit": "Gpts/s", "impl": "reference",
                    "n_gpus": world, "steps": args.steps, "warmup": 0, "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                    "config": config_dict(world, "reference float (stock build, no FMA)"),
                    "cpu_baseline": r, "e2e": {"value": round(val, 5), "unit": "Gpts/s", "h2d_bytes_per_step": 0,
                                               "d2h_bytes_per_step": 0}}
            print(json.dumps(line))
        return

    rank, world, local = dist_init(args)
    if args.workload == "acoustic3d":
        import torch
        torch.cuda.set_device(local)
        r = run_a3d(args, device=local)
        models = r.pop("models")
        cpu = None if args.no_cpu_baseline else cpu_a3d_reference(models)
        line = {"metric": "Gpts/s", "value": r["value"], "unit": "Gpts/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded dipping layers, windowed shots)",
                "config": a3d_config(args.shots), "gpu_launches": r["gpu_launches"], "roofline": r["roofline"],
                "clocks": r["clocks"], "acoustic3d": {k: v for k, v in r.items() if k not in ("roofline", "clocks")},
                "cpu_baseline": cpu}
        print(json.dumps(line))
        return
    if args.workload == "acoustic3d_rtm":
        if world > 1:
            raise SystemExit("the 3D RTM line is a one-GPU measurement")
        import torch
        torch.cuda.set_device(local)
        r = run_rtm3d(args, device=local)
        models = r.pop("models")
        cpu = None if args.no_cpu_baseline else cpu_rtm3d_reference(models, args.rtm_nt, RTM3["ncheck"])
        line = {"metric": "RTM images/s", "value": r["images_per_s"], "unit": "images/s", "n_gpus": 1,
                "steps": args.fwi_steps, "warmup": 1, "ms_per_step": round(r["s_per_batch"] * 1e3, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded dipping layers, windowed shots; data modelled in the same model)",
                "config": rtm3d_config(args.rtm_nt, args.shots), "gpu_launches": r["gpu_launches"],
                "roofline": r["roofline"], "clocks": r["clocks"],
                "rtm_image": {k: v for k, v in r.items() if k not in ("roofline", "clocks")}, "cpu_baseline": cpu}
        print(json.dumps(line))
        return
    if args.workload == "elastic3d":
        import torch
        torch.cuda.set_device(local)
        r = run_e3d_forward(args, device=local)
        line = {"metric": "Gpts/s", "value": r["value"], "unit": "Gpts/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded layers + Gaussian blobs)",
                "config": r["config"], "gpu_launches": r["gpu_launches"], "roofline": r["roofline"],
                "clocks": r["clocks"], "cpu_baseline": None}
        print(json.dumps(line))
        return
    if args.workload == "elastic3d_fwi":
        if world > 1:
            raise SystemExit("the elastic 3D FWI gradient line is a one-GPU measurement")
        import torch
        torch.cuda.set_device(local)
        r = run_e3d(args, device=local)
        cpu = None if args.no_cpu_baseline else cpu_e3d_reference(r["ncheck"], args.e3d_nt)
        line = {"metric": "FWI gradient shots/s", "value": r["shots_per_s_batched"], "unit": "shots/s", "n_gpus": 1,
                "steps": args.fwi_steps, "warmup": 1, "ms_per_step": round(r["s_per_batch"] * 1e3, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded layers + Gaussian blobs; start model = the layers)",
                "config": r["config"], "gpu_launches": r["gpu_launches"], "roofline": r["roofline"],
                "fwi_gradient": {k: v for k, v in r.items() if k not in ("roofline", "config", "e2e", "clocks")},
                "e2e": r["e2e"], "clocks": r["clocks"], "cpu_baseline": cpu}
        print(json.dumps(line))
        return
    if args.workload == "fwi":
        if world > 1:
            raise SystemExit("the FWI gradient line is a one-GPU measurement")
        cpu = None if args.no_cpu_baseline else cpu_fwi_reference()
        import torch
        torch.cuda.set_device(local)
        r = run_fwi(args, device=local)
        line = {"metric": "FWI gradient shots/s", "value": r["shots_per_s_batched"], "unit": "shots/s", "n_gpus": 1,
                "steps": args.fwi_steps, "warmup": 1, "ms_per_step": round(r["s_per_batch"] * 1e3, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded smooth background + Gaussian anomalies; start model smoothed)",
                "config": r["config"], "gpu_launches": r["gpu_launches"], "roofline": r["roofline"],
                "fwi_gradient": r, "e2e": r.get("e2e"), "clocks": r["clocks"], "cpu_baseline": cpu}
        print(json.dumps(line))
        return
    if args.workload == "acoustic2d":
        cpu = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            cpu = cpu_c1_reference()
        r = run_gpu(args, rank, world, local, physics="acoustic2d")
        if rank == 0:
            print(json.dumps({"metric": "Gpts/s", "value": round(r["value"], 3), "unit": "Gpts/s", "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(r["ms_step"], 3),
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                              "data": "synthetic (seeded layered model, 5 % smooth perturbation, Ricker source)",
                              "config": c1_config(world, args.precision), "gpu_launches": int(r["launches"]),
                              "roofline": r["roofline"], "e2e": r["e2e"], "clocks": r["clocks"],
                              "parity": r["parity"], "cpu_baseline": cpu}))
        return
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference(args.cpu_steps or CPU_BASELINE_STEPS)   # before the first CUDA call (spawned workers)
    r = run_gpu(args, rank, world, local)
    fwi = None
    if rank == 0 and world == 1 and not args.no_fwi:
        try:
            fwi = run_fwi(args)
            if not args.no_cpu_baseline:
                fwi["cpu_baseline"] = cpu_fwi_reference()
        except Exception as exc:          # keep the forward line if the gradient part fails
            fwi = {"error": f"{type(exc).__name__}: {exc}"}
    if rank == 0:
        line = {"metric": "Gpts/s", "value": round(r["value"], 3), "unit": "Gpts/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(r["ms_step"], 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded layered elastic model with lenses, Ricker source)",
                "config": config_dict(world, args.precision, args.nt),
                "gpu_launches": int(r["launches"]),
                "roofline": r["roofline"], "e2e": r["e2e"], "clocks": r["clocks"],
                "parity": r["parity"], "cpu_baseline": cpu}
        if fwi is not None:
            line["fwi_gradient"] = fwi
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""ctypes wrappers of the two CPU checkers (test infrastructure only).

  ORACLE : oracle/librsoracle.so, this repository's C restatement (rs_oracle.c)
  REF    : oracle/_ref/librsref.so, the unmodified reference library plus the
           in-process harness (ref_harness*.cpp); present only where it was built.

Only the test-suite, __graft_entry__.smoke() and bench.py's CPU-baseline arm
import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "librsoracle.so")
REF_SO = os.path.join(HERE, "_ref", "librsref.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "librsref_gpu.so")
INTEGRATION = os.path.join(os.path.dirname(HERE), "integration")
# Root of the reference source tree, from the environment (the build recipe sets it);
# without it only the C restatement is built.
REFSRC_ENV = "RSGPU_REFERENCE_SRC"


def build(ref: bool = True) -> None:
    """Build the checkers (the reference part only where its sources exist)."""
    refsrc = os.environ.get(REFSRC_ENV, "")
    use_ref = ref and bool(refsrc) and os.path.isdir(refsrc)
    targets = ["oracle"] + (["ref", f"REFSRC={refsrc}"] if use_ref else [])
    subprocess.run(["make", "-s", "-C", HERE, f"-j{os.cpu_count() or 4}"] + targets, check=True)
    gpu_lib = os.path.join(os.path.dirname(HERE), "rockseis_b200", "librsgpu.so")
    if use_ref and os.path.exists(gpu_lib):
        subprocess.run(["make", "-s", "-C", INTEGRATION, f"-j{os.cpu_count() or 4}", f"REFSRC={refsrc}"], check=True)


class OrcGrid(C.Structure):
    _fields_ = [("nxp", C.c_int), ("nzp", C.c_int), ("lpml", C.c_int), ("order", C.c_int), ("fs", C.c_int),
                ("dx", C.c_float), ("dz", C.c_float), ("dt", C.c_float), ("nt", C.c_int)]


class OrcGrid3(C.Structure):
    _fields_ = [("nxp", C.c_int), ("nyp", C.c_int), ("nzp", C.c_int), ("lpml", C.c_int), ("order", C.c_int),
                ("fs", C.c_int), ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float), ("dt", C.c_float),
                ("nt", C.c_int)]


class RefGrid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("lpml", C.c_int), ("order", C.c_int),
                ("fs", C.c_int), ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("ox", C.c_double),
                ("oy", C.c_double), ("oz", C.c_double), ("dt", C.c_double), ("nt", C.c_int)]


def _p(a):
    return None if a is None else a.ctypes.data


_oracle = None
_ref = None


def oracle() -> C.CDLL:
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        _oracle = C.CDLL(ORACLE_SO)
        V, I = C.c_void_p, C.c_int
        _oracle.orc_mod_a2d.argtypes = [C.POINTER(OrcGrid)] + [V] * 4 + [I, V, V, V, I, I, V, V, I, V, I, V]
        _oracle.orc_mod_e2d.argtypes = [C.POINTER(OrcGrid)] + [V] * 6 + [I, V, V, V, I, I, V, V, I, V, V, I, V]
        _oracle.orc_e2d_adjoint_steps.argtypes = [C.POINTER(OrcGrid)] + [V] * 6 + [I, V]
        _oracle.orc_fwi_a2d.argtypes = [C.POINTER(OrcGrid), I, I] + [V] * 6 + [I, V, V, V, I, V, V, V, I, V, V,
                                                                                  V, V, V, V]
        _oracle.orc_rtm_a2d.argtypes = [C.POINTER(OrcGrid), I, I] + [V] * 4 + [I, V, V, V, I, V, V, V, I, I, V]
        _oracle.orc_der2d.argtypes = [I, I, I, C.c_float, C.c_float, I, V, V]
        _oracle.orc_fwi_e2d.argtypes = [C.POINTER(OrcGrid), I, I] + [V] * 3 + [V] * 6 + [I, V, V, V, I, I, V, V, V, I] + \
            [V] * 4 + [V, V, V]
        _oracle.orc_fwi_a3d.argtypes = [C.POINTER(OrcGrid3), I, I, I] + [V] * 7 + [I, V, V, V, I, V, V, V, I] + \
            [V] * 5 + [V]
        _oracle.orc_interp.argtypes = [I, I, I, C.c_float, C.c_float, V, I, C.c_float, C.c_float, V]
        _oracle.orc_rtm_a3d.argtypes = [C.POINTER(OrcGrid3), I, I, I] + [V] * 5 + [I, V, V, V, I, V, V, V, I, I, I, V]
        _oracle.orc_mod_a3d.argtypes = [C.POINTER(OrcGrid3)] + [V] * 5 + [I, V, V, V, I, I, V, V, I, V, I, V]
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _load_ref(path: str) -> C.CDLL:
    """The harness library at path with its argument types declared."""
    lib = C.CDLL(path)
    V, I, D = C.c_void_p, C.c_int, C.c_double
    G = C.POINTER(RefGrid)
    for t in ("f", "d"):
        getattr(lib, f"ref_der_{t}").argtypes = [I, I, I, D, D, D, I, I, V, V]
        getattr(lib, f"ref_pml_tables_{t}").argtypes = [I, D, V]
        getattr(lib, f"ref_mod_a2d_{t}").argtypes = [G, V, V, I, V, V, I, I, V, I, V]
        getattr(lib, f"ref_mod_e2d_{t}").argtypes = [G, V, V, V, I, V, V, I, I, V, I, V]
        getattr(lib, f"ref_fwi_a2d_{t}").argtypes = [G, V, V, I, V, V, I, V, V, I, I, V, V, V, V, V, V]
    lib.ref_mod_a3d_f.argtypes = [G, V, V, I, V, V, I, I, V, I, V]
    lib.ref_mod_e3d_f.argtypes = [G, V, V, V, I, V, V, I, I, V, I, V]
    lib.ref_fwi_e2d_f.argtypes = [G, V, V, V, I, V, V, I, I, V, V, V, V, I] + [V] * 6 + [V]
    lib.ref_fwi_e2d_corr_f.argtypes = [G, V, V, V, I, V, V, I, I, V, V, V, V, I] + [V] * 6 + [V]
    lib.ref_fwi_e2d_misfit_f.argtypes = [G, V, V, V, I, V, V, I, I, V, V, V, V, I] + [V] * 6 + [V, I]
    if hasattr(lib, "ref_fwi_e2d_full_f"):
        lib.ref_fwi_e2d_full_f.argtypes = [G, V, V, V, I, V, V, I, I, V, V, V, V, I] + [V] * 6 + [V]
    lib.ref_fwi_a2d_ilum_f.argtypes = [G, V, V, I, V, V, I, V, V, I, I] + [V] * 5 + [V, V]
    lib.ref_fwi_a2d_full_f.argtypes = [G, V, V, I, V, V, I, V, V, I, I, I] + [V] * 5 + [V]
    lib.ref_rtm_a2d_full_f.argtypes = [G, V, V, I, V, V, I, V, V, I, I, I, V]
    lib.ref_rtm_a2d_edge_f.argtypes = [G, V, V, I, V, V, I, V, V, I, I, I, V]
    lib.ref_localsize2d_f.argtypes = [G, I, V, V, D, I, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    lib.ref_localsize3d_f.argtypes = [G, I, V, V, D, D, I, V]
    lib.ref_fwi_e3d_f.argtypes = [G, V, V, V, I, V, V, I, I, V, V, V, V, I] + [V] * 6 + [V]
    lib.ref_fwi_a3d_f.argtypes = [G, V, V, I, V, V, I, V, V, I] + [V] * 5 + [V]
    lib.ref_fwi_a3d_corr_f.argtypes = [G, V, V, I, V, V, I, V, V, I] + [V] * 5 + [V]
    lib.ref_fwi_a3d_misfit_f.argtypes = [G, V, V, I, V, V, I, V, V, I] + [V] * 5 + [V, I]
    lib.ref_interp_f.argtypes = [I, I, I, C.c_float, C.c_float, V, I, C.c_float, C.c_float, V]
    lib.ref_rtm_a3d_f.argtypes = [G, V, V, I, V, V, I, V, V, I, I, I, I, V]
    lib.ref_rtm_a3d_full_f.argtypes = [G, V, V, I, V, V, I, V, V, I, I, I, I, V]
    lib.ref_rtm_a2d_f.argtypes = [G, V, V, I, V, V, I, V, V, I, I, I, V]
    lib.ref_stagger_a2d_f.argtypes = [G, V, V, V, V, V]
    lib.ref_stagger_e2d_f.argtypes = [G, V, V, V, V, V, V, V, V]
    lib.ref_stagger_a3d_f.argtypes = [G, V, V, V, V, V, V]
    lib.ref_stagger_e3d_f.argtypes = [G, V, V, V] + [V] * 8
    lib.ref_makemap2d_f.argtypes = [G, I, V, I, V, V]
    lib.ref_makemap2d_field_f.argtypes = [G, I, V, I, I, V, V]
    lib.ref_makemap3d_f.argtypes = [G, I, V, I, V, V]
    lib.ref_makemap3d_field_f.argtypes = [G, I, V, I, I, V, V]
    lib.ref_revolve_trace.argtypes = [I, I, V, V, V, I]
    if hasattr(lib, "ref_data_write_f"):          # file / sort harness (oracle/ref_harness_io.cpp)
        S, LL = C.c_char_p, C.POINTER(C.c_longlong)
        lib.ref_data_write_f.argtypes = [S, I, I, D, D, I, V, V, V]
        lib.ref_data_write_d.argtypes = [S, I, I, D, D, I, V, V, V]
        lib.ref_data_read2d_f.argtypes = [S, I, I, V, V, V]
        lib.ref_model_write_f.argtypes = [S, I, I, D, D, D, D, V]
        lib.ref_sort_gather_f.argtypes = [S, I, I, D, D, I, I, I, LL, V, V, V, I]
        lib.ref_sort_gather_d.argtypes = [S, I, I, D, D, I, I, I, LL, V, V, V, I]
        lib.ref_sort_put2d_f.argtypes = [S, S, I, I, D, D, V]
    lib.ref_revolve_numforw.argtypes = [I, I]
    lib.ref_revolve_adjust.argtypes = [I]
    lib.ref_steps_e2d_f.argtypes = [G, V, V, V, I, V, V, I, I, I, V]
    lib.ref_steps_a2d_f.argtypes = [G, V, V, I, V, V, I, I, V]
    lib.ref_steps_e3d_f.argtypes = [G, V, V, V, I, V, V, I, I, I, V]
    return lib


def ref() -> C.CDLL:
    """The unmodified reference library and its harness."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError("reference oracle not built (oracle/_ref/librsref.so)")
        _ref = _load_ref(REF_SO)
    return _ref


_ref_gpu = None


def ref_gpu_available() -> bool:
    return os.path.exists(REF_GPU_SO)


def ref_gpu() -> C.CDLL:
    """The reference library built with the GPU binding (integration/rockseis_gpu.cpp):
    its ModellingAcoustic2D/ModellingElastic2D<float>::run and
    FwiAcoustic2D<float>::run_optimal call librsgpu; same harness entry points."""
    global _ref_gpu
    if _ref_gpu is None:
        if not os.path.exists(REF_GPU_SO):
            raise FileNotFoundError("reference build with the GPU binding missing (oracle/_ref/librsref_gpu.so)")
        _ref_gpu = _load_ref(REF_GPU_SO)
    return _ref_gpu


# ---------------------------------------------------------------- problem description
class Problem2D:
    """One 2D shot in the form both checkers and the GPU library consume."""

    def __init__(self, nx, nz, dx, dz, lpml, order, fs, dt, nt, vp, rho, vs=None, ox=0.0, oz=0.0):
        self.nx, self.nz, self.dx, self.dz, self.lpml, self.order, self.fs = nx, nz, dx, dz, lpml, order, fs
        self.dt, self.nt, self.ox, self.oz = dt, nt, ox, oz
        self.vp, self.rho, self.vs = vp, rho, vs
        self.src = self.rec = None

    def ref_grid(self) -> RefGrid:
        return RefGrid(self.nx, 1, self.nz, self.lpml, self.order, int(self.fs), self.dx, 1.0, self.dz, self.ox,
                       0.0, self.oz, self.dt, self.nt)

    def orc_grid(self) -> OrcGrid:
        return OrcGrid(self.nx + 2 * self.lpml, self.nz + 2 * self.lpml, self.lpml, min(max(self.order, 1), 8),
                       int(self.fs), self.dx, self.dz, self.dt, self.nt)


def ref_modelling_a2d(pb, scoords, wav, sfield, gcoords, rfield, dtype=np.float32, lib=None):
    t = "f" if dtype == np.float32 else "d"
    out = np.zeros((len(gcoords), pb.nt), dtype)
    g = pb.ref_grid()
    sc, gc = np.ascontiguousarray(scoords, np.float64), np.ascontiguousarray(gcoords, np.float64)
    vp, rho, w = (np.ascontiguousarray(a, dtype) for a in (pb.vp, pb.rho, wav))
    r = getattr(lib or ref(), f"ref_mod_a2d_{t}")(C.byref(g), _p(vp), _p(rho), len(sc), _p(sc), _p(w), sfield, len(gc),
                                           _p(gc), rfield, _p(out))
    assert r == 1
    return out


def ref_modelling_e2d(pb, scoords, wav, sfield, gcoords, rfield, dtype=np.float32, lib=None):
    t = "f" if dtype == np.float32 else "d"
    out = np.zeros((len(gcoords), pb.nt), dtype)
    g = pb.ref_grid()
    sc, gc = np.ascontiguousarray(scoords, np.float64), np.ascontiguousarray(gcoords, np.float64)
    vp, vs, rho = (np.ascontiguousarray(a, dtype) for a in (pb.vp, pb.vs, pb.rho))
    w = np.ascontiguousarray(wav, dtype)
    r = getattr(lib or ref(), f"ref_mod_e2d_{t}")(C.byref(g), _p(vp), _p(vs), _p(rho), len(sc), _p(sc), _p(w), sfield,
                                           len(gc), _p(gc), rfield, _p(out))
    assert r == 1
    return out


def _keep(*arrs, dtype=None):
    """Contiguous copies bound to the caller so the buffers outlive the C call."""
    return [None if a is None else np.ascontiguousarray(a, dtype if dtype is not None else a.dtype) for a in arrs]


def ref_fwi_a2d(pb, scoords, wav, gcoords, obs, ncheck, dtype=np.float32, misfit=0, srcilum=False, lib=None):
    """FwiAcoustic2D::run_optimal; with srcilum (float only) also the source illumination image."""
    t = "f" if dtype == np.float32 else "d"
    g = pb.ref_grid()
    sc, gc = np.ascontiguousarray(scoords, np.float64), np.ascontiguousarray(gcoords, np.float64)
    ns, nr = len(sc), len(gc)
    vpg = np.zeros((pb.nz, pb.nx), dtype)
    rhog = np.zeros((pb.nz, pb.nx), dtype)
    wg = np.zeros((ns, pb.nt), dtype)
    dm = np.zeros((nr, pb.nt), dtype)
    dr = np.zeros((nr, pb.nt), dtype)
    mis = C.c_double()
    vp, rho, w, ob = _keep(pb.vp, pb.rho, wav, obs, dtype=dtype)
    if srcilum:
        il = np.zeros((pb.nz, pb.nx), np.float32)
        r = (lib or ref()).ref_fwi_a2d_ilum_f(C.byref(g), _p(vp), _p(rho), ns, _p(sc), _p(w), nr, _p(gc), _p(ob), ncheck,
                                     misfit, _p(vpg), _p(rhog), _p(wg), _p(dm), _p(dr), C.byref(mis), _p(il))
        assert r == 1
        return dict(vpgrad=vpg, rhograd=rhog, wavgrad=wg, datamod=dm, datares=dr, misfit=mis.value, srcilum=il)
    r = getattr(lib or ref(), f"ref_fwi_a2d_{t}")(C.byref(g), _p(vp), _p(rho), ns, _p(sc), _p(w), nr, _p(gc), _p(ob),
                                           ncheck, misfit, _p(vpg), _p(rhog), _p(wg), _p(dm), _p(dr), C.byref(mis))
    assert r == 1
    return dict(vpgrad=vpg, rhograd=rhog, wavgrad=wg, datamod=dm, datares=dr, misfit=mis.value)


def ref_fwi_a2d_full(pb, scoords, wav, gcoords, obs, snapinc, noreverse=0, misfit=0, lib=None):
    """FwiAcoustic2D::run, the full-snapshot gradient (snapshots every snapinc steps)."""
    g = pb.ref_grid()
    sc, gc = np.ascontiguousarray(scoords, np.float64), np.ascontiguousarray(gcoords, np.float64)
    ns, nr = len(sc), len(gc)
    out = dict(vpgrad=np.zeros((pb.nz, pb.nx), np.float32), rhograd=np.zeros((pb.nz, pb.nx), np.float32),
               wavgrad=np.zeros((ns, pb.nt), np.float32), datamod=np.zeros((nr, pb.nt), np.float32),
               datares=np.zeros((nr, pb.nt), np.float32))
    mis = C.c_double()
    vp, rho, w, ob = _keep(pb.vp, pb.rho, wav, obs, dtype=np.float32)
    r = (lib or ref()).ref_fwi_a2d_full_f(C.byref(g), _p(vp), _p(rho), ns, _p(sc), _p(w), nr, _p(gc), _p(ob),
                                          snapinc, noreverse, misfit, _p(out["vpgrad"]), _p(out["rhograd"]),
                                          _p(out["wavgrad"]), _p(out["datamod"]), _p(out["datares"]), C.byref(mis))
    assert r == 1
    out["misfit"] = mis.value
    return out


def ref_rtm_a2d_full(pb, scoords, wav, gcoords, data, snapinc, nhx=1, nhz=1, edges=False):
    """RtmAcoustic2D::run, the full-snapshot image (edges: RtmAcoustic2D::run_edge)."""
    g = pb.ref_grid()
    sc, gc = np.ascontiguousarray(scoords, np.float64), np.ascontiguousarray(gcoords, np.float64)
    img = np.zeros((nhz, nhx, pb.nz, pb.nx), np.float32)
    vp, rho, w, d = _keep(pb.vp, pb.rho, wav, data, dtype=np.float32)
    fn = ref().ref_rtm_a2d_edge_f if edges else ref().ref_rtm_a2d_full_f
    r = fn(C.byref(g), _p(vp), _p(rho), len(sc), _p(sc), _p(w), len(gc), _p(gc), _p(d), snapinc, nhx, nhz, _p(img))
    assert r == 1
    return img


def ref_rtm_a2d(pb, scoords, wav, gcoords, data, ncheck, nhx=1, nhz=1):
    g = pb.ref_grid()
    sc, gc = np.ascontiguousarray(scoords, np.float64), np.ascontiguousarray(gcoords, np.float64)
    img = np.zeros((nhz, nhx, pb.nz, pb.nx), np.float32)
    vp, rho, w, d = _keep(pb.vp, pb.rho, wav, data, dtype=np.float32)
    r = ref().ref_rtm_a2d_f(C.byref(g), _p(vp), _p(rho), len(sc), _p(sc), _p(w), len(gc), _p(gc), _p(d), ncheck,
                            nhx, nhz, _p(img))
    assert r == 1
    return img


def ref_revolve_trace(nt, ncheck, maxn=200000):
    a = np.zeros(maxn, np.int32)
    c = np.zeros(maxn, np.int32)
    k = np.zeros(maxn, np.int32)
    n = ref().ref_revolve_trace(nt, ncheck, _p(a), _p(c), _p(k), maxn)
    assert n > 0
    return a[:n], c[:n], k[:n]


# ---------------------------------------------------------------- restated oracle drivers
def orc_modelling_a2d(pb, padded, tab, smap, sshift, wav, sfield, gmap, gshift, rfield, nsteps=None,
                      want_state=False):
    g = pb.orc_grid()
    nr = len(gmap)
    out = np.zeros((nr, pb.nt), np.float32)
    nxp, nzp = pb.nx + 2 * pb.lpml, pb.nz + 2 * pb.lpml
    st = np.zeros((3, nzp, nxp), np.float32) if want_state else None
    Rx, Rz, L, tb, ss, w, gs = _keep(*padded, tab, sshift, wav, gshift, dtype=np.float32)
    sm, gm = _keep(smap, gmap, dtype=np.int32)
    oracle().orc_mod_a2d(C.byref(g), _p(Rx), _p(Rz), _p(L), _p(tb), len(sm), _p(sm), _p(ss), _p(w), sfield, nr,
                         _p(gm), _p(gs), rfield, _p(out), pb.nt if nsteps is None else nsteps, _p(st))
    return (out, st) if want_state else out


def orc_modelling_e2d(pb, padded, tab, smap, sshift, wav, sfield, gmap, gshift, rfield, factor=None, nsteps=None,
                      want_state=False):
    g = pb.orc_grid()
    nr = len(gmap)
    out = np.zeros((nr, pb.nt), np.float32)
    nxp, nzp = pb.nx + 2 * pb.lpml, pb.nz + 2 * pb.lpml
    st = np.zeros((5, nzp, nxp), np.float32) if want_state else None
    Rx, Rz, L, L2M, M, tb, ss, w, gs, fac = _keep(*padded, tab, sshift, wav, gshift, factor, dtype=np.float32)
    sm, gm = _keep(smap, gmap, dtype=np.int32)
    oracle().orc_mod_e2d(C.byref(g), _p(Rx), _p(Rz), _p(L), _p(L2M), _p(M), _p(tb), len(sm), _p(sm), _p(ss), _p(w),
                         sfield, nr, _p(gm), _p(gs), rfield, _p(fac), _p(out), pb.nt if nsteps is None else nsteps,
                         _p(st))
    return (out, st) if want_state else out


def orc_fwi_a2d(pb, padded, tab, smap, sshift, wav, gmap, gshift, obs, misfit=0):
    g = pb.orc_grid()
    ns, nr = len(smap), len(gmap)
    vpg = np.zeros((pb.nz, pb.nx), np.float32)
    rhog = np.zeros((pb.nz, pb.nx), np.float32)
    wg = np.zeros((ns, pb.nt), np.float32)
    dm = np.zeros((nr, pb.nt), np.float32)
    dr = np.zeros((nr, pb.nt), np.float32)
    mis = C.c_double()
    Rx, Rz, L, tb, ss, w, gs, ob, vp, rho = _keep(*padded, tab, sshift, wav, gshift, obs, pb.vp, pb.rho,
                                                  dtype=np.float32)
    sm, gm = _keep(smap, gmap, dtype=np.int32)
    r = oracle().orc_fwi_a2d(C.byref(g), pb.nx, pb.nz, _p(vp), _p(rho), _p(Rx), _p(Rz), _p(L), _p(tb), ns, _p(sm),
                             _p(ss), _p(w), nr, _p(gm), _p(gs), _p(ob), misfit, _p(vpg), _p(rhog), _p(wg), _p(dm),
                             _p(dr),
                             C.byref(mis))
    assert r == 0
    return dict(vpgrad=vpg, rhograd=rhog, wavgrad=wg, datamod=dm, datares=dr, misfit=mis.value)


def orc_rtm_a2d(pb, padded, tab, smap, sshift, wav, gmap, gshift, data, nhx=1, nhz=1):
    g = pb.orc_grid()
    img = np.zeros((nhz, nhx, pb.nz, pb.nx), np.float32)
    Rx, Rz, L, tb, ss, w, gs, d = _keep(*padded, tab, sshift, wav, gshift, data, dtype=np.float32)
    sm, gm = _keep(smap, gmap, dtype=np.int32)
    r = oracle().orc_rtm_a2d(C.byref(g), pb.nx, pb.nz, _p(Rx), _p(Rz), _p(L), _p(tb), len(sm), _p(sm), _p(ss), _p(w),
                             len(gm), _p(gm), _p(gs), _p(d), nhx, nhz, _p(img))
    assert r == 0
    return img


# ---------------------------------------------------------------- 3D
class Problem3D:
    """One 3D shot: unpadded models [nz][ny][nx] and the grid."""

    def __init__(self, nx, ny, nz, dx, dy, dz, lpml, order, fs, dt, nt, vp, rho, vs=None, ox=0.0, oy=0.0, oz=0.0):
        self.nx, self.ny, self.nz, self.dx, self.dy, self.dz = nx, ny, nz, dx, dy, dz
        self.lpml, self.order, self.fs, self.dt, self.nt = lpml, order, fs, dt, nt
        self.vp, self.rho, self.vs, self.ox, self.oy, self.oz = vp, rho, vs, ox, oy, oz

    def ref_grid(self) -> RefGrid:
        return RefGrid(self.nx, self.ny, self.nz, self.lpml, self.order, int(self.fs), self.dx, self.dy, self.dz,
                       self.ox, self.oy, self.oz, self.dt, self.nt)

    def orc_grid(self) -> OrcGrid3:
        L = self.lpml
        return OrcGrid3(self.nx + 2 * L, self.ny + 2 * L, self.nz + 2 * L, L, min(max(self.order, 1), 8),
                        int(self.fs), self.dx, self.dy, self.dz, self.dt, self.nt)


def ref_modelling_a3d(pb, scoords, wav, sfield, gcoords, rfield):
    out = np.zeros((len(gcoords), pb.nt), np.float32)
    g = pb.ref_grid()
    sc, gc = np.ascontiguousarray(scoords, np.float64), np.ascontiguousarray(gcoords, np.float64)
    vp, rho, w = _keep(pb.vp, pb.rho, wav, dtype=np.float32)
    r = ref().ref_mod_a3d_f(C.byref(g), _p(vp), _p(rho), len(sc), _p(sc), _p(w), sfield, len(gc), _p(gc), rfield,
                            _p(out))
    assert r == 1
    return out


def ref_stagger_a3d(pb):
    g = pb.ref_grid()
    L = pb.lpml
    n = (pb.nx + 2 * L) * (pb.ny + 2 * L) * (pb.nz + 2 * L)
    out = np.zeros((4, n), np.float32)
    vp, rho = _keep(pb.vp, pb.rho, dtype=np.float32)
    ref().ref_stagger_a3d_f(C.byref(g), _p(vp), _p(rho), *[out[k].ctypes.data for k in range(4)])
    return out.reshape(4, pb.nz + 2 * L, pb.ny + 2 * L, pb.nx + 2 * L)


def ref_makemap3d(pb, coords, which, field=0):
    g = pb.ref_grid()
    c = np.ascontiguousarray(coords, np.float64)
    mp = np.zeros((len(c), 3), np.int32)
    sh = np.zeros((len(c), 3), np.float32)
    ref().ref_makemap3d_field_f(C.byref(g), len(c), _p(c), which, field, _p(mp), _p(sh))
    return mp, sh


def orc_modelling_a3d(pb, padded, tab, smap, sshift, wav, sfield, gmap, gshift, rfield, nsteps=None, want_state=False):
    g = pb.orc_grid()
    nr = len(gmap)
    out = np.zeros((nr, pb.nt), np.float32)
    st = np.zeros((4, g.nzp, g.nyp, g.nxp), np.float32) if want_state else None
    Rx, Ry, Rz, L, tb, ss, w, gs = _keep(*padded, tab, sshift, wav, gshift, dtype=np.float32)
    sm, gm = _keep(smap, gmap, dtype=np.int32)
    oracle().orc_mod_a3d(C.byref(g), _p(Rx), _p(Ry), _p(Rz), _p(L), _p(tb), len(sm), _p(sm), _p(ss), _p(w), sfield,
                         nr, _p(gm), _p(gs), rfield, _p(out), pb.nt if nsteps is None else nsteps, _p(st))
    return (out, st) if want_state else out


# ---------------------------------------------------------------- elastic FWI
def ref_fwi_e2d(pb, scoords, wav, sfield, gcoords, obs3, ncheck, misfit=0, full_snapinc=0):
    """FwiElastic2D::run_optimal; obs3 = [P, Ux, Uz] observed data, each [nr][nt].  With
    full_snapinc > 0: FwiElastic2D::run (full Vx/Vz snapshots every full_snapinc steps,
    DIFFERENCE misfit)."""
    g = pb.ref_grid()
    sc, gc = np.ascontiguousarray(scoords, np.float64), np.ascontiguousarray(gcoords, np.float64)
    ns, nr = len(sc), len(gc)
    out = {k: np.zeros((pb.nz, pb.nx), np.float32) for k in ("vpgrad", "vsgrad", "rhograd")}
    wg = np.zeros((ns, pb.nt), np.float32)
    mods = np.zeros((3, nr, pb.nt), np.float32)
    ress = np.zeros((3, nr, pb.nt), np.float32)
    mis = C.c_double()
    vp, vs, rho, w, op, ox, oz = _keep(pb.vp, pb.vs, pb.rho, wav, obs3[0], obs3[1], obs3[2], dtype=np.float32)
    if full_snapinc > 0:
        r = ref().ref_fwi_e2d_full_f(C.byref(g), _p(vp), _p(vs), _p(rho), ns, _p(sc), _p(w), sfield, nr, _p(gc),
                                     _p(op), _p(ox), _p(oz), full_snapinc, _p(out["vpgrad"]), _p(out["vsgrad"]),
                                     _p(out["rhograd"]), _p(wg), _p(mods), _p(ress), C.byref(mis))
    else:
        r = ref().ref_fwi_e2d_misfit_f(C.byref(g), _p(vp), _p(vs), _p(rho), ns, _p(sc), _p(w), sfield, nr, _p(gc),
                                       _p(op), _p(ox), _p(oz), ncheck, _p(out["vpgrad"]), _p(out["vsgrad"]),
                                       _p(out["rhograd"]), _p(wg), _p(mods), _p(ress), C.byref(mis), misfit)
    assert r == 1
    out.update(wavgrad=wg, datamod=mods, datares=ress, misfit=mis.value)
    return out


def ref_localsize2d(grid, scoords, gcoords, aperture, map_):
    """Model::getLocalsize2d: (start, size) of the x window of traces (sx, sz) / (gx, gz)."""
    sc, gc = np.ascontiguousarray(scoords, np.float64), np.ascontiguousarray(gcoords, np.float64)
    st, sz = C.c_longlong(), C.c_longlong()
    ref().ref_localsize2d_f(C.byref(grid), len(sc), _p(sc), _p(gc), float(aperture), int(map_), C.byref(st),
                            C.byref(sz))
    return st.value, sz.value


def ref_localsize3d(grid, scoords, gcoords, apx, apy, map_):
    """Model::getLocalsize3d: ((start_x, size_x), (start_y, size_y))."""
    sc, gc = np.ascontiguousarray(scoords, np.float64), np.ascontiguousarray(gcoords, np.float64)
    out = np.zeros(4, np.int64)
    ref().ref_localsize3d_f(C.byref(grid), len(sc), _p(sc), _p(gc), float(apx), float(apy), int(map_), _p(out))
    return (int(out[0]), int(out[1])), (int(out[2]), int(out[3]))


def ref_fwi_e3d(pb, scoords, wav, sfield, gcoords, obs3, ncheck):
    """FwiElastic3D::run_optimal; obs3 = [Ux, Uy, Uz] observed data, each [nr][nt]."""
    g = pb.ref_grid()
    sc, gc = np.ascontiguousarray(scoords, np.float64), np.ascontiguousarray(gcoords, np.float64)
    ns, nr = len(sc), len(gc)
    out = {k: np.zeros((pb.nz, pb.ny, pb.nx), np.float32) for k in ("vpgrad", "vsgrad", "rhograd")}
    wg = np.zeros((ns, pb.nt), np.float32)
    mods = np.zeros((3, nr, pb.nt), np.float32)
    ress = np.zeros((3, nr, pb.nt), np.float32)
    mis = C.c_double()
    vp, vs, rho, w, ox, oy, oz = _keep(pb.vp, pb.vs, pb.rho, wav, obs3[0], obs3[1], obs3[2], dtype=np.float32)
    r = ref().ref_fwi_e3d_f(C.byref(g), _p(vp), _p(vs), _p(rho), ns, _p(sc), _p(w), sfield, nr, _p(gc), _p(ox),
                            _p(oy), _p(oz), ncheck, _p(out["vpgrad"]), _p(out["vsgrad"]), _p(out["rhograd"]),
                            _p(wg), _p(mods), _p(ress), C.byref(mis))
    assert r == 1
    out.update(wavgrad=wg, datamod=mods, datares=ress, misfit=mis.value)
    return out


def orc_fwi_e2d(pb, padded, tab, smap, sshift, wav, sfield, gmaps, gshifts, obs3, misfit=0):
    g = pb.orc_grid()
    ns, nr = len(smap), len(gmaps[0])
    out = {k: np.zeros((pb.nz, pb.nx), np.float32) for k in ("vpgrad", "vsgrad", "rhograd")}
    wg = np.zeros((ns, pb.nt), np.float32)
    mods = np.zeros((3, nr, pb.nt), np.float32)
    ress = np.zeros((3, nr, pb.nt), np.float32)
    mis = C.c_double()
    Rx, Rz, L, L2M, M, tb, ss, w, vp, vs, rho = _keep(*padded, tab, sshift, wav, pb.vp, pb.vs, pb.rho,
                                                      dtype=np.float32)
    ob = np.ascontiguousarray(np.stack(obs3), np.float32)
    sm = np.ascontiguousarray(smap, np.int32)
    gm = [np.ascontiguousarray(m, np.int32) for m in gmaps]
    gs = [np.ascontiguousarray(s, np.float32) for s in gshifts]
    gmp = (C.c_void_p * 3)(*[m.ctypes.data for m in gm])
    gsp = (C.c_void_p * 3)(*[s.ctypes.data for s in gs])
    r = oracle().orc_fwi_e2d(C.byref(g), pb.nx, pb.nz, _p(vp), _p(vs), _p(rho), _p(Rx), _p(Rz), _p(L), _p(L2M),
                             _p(M), _p(tb), ns, _p(sm), _p(ss), _p(w), sfield, nr, gmp, gsp, _p(ob), misfit,
                             _p(out["vpgrad"]), _p(out["vsgrad"]), _p(out["rhograd"]), _p(wg), _p(mods), _p(ress),
                             C.byref(mis))
    assert r == 0
    out.update(wavgrad=wg, datamod=mods, datares=ress, misfit=mis.value)
    return out


def ref_rtm_a3d(pb, scoords, wav, gcoords, data, ncheck, nhx=1, nhy=1, nhz=1, full_snapinc=0):
    """RtmAcoustic3D::run_optimal, or RtmAcoustic3D::run with snapshots every full_snapinc steps."""
    g = pb.ref_grid()
    sc, gc = np.ascontiguousarray(scoords, np.float64), np.ascontiguousarray(gcoords, np.float64)
    img = np.zeros((nhz, nhy, nhx, pb.nz, pb.ny, pb.nx), np.float32)
    vp, rho, w, d = _keep(pb.vp, pb.rho, wav, data, dtype=np.float32)
    fn, n = (ref().ref_rtm_a3d_full_f, full_snapinc) if full_snapinc > 0 else (ref().ref_rtm_a3d_f, ncheck)
    r = fn(C.byref(g), _p(vp), _p(rho), len(sc), _p(sc), _p(w), len(gc), _p(gc), _p(d), n, nhx, nhy, nhz, _p(img))
    assert r == 1
    return img


def orc_rtm_a3d(pb, padded, tab, smap, sshift, wav, gmap, gshift, data, nhx=1, nhy=1, nhz=1):
    g = pb.orc_grid()
    img = np.zeros((nhz, nhy, nhx, pb.nz, pb.ny, pb.nx), np.float32)
    Rx, Ry, Rz, L, tb, ss, w, gs, d = _keep(*padded, tab, sshift, wav, gshift, data, dtype=np.float32)
    sm, gm = _keep(smap, gmap, dtype=np.int32)
    r = oracle().orc_rtm_a3d(C.byref(g), pb.nx, pb.ny, pb.nz, _p(Rx), _p(Ry), _p(Rz), _p(L), _p(tb), len(sm), _p(sm),
                             _p(ss), _p(w), len(gm), _p(gm), _p(gs), _p(d), nhx, nhy, nhz, _p(img))
    assert r == 0
    return img


def ref_fwi_a3d(pb, scoords, wav, gcoords, obs, ncheck, misfit=0):
    g = pb.ref_grid()
    sc, gc = np.ascontiguousarray(scoords, np.float64), np.ascontiguousarray(gcoords, np.float64)
    ns, nr = len(sc), len(gc)
    o = {k: np.zeros((pb.nz, pb.ny, pb.nx), np.float32) for k in ("vpgrad", "rhograd")}
    wg = np.zeros((ns, pb.nt), np.float32)
    dm = np.zeros((nr, pb.nt), np.float32)
    dr = np.zeros((nr, pb.nt), np.float32)
    mis = C.c_double()
    vp, rho, w, ob = _keep(pb.vp, pb.rho, wav, obs, dtype=np.float32)
    r = ref().ref_fwi_a3d_misfit_f(C.byref(g), _p(vp), _p(rho), ns, _p(sc), _p(w), nr, _p(gc), _p(ob), ncheck,
                                   _p(o["vpgrad"]), _p(o["rhograd"]), _p(wg), _p(dm), _p(dr), C.byref(mis), misfit)
    assert r == 1
    o.update(wavgrad=wg, datamod=dm, datares=dr, misfit=mis.value)
    return o


def orc_fwi_a3d(pb, padded, tab, smap, sshift, wav, gmap, gshift, obs, misfit=0):
    g = pb.orc_grid()
    ns, nr = len(smap), len(gmap)
    o = {k: np.zeros((pb.nz, pb.ny, pb.nx), np.float32) for k in ("vpgrad", "rhograd")}
    wg = np.zeros((ns, pb.nt), np.float32)
    dm = np.zeros((nr, pb.nt), np.float32)
    dr = np.zeros((nr, pb.nt), np.float32)
    mis = C.c_double()
    Rx, Ry, Rz, L, tb, ss, w, gs, ob, vp, rho = _keep(*padded, tab, sshift, wav, gshift, obs, pb.vp, pb.rho,
                                                      dtype=np.float32)
    sm, gm = _keep(smap, gmap, dtype=np.int32)
    r = oracle().orc_fwi_a3d(C.byref(g), pb.nx, pb.ny, pb.nz, _p(vp), _p(rho), _p(Rx), _p(Ry), _p(Rz), _p(L), _p(tb),
                             ns, _p(sm), _p(ss), _p(w), nr, _p(gm), _p(gs), _p(ob), misfit, _p(o["vpgrad"]),
                             _p(o["rhograd"]),
                             _p(wg), _p(dm), _p(dr), C.byref(mis))
    assert r == 0
    o.update(wavgrad=wg, datamod=dm, datares=dr, misfit=mis.value)
    return o


def ref_interp(mode, data, o1, d1, n2, o2, d2):
    """Interp<float>::interp of trace-major data [ntr][n1] onto n2 samples."""
    d = np.ascontiguousarray(data, np.float32)
    out = np.zeros((d.shape[0], n2), np.float32)
    assert ref().ref_interp_f(mode, d.shape[0], d.shape[1], o1, d1, _p(d), n2, o2, d2, _p(out)) == 1
    return out


def orc_interp(mode, data, o1, d1, n2, o2, d2):
    d = np.ascontiguousarray(data, np.float32)
    out = np.zeros((d.shape[0], n2), np.float32)
    assert oracle().orc_interp(mode, d.shape[0], d.shape[1], o1, d1, _p(d), n2, o2, d2, _p(out)) == 0
    return out


def ref_modelling_e3d(pb, scoords, wav, sfield, gcoords, rfield):
    """ModellingElastic3D<float>::run of the reference (traces [nrec][nt])."""
    out = np.zeros((len(gcoords), pb.nt), np.float32)
    g = pb.ref_grid()
    sc, gc = np.ascontiguousarray(scoords, np.float64), np.ascontiguousarray(gcoords, np.float64)
    vp, vs, rho, w = _keep(pb.vp, pb.vs, pb.rho, wav, dtype=np.float32)
    r = ref().ref_mod_e3d_f(C.byref(g), _p(vp), _p(vs), _p(rho), len(sc), _p(sc), _p(w), sfield, len(gc), _p(gc),
                            rfield, _p(out))
    assert r == 1
    return out


def ref_steps_e3d(pb, scoords, wav, sfield, nsteps, state=None):
    """The nine WavesElastic3D fields [9][nzp][nyp][nxp] after nsteps forward steps with
    source injection, or (state given) after nsteps backwardstep* steps from it."""
    shape = (9, pb.nz + 2 * pb.lpml, pb.ny + 2 * pb.lpml, pb.nx + 2 * pb.lpml)
    st = np.zeros(shape, np.float32) if state is None else np.ascontiguousarray(state, np.float32).copy()
    g = pb.ref_grid()
    sc = np.ascontiguousarray(scoords, np.float64)
    vp, vs, rho, w = _keep(pb.vp, pb.vs, pb.rho, wav, dtype=np.float32)
    r = ref().ref_steps_e3d_f(C.byref(g), _p(vp), _p(vs), _p(rho), len(sc), _p(sc), _p(w), sfield, nsteps,
                              0 if state is None else 1, _p(st))
    assert r == 1
    return st


# ---------------------------------------------------------------- shot-gather files and sorting
def ref_data_write(path, dim, nt, dt, ot, scoords, gcoords, data, dtype=np.float32):
    """Data2D::write (dim 2) / Data3D::write (dim 3) of the reference."""
    sc, gc, d = _keep(scoords, gcoords, data, dtype=dtype)
    fn = ref().ref_data_write_f if dtype == np.float32 else ref().ref_data_write_d
    assert fn(str(path).encode(), dim, nt, dt, ot, len(d), _p(sc), _p(gc), _p(d)) == 1


def ref_data_read2d(path, nt, ntrace):
    sc = np.zeros((ntrace, 2), np.float32)
    gc = np.zeros((ntrace, 2), np.float32)
    d = np.zeros((ntrace, nt), np.float32)
    assert ref().ref_data_read2d_f(str(path).encode(), nt, ntrace, _p(sc), _p(gc), _p(d)) == 1
    return sc, gc, d


def ref_model_write(path, vp, dx, dz, ox, oz):
    v = np.ascontiguousarray(vp, np.float32)
    nz, nx = v.shape
    assert ref().ref_model_write_f(str(path).encode(), nx, nz, dx, dz, ox, oz, _p(v)) == 1


def ref_sort_gather(path, dim, key, number, nt, dx=0.0, dy=0.0, order=0, reciprocity=0, dtype=np.float32, maxtr=4096):
    """Sort::create*map then get2DGather/get3DGather(number): (ngathers, scoords, gcoords, data)."""
    sc = np.zeros((maxtr, dim), dtype)
    gc = np.zeros((maxtr, dim), dtype)
    d = np.zeros((maxtr, nt), dtype)
    ng = C.c_longlong()
    fn = ref().ref_sort_gather_f if dtype == np.float32 else ref().ref_sort_gather_d
    n = fn(str(path).encode(), dim, key, dx, dy, order, number, reciprocity, C.byref(ng), _p(sc), _p(gc), _p(d),
           maxtr)
    assert n >= 0, n
    return ng.value, sc[:n], gc[:n], d[:n]


def ref_sort_put2d(survey, out, number, n1, d1, o1, data):
    d = np.ascontiguousarray(data, np.float32)
    return ref().ref_sort_put2d_f(str(survey).encode(), str(out).encode(), number, n1, d1, o1, _p(d))

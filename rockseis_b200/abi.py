"""ctypes binding of the C ABI declared in include/rsgpu.h.

The library is loaded from this package directory (built in-tree by
``python -m rockseis_b200.build``).  There is no fallback: if librsgpu.so is
missing or cannot be loaded, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librsgpu.so")

# status codes
OK, ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_STATE, ERR_TIMEOUT, ERR_UNSUPPORTED, ERR_NODEVICE, ERR_REVOLVE = range(9)
STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_NOMEM", 4: "ERR_STATE", 5: "ERR_TIMEOUT",
                6: "ERR_UNSUPPORTED", 7: "ERR_NODEVICE", 8: "ERR_REVOLVE"}
# physics / precision / fields (rs_field values of the reference, include/utils.h:22)
ACOUSTIC2D, ELASTIC2D, ACOUSTIC3D, ELASTIC3D = 0, 1, 2, 3
F32_EXACT, F32_FAST, F64 = 0, 1, 2
PRESSURE, VX, VY, VZ, SXX, SYY, SZZ, SYZ, SXZ, SXY = range(10)
CKPT_NATIVE, CKPT_F16, CKPT_BF16 = 0, 1, 2
ADVANCE, TAKESHOT, RESTORE, FIRSTURN, YOUTURN, TERMINATE, ERROR = range(7)
ACCUM_REFERENCE, ACCUM_F64 = 0, 1
MISFIT_DIFFERENCE, MISFIT_CORRELATION, MISFIT_ADAPTIVE_GAUSS, MISFIT_ADAPTIVE_LINEAR, MISFIT_ADAPTIVE_SINGLE = 0, 1, 2, 3, 4
INTERP_LINEAR, INTERP_BSPLINE, INTERP_SINC = 0, 1, 2
KIND_FWI, KIND_RTM = 0, 1


class RsgpuError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"rsgpu {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class Config(C.Structure):
    _fields_ = [("physics", C.c_int), ("precision", C.c_int), ("lpml", C.c_int), ("order", C.c_int),
                ("fs", C.c_int), ("nt", C.c_int), ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("dt", C.c_double), ("pml", C.c_void_p), ("tile", C.c_int), ("zchunk", C.c_int),
                ("launch_mode", C.c_int), ("reserved", C.c_int * 5)]


class Shot(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("model", C.c_void_p * 8),
                ("nsrc", C.c_int), ("smap", C.c_void_p), ("sshift", C.c_void_p), ("wavelet", C.c_void_p),
                ("src_field", C.c_int), ("nrec", C.c_int), ("gmap", C.c_void_p), ("gshift", C.c_void_p),
                ("rec_field", C.c_int), ("rec_factor", C.c_void_p), ("rec_out", C.c_void_p)]


SNAP_OPTIMAL, SNAP_FULL, SNAP_EDGES = 0, 1, 2


class AdjointOpts(C.Structure):
    _fields_ = [("ncheck", C.c_int), ("ckpt_precision", C.c_int), ("accum", C.c_int), ("misfit", C.c_int),
                ("nhx", C.c_int), ("nhz", C.c_int), ("nhy", C.c_int), ("snapmethod", C.c_int), ("snapinc", C.c_int),
                ("noreverse", C.c_int), ("reserved", C.c_int * 6)]


class AdjointShot(C.Structure):
    _fields_ = [("shot", Shot), ("vp", C.c_void_p), ("rho", C.c_void_p), ("data", C.c_void_p),
                ("vpgrad", C.c_void_p), ("rhograd", C.c_void_p), ("wavgrad", C.c_void_p), ("datares", C.c_void_p),
                ("misfit", C.POINTER(C.c_double)), ("image", C.c_void_p),
                ("gmap_vx", C.c_void_p), ("gmap_vz", C.c_void_p), ("gshift_vx", C.c_void_p), ("gshift_vz", C.c_void_p),
                ("data_vx", C.c_void_p), ("data_vz", C.c_void_p), ("vs", C.c_void_p), ("vsgrad", C.c_void_p),
                ("datamod_vx", C.c_void_p), ("datamod_vz", C.c_void_p), ("datares_vx", C.c_void_p),
                ("datares_vz", C.c_void_p), ("gmap_vy", C.c_void_p), ("gshift_vy", C.c_void_p),
                ("data_vy", C.c_void_p), ("datamod_vy", C.c_void_p), ("datares_vy", C.c_void_p),
                ("srcilum", C.c_void_p)]


class RssHeader(C.Structure):
    _fields_ = [("data_format", C.c_int), ("header_format", C.c_int), ("type", C.c_int),
                ("nheader", C.c_longlong), ("ndims", C.c_longlong), ("n", C.c_longlong * 9),
                ("d", C.c_double * 9), ("o", C.c_double * 9)]


RSS_GENERIC, RSS_REGULAR, RSS_DATA2D, RSS_DATA3D = 0, 1, 2, 3
SORT_SOURCE, SORT_RECEIVER, SORT_CMP = 0, 1, 2
GATHER_FINISHED, GATHER_RUNNING, GATHER_NOT_STARTED, GATHER_FAILED = 0, 1, 2, 3


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m rockseis_b200.build`")
    lib = C.CDLL(LIB_PATH)
    P, I, D, V = C.POINTER, C.c_int, C.c_double, C.c_void_p
    sig = {
        "rsgpu_abi_version": (I, []),
        "rsgpu_last_error": (C.c_char_p, []),
        "rsgpu_device_count": (I, []),
        "rsgpu_modelling": (I, [P(Config), I, P(Shot)]),
        "rsgpu_plan_create": (I, [P(Config), I, P(Shot), P(V)]),
        "rsgpu_plan_reset": (I, [V]),
        "rsgpu_plan_run": (I, [V, I, I]),
        "rsgpu_plan_read_traces": (I, [V, I, V]),
        "rsgpu_plan_read_field": (I, [V, I, I, V]),
        "rsgpu_plan_sync": (I, [V]),
        "rsgpu_plan_stream": (V, [V]),
        "rsgpu_plan_launch_count": (C.c_longlong, [V]),
        "rsgpu_plan_enable_timing": (I, [V]),
        "rsgpu_plan_kernel_times": (I, [V, P(C.c_float), P(C.c_float)]),
        "rsgpu_plan_info": (I, [V, P(I), P(I), P(I)]),
        "rsgpu_release_cached_memory": (I, []),
        "rsgpu_plan_destroy": (None, [V]),
        "rsgpu_modelling_a2d_noalloc": (I, [P(Config), P(Shot), V]),
        "rsgpu_selftest_bounded_wait": (I, []),
        "rsgpu_interp_traces": (I, [I, I, I, I, D, D, V, I, D, D, V]),
        "rsgpu_tile_count": (I, [I]),
        "rsgpu_tile_shape": (I, [I, I, P(I), P(I), P(I), P(I)]),
        "rsgpu_pml_tables": (I, [I, D, I, V]),
        "rsgpu_stagger_model": (I, [I, I, I, I, I, I, I, V, V, V, P(V)]),
        "rsgpu_make_map": (I, [I, I, I, P(D), P(I), P(D), P(D), P(D), P(I), V]),
        "rsgpu_revolve_trace": (I, [I, I, I, P(I), P(I), P(I), P(I)]),
        "rsgpu_revolve_numforw": (I, [I, I]),
        "rsgpu_fwi_gradient": (I, [P(Config), P(AdjointOpts), I, P(AdjointShot)]),
        "rsgpu_rtm_image": (I, [P(Config), P(AdjointOpts), I, P(AdjointShot)]),
        "rsgpu_adjoint_create": (I, [P(Config), P(AdjointOpts), I, I, P(AdjointShot), P(V)]),
        "rsgpu_adjoint_run": (I, [V]),
        "rsgpu_adjoint_read": (I, [V, I, P(AdjointShot)]),
        "rsgpu_adjoint_stats": (I, [V] + [P(C.c_longlong)] * 4),
        "rsgpu_adjoint_stream": (V, [V]),
        "rsgpu_adjoint_destroy": (None, [V]),
        "rsgpu_adjoint_stack": (I, [V, I, I, P(I), P(I), V, V, V]),
        "rsgpu_rss_read_header": (I, [C.c_char_p, P(RssHeader)]),
        "rsgpu_rss_write_traces": (I, [C.c_char_p, I, I, C.c_longlong, D, D, C.c_longlong, V, V, V]),
        "rsgpu_rss_read_traces": (I, [C.c_char_p, I, C.c_longlong, C.c_longlong, V, V, V]),
        "rsgpu_rss_write_model": (I, [C.c_char_p, I, I, I, I, D, D, D, D, D, D, V]),
        "rsgpu_rss_read_model": (I, [C.c_char_p, I, C.c_longlong, V]),
        "rsgpu_sort_create": (I, [C.c_char_p, I, D, D, I, P(V)]),
        "rsgpu_sort_destroy": (None, [V]),
        "rsgpu_sort_info": (I, [V, P(C.c_longlong), P(C.c_longlong), P(C.c_longlong)]),
        "rsgpu_sort_gather_size": (C.c_longlong, [V, C.c_longlong]),
        "rsgpu_sort_next": (C.c_longlong, [V]),
        "rsgpu_sort_status": (I, [V, C.c_longlong]),
        "rsgpu_sort_set_status": (I, [V, C.c_longlong, I]),
        "rsgpu_sort_read_gather": (I, [V, C.c_longlong, I, V, V, V]),
        "rsgpu_sort_create_output": (I, [V, C.c_char_p, C.c_longlong, D, D]),
        "rsgpu_sort_write_gather": (I, [V, C.c_char_p, C.c_longlong, I, C.c_longlong, V, V, V]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int) -> None:
    if status != OK:
        raise RsgpuError(status, lib.rsgpu_last_error().decode())


def ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays crossing the C ABI must be C-contiguous"
    return a.ctypes.data


def real_dtype(precision: int):
    return np.float64 if precision == F64 else np.float32

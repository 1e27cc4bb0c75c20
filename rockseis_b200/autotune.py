"""Tile-shape autotuner of the 2D propagators, with a JSON cache.

The 2D kernels are compiled for several tile shapes (x and z extent of the tile a
CTA updates, rows per thread, CTAs per SM; rsgpu_tile_count / rsgpu_tile_shape).
Which one is fastest depends on the physics, the arithmetic and how many padded
points the batch holds: a few small shots want small tiles to fill 148 SMs, a
large batch wants the shape with the most loads in flight.  `tune_tile` builds
the batch once per shape as a device-resident plan, replays a short stretch of
the time loop, reads the per-launch kernel times the plan records with CUDA
events, and keeps the shape with the shortest velocity + stress half-steps.  The
choice is cached in JSON under a key made of the device name, physics,
arithmetic, order, shot count and padded grid sizes, so the search runs once per
problem class.  Every shape computes the same numbers (the tile only changes
which CTA updates a point), so the choice never changes results.
"""
from __future__ import annotations

import json
import os
import time

from . import abi
from .rockseis import Plan

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "rockseis_b200", "tiles.json")
AUTO = -2          # tile value that asks the Python drivers to autotune


def cache_path() -> str:
    return os.environ.get("RSGPU_TILE_CACHE", DEFAULT_CACHE)


def tile_shapes(precision: int) -> dict[int, tuple[int, int, int, int]]:
    """{index: (tx, tz, rows_per_thread, ctas_per_sm)} of the shapes built for `precision`."""
    import ctypes as C
    out = {}
    for i in range(abi.lib.rsgpu_tile_count(precision)):
        v = [C.c_int() for _ in range(4)]
        if abi.lib.rsgpu_tile_shape(precision, i, *[C.byref(x) for x in v]) == abi.OK:
            out[i] = tuple(x.value for x in v)
    return out


def _device_name() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(torch.cuda.current_device())
    except Exception:
        pass
    return "unknown-device"


def problem_key(models, order: int, precision: int) -> str:
    dims = sorted((m.getNx_pml(), m.getNz_pml()) for m in models)
    pts = sum(a * b for a, b in dims)
    return (f"{_device_name()}|physics{models[0].physics}|prec{precision}|order{order}|shots{len(models)}|"
            f"pts{pts}|max{max(d[0] for d in dims)}x{max(d[1] for d in dims)}")


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(path, table):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def measure_tile(models, sources, receivers, order, precision, tile, warm=8, steps=32) -> float:
    """Mean velocity + stress half-step time (ms) of shape `tile` over `steps` time steps."""
    nt = sources[0].nt
    warm, steps = min(warm, max(nt - 1, 0)), max(1, min(steps, nt - min(warm, nt - 1)))
    plan = Plan(models, sources, receivers, order, precision, tile)
    try:
        plan.enable_timing()
        plan.run(0, warm)
        plan.run(warm, steps)
        plan.sync()
        v, s = plan.kernel_times()
    finally:
        plan.close()
    return float(v + s)


def tune_tile(models, sources, receivers, order, precision=abi.F32_EXACT, cache: str | None = None,
              refresh: bool = False, warm: int = 8, steps: int = 32) -> int:
    """Fastest tile shape index for this batch, from the cache or by measurement."""
    path = cache or cache_path()
    key = problem_key(models, order, precision)
    table = _load(path)
    if not refresh and key in table:
        return int(table[key]["tile"])
    shapes = tile_shapes(precision)
    if not shapes:
        abi.check(abi.ERR_ARG)
    ms = {}
    t0 = time.perf_counter()
    for i in shapes:
        ms[i] = measure_tile(models, sources, receivers, order, precision, i, warm, steps)
    best = min(ms, key=ms.get)
    table = _load(path)          # merge with entries written meanwhile
    table[key] = {"tile": best, "shape": list(shapes[best]), "ms_per_step": {str(k): round(v, 5) for k, v in ms.items()},
                  "search_s": round(time.perf_counter() - t0, 3)}
    _store(path, table)
    return best


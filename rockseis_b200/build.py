"""Build librsgpu.so (the C-ABI library of include/rsgpu.h) in-tree.

Every CUDA translation unit is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``); host C++ is compiled with the
same nvcc driver.  Objects go to ``rockseis_b200/_build`` and are rebuilt only
when a source or header is newer.  Translation units compile in parallel.

Usage:  python -m rockseis_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "librsgpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
              "-I" + INCLUDE, "-I" + CSRC]
HOST_FLAGS = ["-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
              "-I" + INCLUDE, "-I" + CSRC]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build librsgpu")
    return path


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(obj: str, src: str, hdr_mtime: float) -> bool:
    if not os.path.exists(obj):
        return True
    m = os.path.getmtime(obj)
    return m < os.path.getmtime(src) or m < hdr_mtime


def _compile(src: str, obj: str, verbose: bool) -> None:
    if src.endswith(".cu"):
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
    else:
        cmd = [nvcc()] + HOST_FLAGS + ["-x", "c++", "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {os.path.basename(src)}\n{r.stdout}\n{r.stderr}")


# Kernel instantiations of the 2D propagators: (name, T, MODE) x tile configs
# (TX, TZ, RZ, MINB).  The config index is the `tile` field of rsgpu_config.
# One small translation unit each so nvcc compiles them in parallel.
VARIANTS_2D = [("f32x", "float", "MODE_IEEE"), ("f32f", "float", "MODE_FAST"), ("f64", "double", "MODE_IEEE")]
TILES_2D = [(64, 32, 4, 1), (64, 64, 4, 1), (32, 32, 4, 1), (32, 16, 4, 1), (32, 32, 2, 1), (64, 32, 2, 1),
            (32, 32, 2, 6), (32, 32, 2, 8), (64, 32, 2, 3), (32, 16, 2, 8)]
TILES_F64 = (0, 3)   # FP64 oracle propagator: two shapes


def _generate() -> list[str]:
    gen = os.path.join(BUILD, "gen")
    os.makedirs(gen, exist_ok=True)
    out, table = [], []
    for name, t, mode in VARIANTS_2D:
        for idx, (tx, tz, rz, mb) in enumerate(TILES_2D):
            if t == "double" and idx not in TILES_F64:
                continue
            fn = f"launch_2d_{name}_{tx}x{tz}r{rz}m{mb}"
            src = ("// generated by rockseis_b200/build.py\n#include \"fd2d_kernels.cuh\"\nnamespace rsgpu {\n"
                   f"cudaError_t {fn}(int physics, int half, int flags, const void *args, const void *coefs, "
                   "const void *maps, int *err, int grid, cudaStream_t st)\n{\n"
                   f"    return launch_2d_cfg<{t}, {mode}, {tx}, {tz}, {rz}, {mb}>(physics, half, flags, "
                   f"*static_cast<const Step2DArgs<{t}> *>(args), static_cast<const CoefSet<{t}> *>(coefs), "
                   "static_cast<const CUtensorMap *>(maps), err, grid, st);\n}\n}  // namespace rsgpu\n")
            path = os.path.join(gen, fn + ".cu")
            if not os.path.exists(path) or open(path).read() != src:
                with open(path, "w") as f:
                    f.write(src)
            out.append(path)
            table.append((name, idx, fn))
    decl = "".join(f"cudaError_t {fn}(int, int, int, const void *, const void *, const void *, int *, int, "
                   "cudaStream_t);\n" for _, _, fn in table)
    cases = ""
    for name in [v[0] for v in VARIANTS_2D]:
        cases += f"    if (variant == \"{name}\") {{\n        switch (cfg) {{\n"
        for n2, idx, fn in table:
            if n2 == name:
                cases += f"        case {idx}: return {fn};\n"
        cases += "        default: return nullptr;\n        }\n    }\n"
    shapes = "".join(f"    case {i}: return {{{tx}, {tz}, {rz}, {mb}}};\n" for i, (tx, tz, rz, mb) in enumerate(TILES_2D))
    disp = ("// generated by rockseis_b200/build.py\n#include <string>\n#include \"rsgpu_kernels.h\"\n"
            "namespace rsgpu {\n" + decl +
            "Launch2DFn launch_2d_table(const char *v, int cfg)\n{\n    std::string variant(v);\n" + cases +
            "    return nullptr;\n}\n"
            "TileShape tile_shape_2d(int cfg)\n{\n    switch (cfg) {\n" + shapes +
            "    default: return {0, 0, 0, 0};\n    }\n}\n"
            f"int tile_count_2d() {{ return {len(TILES_2D)}; }}\n"
            "}  // namespace rsgpu\n")
    path = os.path.join(gen, "fd2d_table.cpp")
    if not os.path.exists(path) or open(path).read() != disp:
        with open(path, "w") as f:
            f.write(disp)
    out.append(path)
    return out


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp"))) + _generate()
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [0.0])
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(o, s, hdr_mtime):
            jobs.append((s, o))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
            futs = [ex.submit(_compile, s, o, verbose) for s, o in jobs]
            for f in futs:
                f.result()
    if jobs or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    sys.exit(0)

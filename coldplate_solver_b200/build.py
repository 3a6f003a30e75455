"""Build recipe for libcps.so (sm_100a) -- compiled in-tree so it travels with
the repository snapshot.

The tile shape of the kernels is a compile-time constant, so each shape is
its own library with the same C ABI: libcps.so (8 x 32 tiles, the default and
the one the C++ drop-in links), libcps_t16.so (16 x 16) and libcps_t64.so
(4 x 64).  The three compile in parallel.

``--fmad=false``: the FP64 path keeps the reference's separate multiply and
add roundings, so per-point values match the FP64 reference exactly; the
kernels are bound by memory and barrier latency, not by FP64 issue rate.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)
LIB_PATH = os.path.join(PKG_DIR, "libcps.so")
TILE_WIDTHS = (32, 16, 64)  # tile columns; rows = 256 / columns


def lib_path(tile_j: int = 32) -> str:
    """The library built with tiles of ``tile_j`` columns."""
    if tile_j not in TILE_WIDTHS:
        raise ValueError(f"tile width {tile_j} is not built (have {TILE_WIDTHS})")
    return LIB_PATH if tile_j == 32 else os.path.join(PKG_DIR, f"libcps_t{tile_j}.so")


SOURCES = [os.path.join(PKG_DIR, "csrc", f) for f in ("cps_api.cu", "cps_noalloc.cu", "cps_thermal.cu", "cps_io.cpp",
                                                              "cps_thermal_io.cpp")]
HEADERS = [os.path.join(PKG_DIR, "csrc", f) for f in os.listdir(os.path.join(PKG_DIR, "csrc")) if f.endswith(".cuh")]
HEADERS.append(os.path.join(REPO_DIR, "include", "cps.h"))
HEADERS.append(os.path.join(REPO_DIR, "include", "cps_thermal.h"))

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def needs_build(path: str = LIB_PATH) -> bool:
    if not os.path.exists(path):
        return True
    t = os.path.getmtime(path)
    return any(os.path.getmtime(f) > t for f in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> str:
    """Build every tile-shape library that is missing or older than its
    sources (all of them with ``force``); returns the default library's path."""
    todo = [j for j in TILE_WIDTHS if force or needs_build(lib_path(j))]
    env = dict(os.environ)
    env.pop("CXX", None)
    env.pop("CC", None)
    procs = []
    for j in todo:
        cmd = [nvcc(), *NVCC_FLAGS, f"-DCPS_TILE_J={j}", "-o", lib_path(j), *SOURCES]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), file=sys.stderr)
        procs.append((j, subprocess.Popen(cmd, env=env)))
    failed = [j for j, p in procs if p.wait() != 0]
    if failed:
        raise RuntimeError(f"nvcc failed for tile widths {failed}")
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)

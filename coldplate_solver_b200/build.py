"""Build recipe for libcps.so (sm_100a) -- compiled in-tree so it travels with
the repository snapshot.

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


def needs_build() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    return any(os.path.getmtime(f) > t for f in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB_PATH
    cmd = [nvcc(), *NVCC_FLAGS, "-o", LIB_PATH, *SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    env = dict(os.environ)
    env.pop("CXX", None)
    env.pop("CC", None)
    subprocess.run(cmd, check=True, env=env)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)

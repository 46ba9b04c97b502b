"""Builds the sm_100a lane library in-tree: egspice_b200/_lib/libespice_lanes.so."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libespice_lanes.so")
SOURCES = ["espice_lanes.cu", "tape.cpp", "mlp.cu"]
HEADERS = ["lane_engine.cuh", "lane_kernels.cuh", "lane_models.cuh", "lane_smem.cuh", "lane_tile.cuh", "lane_band.cuh", "lane_meas.cuh", "lane_ac.cuh", "lane_ac_core.cuh", "tape.h",
           "mlp_gemm.cuh", "lane_gates.cuh", "lane_learned.cuh", "lane_levels.cuh", "../../include/espice_learned.h",
           "../../include/espice_lanes.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
         "--expt-relaxed-constexpr", "-Xptxas", "-v"]


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(SRC, f) for f in SOURCES + HEADERS]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    for f in SOURCES:
        o = os.path.join(OUT_DIR, f + ".o")
        cmd = [NVCC] + FLAGS + ["-c", os.path.join(SRC, f), "-o", o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {f}")
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(o)
    tmp = LIB + ".tmp"
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

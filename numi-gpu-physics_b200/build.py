"""Builds libbfx.so (the CUDA library behind include/bfx.h) in-tree for sm_100a.

    python numi-gpu-physics_b200/build.py [--verbose]

nvcc cross-compiles without a GPU.  --fmad=false keeps every a*b+c unfused so
the FP32 step reproduces the reference operation order bit for bit; the host
compiler gets -ffp-contract=off for the same reason.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libbfx.so")
SOURCES = ["bfx_fluid.cu", "bfx_fluid_fast.cu", "bfx_geometry.cu", "bfx_adjoint.cu", "bfx_ledger.cu", "bfx_api.cu",
           "bfx_noalloc.cu", "bfx_fields.cu"]
# translation units built with FMA contraction (see csrc/bfx_bulk.cuh)
CONTRACTED = {"bfx_fluid_fast.cu"}
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]


def build(verbose: bool = False, force: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    deps.append(os.path.abspath(__file__))
    deps.append(os.path.join(HERE, "..", "include", "bfx.h"))
    if not force and os.path.exists(OUT):
        newest = max(os.path.getmtime(d) for d in deps)
        if os.path.getmtime(OUT) >= newest:
            return OUT
    objs = []
    build_dir = os.path.join(HERE, "_build")
    os.makedirs(build_dir, exist_ok=True)
    procs = []
    for src in srcs:
        obj = os.path.join(build_dir, os.path.basename(src) + ".o")
        flags = [("--fmad=true" if f == "--fmad=false" and os.path.basename(src) in CONTRACTED else f) for f in FLAGS]
        cmd = [NVCC, *flags, "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        procs.append((subprocess.Popen(cmd), cmd))
        objs.append(obj)
    failed = [cmd for p, cmd in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    link = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", OUT, "-lcudart"]
    subprocess.run(link, check=True)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build(verbose=args.verbose, force=args.force))
    sys.exit(0)

"""Builds the in-tree CUDA library ``celeris_b200/_build/libceleris_b200.so`` for sm_100a.

``python -m celeris_b200.build`` (or ``__graft_entry__.build()``) compiles every source with
nvcc (it cross-compiles without a GPU) and links one shared library that exports the C ABI of
include/celeris_b200.h.  The plain form is compiled with ``-fmad=false`` so its single-precision
arithmetic follows the FP32 transcription operation by operation; the fused forms keep FMA
contraction.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libceleris_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]

UNITS = [
    ("params.cpp", []),
    ("setup.cpp", []),
    ("logio.cpp", []),
    ("spectrum.cpp", []),
    ("capi.cpp", []),
    ("lanes.cpp", []),
    ("plain.cu", ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"]),
    ("fused.cu", ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]),
]
HEADERS = ["celeris_internal.hpp", "engine_iface.hpp", "scheme.hpp", "device_math.cuh", "batch.hpp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_compiler() -> list:
    # The system g++ (the environment's CXX wrapper may not carry every runtime spec file).
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    inc = os.path.join(HERE, "..", "include")
    hdr_mtime = max(os.path.getmtime(os.path.join(SRC, h)) for h in HEADERS)
    hdr_mtime = max(hdr_mtime, os.path.getmtime(os.path.join(inc, "celeris_b200.h")))
    objs = []
    changed = False
    for src, extra in UNITS:
        s = os.path.join(SRC, src)
        o = os.path.join(OUT, src + ".o")
        objs.append(o)
        if os.path.exists(o) and os.path.getmtime(o) > max(os.path.getmtime(s), hdr_mtime) and not ptxas_info:
            continue
        # CEL_NVCC_FLAGS: extra nvcc flags for the CUDA units (tuning builds, e.g. -DCEL_MARCH_MIN_CTAS=5)
        tune = os.environ.get("CEL_NVCC_FLAGS", "").split() if src.endswith(".cu") else []
        cmd = [nvcc(), *_host_compiler(), *ARCH, *COMMON, *extra, *tune, "-I", inc, "-c", s, "-o", o]
        if ptxas_info and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src}")
        if ptxas_info and r.stderr:
            sys.stderr.write(r.stderr)
        changed = True
    if changed or not os.path.exists(LIB):
        cmd = [nvcc(), *_host_compiler(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-ldl", "-lrt",
               "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))

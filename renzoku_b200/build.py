"""Builds librzk_cuda.so in-tree for sm_100a (no JIT cache: the library travels with the
repository copy).

Flags: -fmad=false with IEEE division and square root keeps every geometric operation a
separately rounded IEEE single-precision operation in the reference's order, which is
what makes Morton codes, the BVH, ray predicates and primary hits bit-identical to the
reference.  Host code is compiled with -ffp-contract=off for the same reason.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "librzk_cuda.so")
SOURCES = ["rzk_bvh.cu", "rzk_trace.cu", "rzk_gather.cu", "rzk_vplgen.cu", "rzk_capi.cu",
           "rzk_noalloc.cu", "rzk_cluster.cu", "rzk_batch.cu", "rzk_lightslice.cu", "rzk_guided.cu", "rzk_server.cu", "rzk_sah.cu", "rzk_mrcs.cu",
           "rzk_serial.cu", "rzk_obj.cu", "rzk_json.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-fmad=false",
         "-prec-div=true", "-prec-sqrt=true", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
         "-shared"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps += [os.path.join(HERE, "..", "include", f) for f in os.listdir(os.path.join(HERE, "..", "include"))]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if force or _stale():
        cmd = [NVCC, *FLAGS, "-o", LIB, *[os.path.join(CSRC, s) for s in SOURCES]]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)

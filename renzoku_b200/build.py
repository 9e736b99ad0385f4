"""Builds librzk_cuda.so in-tree for sm_100a (no JIT cache: the library travels with the
repository copy).

Flags: -fmad=false with IEEE division and square root keeps every geometric operation a
separately rounded IEEE single-precision operation in the reference's order, which is
what makes Morton codes, the BVH, ray predicates and primary hits bit-identical to the
reference.  Host code is compiled with -ffp-contract=off for the same reason.

Each translation unit is compiled to its own object in parallel (no relocatable device
code: no device symbol crosses a file), then the objects are linked into the library.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference source tree, read only for its headers by the drop-in classes (absent where
# the prebuilt librzk_dropin.so travels without it)
REFERENCE_TREE = os.environ.get("RZK_REFERENCE_TREE", "/root/reference")
DROPIN = os.path.join(HERE, "librzk_dropin.so")
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "librzk_cuda.so")
OBJ = os.path.join(HERE, "_build")
SOURCES = ["rzk_bvh.cu", "rzk_trace.cu", "rzk_gather.cu", "rzk_vplgen.cu", "rzk_capi.cu",
           "rzk_noalloc.cu", "rzk_cluster.cu", "rzk_batch.cu", "rzk_lightslice.cu", "rzk_guided.cu", "rzk_server.cu", "rzk_sah.cu", "rzk_mrcs.cu",
           "rzk_serial.cu", "rzk_obj.cu", "rzk_json.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [*ARCH, "-O3", "-lineinfo", "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-std=c++17",
         "-Xcompiler", "-fPIC,-ffp-contract=off"]


def _deps():
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    inc = os.path.join(HERE, "..", "include")
    return deps + [os.path.join(inc, f) for f in os.listdir(inc)]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in _deps())


def _obj(src: str) -> str:
    return os.path.join(OBJ, src.replace(".cu", ".o"))


def build(force: bool = False, verbose: bool = False) -> str:
    if not (force or _stale()):
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    newest_dep = max(os.path.getmtime(d) for d in _deps())

    def compile_one(src):
        o = _obj(src)
        # every object depends on the shared headers, so any change rebuilds all of them
        if not force and os.path.exists(o) and os.path.getmtime(o) > newest_dep:
            return
        cmd = [NVCC, *FLAGS, "-c", "-o", o, os.path.join(CSRC, src)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        list(ex.map(compile_one, SOURCES))
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *[_obj(s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


def build_dropin(force: bool = False) -> str | None:
    """librzk_dropin.so (renzoku_b200/dropin): the C++ classes behind the reference's
    Aggregate / IVplGenerator / Integrator interfaces.  Needs the reference's headers; where
    they are absent the prebuilt library is used as it is (None if there is none)."""
    build()
    if os.path.isdir(REFERENCE_TREE):
        args = ["make", "-s", "-C", os.path.join(HERE, "dropin"), f"REF={REFERENCE_TREE}"]
        if force:
            args.append("-B")
        subprocess.run(args, check=True)
    return DROPIN if os.path.exists(DROPIN) else None


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    build_dropin(force="--force" in sys.argv)

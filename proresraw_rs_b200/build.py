"""Builds the package's native libraries in-tree.

 - lib/libprr.so        CUDA sm_100a kernels + the C ABI of include/prr.h
                        (and the host movie reader and DNG container)
 - lib/libprr_synth.so  host C++ synthetic-input generator and encoder

Float flags matter for bit-exactness: -fmad=false (the device code spells
its IEEE operations as _rn intrinsics anyway), IEEE division and square
root, no flush-to-zero, and -ffp-contract=off for host code (the f64
parameter math must not be contracted).

Usage: python -m proresraw_rs_b200.build [--verbose]
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O3",
    "-shared",
]
CUDA_SOURCES = ["api.cu", "batch.cu", "clip.cu", "decode.cu", "develop.cu", "learned.cu", "lj92.cu", "noalloc.cu"]
# Host-only parts of libprr.so (the movie reader, the DNG container); nvcc
# hands them to g++.
HOST_SOURCES = ["dng.cpp", "mov.cpp"]
CXX_FLAGS = ["-O3", "-march=x86-64-v3", "-std=c++17", "-fPIC", "-pthread", "-ffp-contract=off", "-shared"]


def nvcc() -> str:
    for cand in [os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")]:
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stdout.write(r.stdout)
        sys.stderr.write(r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}")
    return r


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> None:
    os.makedirs(LIB, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers += [os.path.join(HERE, "..", "include", "prr.h"), os.path.join(HERE, "..", "include", "prr_synth.h")]
    cu = [os.path.join(CSRC, f) for f in CUDA_SOURCES + HOST_SOURCES]
    out = os.path.join(LIB, "libprr.so")
    if force or _stale(out, cu + headers):
        cmd = [nvcc(), *NVCC_FLAGS, *(["-Xptxas", "-v"] if ptxas_info else []), "-o", out, *cu]
        _run(cmd, verbose or ptxas_info)
    syn_src = os.path.join(CSRC, "synth.cpp")
    syn_out = os.path.join(LIB, "libprr_synth.so")
    if force or _stale(syn_out, [syn_src] + headers):
        _run([os.environ.get("CXX", "g++"), *CXX_FLAGS, "-o", syn_out, syn_src], verbose)


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)

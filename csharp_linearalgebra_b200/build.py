"""Build the sm_100a CUDA library in-tree: csharp_linearalgebra_b200/libtensile_b200.so.

nvcc cross-compiles for sm_100a without a GPU. Device code is compiled with
--fmad=false so that no multiply and add are contracted unless the source asks
for a fused multiply-add explicitly (the DMMA tensor-core instructions and
explicit fma() calls); host code with -ffp-contract=off for the same reason.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtensile_b200.so")
OBJ = os.path.join(HERE, "_build")

SOURCES = ["context.cu", "gemm.cu", "blas1.cu", "lu.cu", "algos.cu", "expm_batched.cu", "expmv_batched.cu", "capi.cu",
           "noalloc.cu",
           "ozaki.cu", "frechet.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-Xptxas", "-warn-spills",
]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "tensile_b200.h"))
    objs, procs = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if _stale(o, [s] + headers):
            cmd = [_nvcc(), *NVCC_FLAGS, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
            while len([p for _, p in procs if p.poll() is None]) >= jobs:
                procs[0][1].wait()
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            failed.append((src, text))
        elif verbose and text.strip():
            print(text)
    if failed:
        for src, text in failed:
            sys.stderr.write(f"--- {src}\n{text}\n")
        raise RuntimeError("nvcc failed for " + ", ".join(s for s, _ in failed))
    if _stale(LIB, objs):
        cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

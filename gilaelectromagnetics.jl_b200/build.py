"""Build libgila_b200.so in-tree with nvcc for sm_100a.

Usage:  python gilaelectromagnetics.jl_b200/build.py [--force] [--verbose]

The library is a plain C-ABI shared object (see include/gila_b200.h); it links
the CUDA runtime statically so that it loads next to PyTorch or Julia's
CUDA.jl without symbol clashes.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgila_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["gila.cu", "matvec.cu", "matvec_c128.cu", "matvec_c64.cu", "noalloc.cu", "slab.cu", "kerbuild.cu",
           "solver.cu", "server.cu"]
HEADERS = ["fft.cuh", "fft_ct.cuh", "matvec.cuh", "matvec_impl.cuh", "internal.h", "solver.h"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra_flags=None, out: str = LIB,
          objdir: str | None = None) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "gila_b200.h")]
    if not force and not _stale(out, deps):
        return out
    objdir = objdir or os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    nvcc = _nvcc()
    flags = NVCC_FLAGS + list(extra_flags or [])
    objs = [os.path.join(objdir, os.path.basename(s) + ".o") for s in srcs]
    cmds = [[nvcc, *flags, "-I", INCLUDE, "-c", s, "-o", o] for s, o in zip(srcs, objs)]
    if verbose:
        for c in cmds:
            print(" ".join(c), flush=True)
    # the translation units compile in parallel
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for r in ex.map(lambda c: subprocess.run(c, check=True), cmds):
            pass
    cmd = [nvcc, *flags, "-shared", "-o", out, *objs, "-lcudart_static", "-lrt", "-lpthread", "-ldl"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register / smem use")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_v else []
    print(build(force=a.force or a.ptxas_v, verbose=a.verbose, extra_flags=extra))
    sys.exit(0)

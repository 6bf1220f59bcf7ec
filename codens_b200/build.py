"""Build recipe of the CUDA library ``libcodens_b200.so`` (sm_100a only).

The library is built in-tree so that it travels with the source tree; it is
a plain C-ABI shared object (include/cns_abi.h) with no Python or torch
dependency.  ``--fmad=false`` keeps every FP64 multiply and add separately
rounded, which is what makes the results bit-identical to the reference
arithmetic.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcodens_b200.so")
# FP64 parity sources: no FMA contraction, every product and sum rounded as
# written.  The FP32 half of the mixed-precision form (cns_mixed.cu) is not a
# parity path: it is built with contraction and with the approximate
# single-precision division and square root (-prec-div/-prec-sqrt affect FP32
# only; its FP64 residual keeps IEEE division), which the mixed form's FP64
# fixed point does not depend on.
SOURCES = ["cns_geom.cu", "cns_flow.cu", "cns_jameson.cu", "cns_turb.cu", "cns_sa.cu",
           "cns_adjoint.cu", "cns_abi.cu", "cns_noalloc.cu", "cns_io.cu", "cns_weno.cu",
           "cns_ke.cu"]
SOURCES_FMA = ["cns_mixed.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
OBJDIR = os.path.join(HERE, "_build")

COMMON = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
    "-I" + os.path.join(ROOT, "include"),
]
FLAGS = COMMON + ["--fmad=false"]
FLAGS_FMA = COMMON + ["--fmad=true", "-prec-div=false", "-prec-sqrt=false"]


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES + SOURCES_FMA]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC)
                        if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(ROOT, "include", "cns_abi.h"))
    return all(os.path.getmtime(d) <= t for d in deps)


def _run(cmd, verbose):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libcodens_b200.so")
    if verbose:
        sys.stderr.write(r.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose else []
    objs = []
    for names, flags in ((SOURCES, FLAGS), (SOURCES_FMA, FLAGS_FMA)):
        for s in names:
            o = os.path.join(OBJDIR, s.replace(".cu", ".o"))
            _run([NVCC] + flags + extra + ["-c", os.path.join(CSRC, s), "-o", o], verbose)
            objs.append(o)
    _run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a"] + objs
         + ["-o", LIB], verbose)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose="-v" in sys.argv)
    print(LIB)

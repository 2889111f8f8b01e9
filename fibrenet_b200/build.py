"""Builds the native library in-tree: fibrenet_b200/libfibrenet.so.

nvcc compiles the CUDA kernels for sm_100a only, with -fmad=false so no
a*b+c is contracted into an FMA (the results stay bit-identical to a host
mirror of the same arithmetic), and links the C++ host engine behind the C
ABI declared in include/fibrenet.h.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfibrenet.so")
CLI = os.path.join(HERE, "fibrenet_run")
SOURCES = ["fn_kernels.cu", "fn_engine.cu", "fn_adjoint.cu", "fn_upload.cu", "fn_generate.cpp", "fn_io.cpp"]
HEADERS = ["fn_kernels.h", "fn_types.h", "fn_detmath.h", "fn_device.cuh", "fn_engine_internal.h",
           "fn_cli.cpp"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off",
    "-Xptxas", "-warn-spills",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(CLI):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps += [os.path.join(ROOT, "include", h) for h in ("fibrenet.h", "fibrenet_generate.h", "fibrenet_io.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, "-shared", "-o", LIB + ".tmp",
           *[os.path.join(CSRC, s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    out = subprocess.run(cmd, capture_output=True, text=True, cwd=CSRC)
    if out.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + out.stdout + out.stderr)
    os.replace(LIB + ".tmp", LIB)
    cli = [nvcc(), "-O2", "-std=c++17", "-o", CLI, os.path.join(CSRC, "fn_cli.cpp"), "-L", HERE,
           "-lfibrenet", "-Xlinker", "-rpath,$ORIGIN"]
    out = subprocess.run(cli, capture_output=True, text=True, cwd=CSRC)
    if out.returncode != 0:
        raise RuntimeError("building the command-line runner failed:\n" + out.stdout + out.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

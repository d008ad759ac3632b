"""In-tree build of the CUDA library (sm_100a) with nvcc."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRCS = [os.path.join(HERE, "csrc", f) for f in ("cfd_capi.cu", "cfd_noalloc.cu")]
DEPS = SRCS + [os.path.join(HERE, "csrc", f) for f in sorted(os.listdir(os.path.join(HERE, "csrc")))
               if f.endswith(".cuh")] + [os.path.join(os.path.dirname(HERE), "include", "cfd_b200.h")]
OUT = os.path.join(HERE, "_lib", "libcfdb200.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def nvcc() -> str:
    for p in (os.environ.get("CUDA_HOME", ""), "/usr/local/cuda"):
        cand = os.path.join(p, "bin", "nvcc") if p else ""
        if cand and os.path.exists(cand):
            return cand
    return "nvcc"


def build_library(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    stale = force or not os.path.exists(OUT) or \
        any(os.path.getmtime(d) > os.path.getmtime(OUT) for d in DEPS)
    if stale:
        cmd = [nvcc()] + NVCC_FLAGS + ["-o", OUT] + SRCS
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT

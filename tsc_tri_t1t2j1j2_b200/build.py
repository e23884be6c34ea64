"""Build the in-tree CUDA library libtscgpu.so for sm_100a with nvcc."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = ["tsc_kernels.cu", "tsc_host.cu", "tsc_hpsi.cu", "tsc_dmrg.cu", "tsc_capi.cu", "tsc_noalloc.cu", "tsc_split.cu", "tsc_blocksparse.cu", "tsc_measure.cu", "tsc_nullspace.cu", "tsc_checkpoint.cu", "tsc_correlate.cu"]
DEPS = SRC + ["tsc_kernels.cuh", "tsc_engine.hpp", "tsc_ctx.hpp"]
OUT = os.path.join(HERE, "_lib", "libtscgpu.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", "-diag-suppress", "177"]


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    hdr = os.path.join(HERE, os.pardir, "include", "tsc_gpu.h")
    return any(os.path.getmtime(os.path.join(HERE, "csrc", f)) > t for f in DEPS) or os.path.getmtime(hdr) > t


def build(force: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["nvcc", *NVCC_FLAGS, "-o", OUT, *[os.path.join(HERE, "csrc", f) for f in SRC], "-lcusolver", "-lcublas"]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))

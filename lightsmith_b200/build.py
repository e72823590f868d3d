"""Build ``liblsfdtd.so`` in-tree for sm_100a with nvcc (no GPU needed to build)."""

from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("lsfdtd.cu", "noalloc.cu", "voxel.cu")]
HEADERS = [os.path.join(HERE, "csrc", f) for f in ("common.cuh", "yee.cuh", "yee_vec.cuh", "fused.cuh",
                                                   "fused_tma.cuh", "fused_pml.cuh", "shell.cuh", "batch.cuh", "adjoint.cuh", "ade.cuh", "sources.cuh",
                                                   "monitors.cuh", "tensor.cuh")] + \
    [os.path.join(REPO, "include", "lsfdtd.h")]
OUT = os.path.join(HERE, "liblsfdtd.so")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "--threads", "0", "-Xcompiler", "-fPIC",
         "-shared", "-I" + os.path.join(REPO, "include")]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build lightsmith-b200")
    return path


def stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(p) > t for p in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the CUDA library if a source is newer than it; returns its path."""
    if force or stale():
        cmd = [nvcc(), *FLAGS, "-o", OUT, *SOURCES]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force=True, verbose=True)

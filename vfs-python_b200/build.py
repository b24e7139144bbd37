"""Builds libvfs_b200.so in place with nvcc for sm_100a.

    python vfs-python_b200/build.py [--debug]

The library is self-contained (CUDA runtime only, no torch) and exposes the C
ABI declared in include/vfs_b200.h.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "vfs_b200", "libvfs_b200.so")
SOURCES = ["vfs_capi.cu", "vfs_kernels.cu", "vfs_tgv.cu", "vfs_tgv_cluster.cu", "vfs_plan.cu", "vfs_batch.cu", "vfs_static.cu", "vfs_grad.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build(verbose: bool = False, extra=None) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    newest = max(os.path.getmtime(p) for p in srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
                 + [os.path.join(os.path.dirname(HERE), "include", "vfs_b200.h")])
    if os.path.exists(OUT) and os.path.getmtime(OUT) >= newest and not extra:
        return OUT
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-Xcompiler",
           "-fvisibility=hidden", "-Xptxas", "-v" if verbose else "-O3", "-o", OUT + ".tmp", *srcs,
           "-lcudart_static", "-lrt", "-ldl", "-lpthread"] + (extra or [])
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

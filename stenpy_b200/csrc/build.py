"""Build libstenpy_b200.so in-tree (nvcc, sm_100a).

    python -m stenpy_b200.csrc.build      # or stenpy_b200.csrc.build.build()

The library holds the C ABI (include/stenpy_b200.h): NVRTC compilation and launch
of the generated per-graph kernels, TMA descriptor encoding and the ahead-of-time
kernels (reduction finalize, cost-model MLP). It links NVRTC dynamically, the CUDA
runtime statically, and resolves the driver API at run time.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
REPO = os.path.dirname(PKG)
LIB = os.path.join(PKG, "libstenpy_b200.so")
SOURCES = ["stenpy_abi.cu", "noalloc.cu", "mlp_kernels.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _cuda_home() -> str:
    for cand in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if cand and os.path.exists(os.path.join(cand, "bin", "nvcc")):
            return cand
    nvcc = shutil.which("nvcc")
    if nvcc:
        return os.path.dirname(os.path.dirname(nvcc))
    raise RuntimeError("nvcc not found (set CUDA_HOME)")


def build(verbose: bool = False) -> str:
    cuda = _cuda_home()
    srcs = [os.path.join(HERE, s) for s in SOURCES if os.path.exists(os.path.join(HERE, s))]
    deps = srcs + [os.path.join(REPO, "include", "stenpy_b200.h")]
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    cmd = [os.path.join(cuda, "bin", "nvcc"), *ARCH, "-lineinfo", "-O3", "-std=c++17",
           "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
           "-I", os.path.join(cuda, "include"), "-I", os.path.join(REPO, "include"),
           *srcs, "-o", LIB + ".tmp",
           "-L", os.path.join(cuda, "lib64"), "-lnvrtc", "-ldl",
           "-Xlinker", "-rpath," + os.path.join(cuda, "lib64")]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
    sys.exit(0)

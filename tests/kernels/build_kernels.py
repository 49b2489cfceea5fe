"""Builds tests/kernels/_build/libpb2_test_kernels.so (the generic kernels of the accelerator tests) for sm_100a,
with the library's arithmetic flags (-fmad=false: every float operation one IEEE operation, as the oracle's)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libpb2_test_kernels.so")


def build() -> str:
    src = os.path.join(HERE, "generic_kernels.cu")
    hdr = os.path.join(HERE, "..", "..", "include", "piper2_b200_device.cuh")
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(src), os.path.getmtime(hdr)):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    nvcc = os.environ.get("NVCC") or ("/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc")
    cmd = [nvcc, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-fmad=false",
           "-Xcompiler", "-fPIC", "-shared", src, "-o", LIB]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("test kernels build failed:\n" + res.stdout + res.stderr)
    return LIB


if __name__ == "__main__":
    print(build())

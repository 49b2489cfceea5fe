"""Builds the CUDA library piper2_b200/_lib/libpiper2_b200.so for sm_100a.

Every translation unit is compiled with
    -gencode arch=compute_100a,code=sm_100a -lineinfo -O3 -fmad=false -Xcompiler -ffp-contract=off
-fmad=false keeps every float operation a single IEEE operation in source order (fused multiply-adds
are written out where wanted), and -ffp-contract=off does the same for host code (the flattening of instance
transforms), which is what makes device paths bit-identical to the CPU oracle.
The generated Sobol tables (piper2_b200/sobol_tables.py) are written to piper2_b200/_build/gen/.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
GEN = os.path.join(BUILD, "gen")
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "libpiper2_b200.so")
ROOT = os.path.dirname(HERE)

SOURCES = ["bvh_build.cu", "accelerator.cu", "traverse.cu", "render.cu", "capi.cu", "nalloc.cu", "guiding.cu", "guiding_tc.cu",
           "guiding_train_tc.cu", "materialize.cpp"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-fmad=false",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return res


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "piper2_b200.h"))
    hs.append(os.path.join(GEN, "sobol_tables.h"))
    return hs


def build(force: bool = False, verbose: bool = False) -> str:
    sys.path.insert(0, ROOT)
    from piper2_b200 import sobol_tables

    os.makedirs(GEN, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    sobol_tables.write_header(os.path.join(GEN, "sobol_tables.h"))
    headers = _headers()
    hdr_time = max(os.path.getmtime(h) for h in headers)
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(path), hdr_time):
            cmd = [_nvcc(), *NVCC_FLAGS, "-I", GEN, "-I", CSRC, "-c", path, "-o", obj]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            r = _run(cmd)
            if verbose:
                sys.stderr.write(r.stderr)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        # export only the C ABI: every pb2_* entry point is declared with default visibility below
        _run([_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB, *objs,
              "-Xlinker", f"--version-script={os.path.join(CSRC, 'exports.map')}"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

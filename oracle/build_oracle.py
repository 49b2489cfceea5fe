"""Builds the CPU oracle (test infrastructure only).

Outputs (git-ignored):
  oracle/_build/sobol_tables.h   generated Sobol tables (same generator as the product)
  oracle/_build/liboracle.so     the C restatement (pb2_oracle.c)
  oracle/_build/liboracle_fp64.so the same source built with -DOR_FP64: double-precision ground truth
  oracle/_ref/librefcpu.so       the reference's own device code compiled natively with a host shim,
                                 only when the reference sources are given (build_ref(reference_dir) or
                                 the PIPER2_REFERENCE variable; see oracle/ref/Makefile)

Flags: -O2 -ffp-contract=off, no -march=native and no fast-math, so every float operation is the one
written in the source.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")

CFLAGS = ["-std=c11", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-Wall",
          "-Wno-unused-function"]


def _run(cmd, cwd=None):
    res = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"command failed: {' '.join(cmd)}")
    return res


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def sobol_header() -> str:
    sys.path.insert(0, ROOT)
    from piper2_b200 import sobol_tables

    path = os.path.join(BUILD, "sobol_tables.h")
    sobol_tables.write_header(path)
    return path


def build_oracle(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    header = sobol_header()
    src = os.path.join(HERE, "pb2_oracle.c")
    out = os.path.join(BUILD, "liboracle.so")
    deps = [src, header, os.path.join(HERE, "pb2_oracle.h"),
            os.path.join(ROOT, "piper2_b200", "csrc", "pb2_math.h"),
            os.path.join(ROOT, "include", "piper2_b200.h")]
    if force or _stale(out, deps):
        _run(["gcc", *CFLAGS, "-I", BUILD, "-shared", "-o", out, src, "-lm"])
    out64 = os.path.join(BUILD, "liboracle_fp64.so")
    if force or _stale(out64, deps):
        _run(["gcc", *CFLAGS, "-DOR_FP64", "-I", BUILD, "-shared", "-o", out64, src, "-lm"])
    return out


def build_ref(reference_dir: str | None = None, force: bool = False) -> str | None:
    """Compile the reference's kernels + shim into oracle/_ref/librefcpu.so.  `reference_dir` (or the
    PIPER2_REFERENCE variable) is the root of a Piper2 checkout; without one, or if it holds no
    Src/BuiltinComponent, nothing is built and None is returned."""
    src = reference_dir or os.environ.get("PIPER2_REFERENCE")
    if not src or not os.path.isdir(os.path.join(src, "Src", "BuiltinComponent")):
        return None
    build_oracle()
    os.makedirs(REF_OUT, exist_ok=True)
    _run(["make", "-s", "-C", os.path.join(HERE, "ref"), f"REFERENCE={src}",
          f"OUT={REF_OUT}", f"ORACLE_BUILD={BUILD}"] + (["-B"] if force else []))
    return os.path.join(REF_OUT, "librefcpu.so")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(args[0] if args else None, force="--force" in sys.argv))

"""piper2_b200 -- B200-native path-tracing accelerator and tracer for Piper2.

The product is the CUDA library libpiper2_b200.so (C ABI in include/piper2_b200.h); this package holds
its build, the ctypes binding (capi), the host API (api) and the seeded workload generators (scenes).
"""
from . import capi, scenes  # noqa: F401

__all__ = ["capi", "scenes", "api", "build"]

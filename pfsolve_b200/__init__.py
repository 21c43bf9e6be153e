"""pfsolve_b200 -- B200-native Jones-Worland step (PfSolve JW path) for sm_100a.

The product is the C ABI library ``libpfsolve_b200.so`` (include/pfsolve_b200.h).
This package holds its sources (``csrc/``), the build recipe, a ctypes binding
and host-side helpers (synthetic workloads, band layouts) used by the tests and
the benchmark.
"""
from .capi import load as load_library  # noqa: F401

__all__ = ["load_library"]

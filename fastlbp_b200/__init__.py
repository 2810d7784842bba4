"""B200-native causal loopy belief propagation (drop-in for FastLBP's CausalBP: the PARALL
sweep, and the SEQFIX / TOPO schedules).

The product is the shared library libfastlbp_b200.so (CUDA sm_100a kernels,
the C ABI of include/fastlbp_b200.h and the libDAI-style C++ API of
include/ext/*.h). This package loads it with ctypes.
"""

from .api import (BatchEngine, CausalBP, CausalFactorGraph, Engine, PropertySet, SetsEngine, seq_batches,  # noqa: F401
                  update_seq)
from ._native import FlbpError, lib  # noqa: F401

__all__ = ["BatchEngine", "CausalBP", "CausalFactorGraph", "Engine", "PropertySet", "SetsEngine", "FlbpError", "lib",
           "seq_batches", "update_seq"]

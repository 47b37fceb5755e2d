"""moonlab_b200 -- a B200 (sm_100a) dense state-vector engine behind the
C API of tsotchke/moonlab's state-vector path.

The engine lives in libmoonlab_b200.so (hand-written CUDA kernels plus a
C++ host runtime, C ABI in include/moonlab_b200.h).  This package is its
Python binding; it computes nothing itself.
"""
from ._lib import LIB_PATH, MlbError, exported_symbols, kernel_launches, load  # noqa: F401
from .statevector import StateVector, gates_to_ops  # noqa: F401

__all__ = ["StateVector", "gates_to_ops", "load", "LIB_PATH", "MlbError", "exported_symbols",
           "kernel_launches"]

"""B200-native batched tridiagonal solver (drop-in for the reference's
PaScaLTDMACUDA / FilteredTDMACUDA / TdmaBackendGPU).

The solve runs in hand-written sm_100a CUDA kernels behind the C ABI of
include/btdma.h (libbtdma.so, built in-tree by ``python -m
filtered_tdma_b200.build``).  There is no CPU implementation: if the library is
missing, the first solver construction raises.
"""
from ._lib import BtdmaError, LIB_PATH  # noqa: F401
from .solver import (FilteredTDMACUDA, PaScaLTDMACUDA, Solver,  # noqa: F401
                     TdmaBackendGPU)

__all__ = ["Solver", "PaScaLTDMACUDA", "FilteredTDMACUDA", "TdmaBackendGPU", "BtdmaError",
           "LIB_PATH"]

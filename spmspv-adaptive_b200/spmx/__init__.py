"""spmx — B200-native adaptive SpMV / SpMSpV engine (host side).

The compute path is libspmx.so (hand-written sm_100a CUDA kernels behind the C
ABI in include/spmx.h); this package binds it with ctypes and mirrors the
reference's SpmspvHandle.  Importing it without the built library fails.
"""
from ._lib import (SpmxError, declared_symbols, last_error, KERNEL_NAMES, FEATURE_NAMES,
                   NUM_KERNELS, NUM_FEATURES, LIB_PATH)
from . import _lib as abi
from . import gen

__all__ = ["SpmxError", "declared_symbols", "last_error", "KERNEL_NAMES", "FEATURE_NAMES",
           "NUM_KERNELS", "NUM_FEATURES", "LIB_PATH", "abi", "gen", "SpmspvHandle"]


def __getattr__(name):
    # torch is imported lazily so the generators and the ABI load without it
    if name == "SpmspvHandle":
        from .handle import SpmspvHandle
        return SpmspvHandle
    raise AttributeError(name)

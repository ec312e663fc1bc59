"""Python entry to the CUDA engine (``libgrpp_b200/libgrpp_b200.so``).

The engine library exports libgrpp's C API plus the batched entry points of
``include/libgrpp_b200.h``; this module only locates and loads it. There is no
CPU fallback: if the library is missing, loading fails.
"""
from __future__ import annotations

import os

from .capi import PRODUCT_LIB, LibGRPP

_LIB = None


def load() -> LibGRPP:
    global _LIB
    if _LIB is None:
        if not os.path.exists(PRODUCT_LIB):
            raise RuntimeError(f"{PRODUCT_LIB} is not built (python -m libgrpp_b200.build)")
        _LIB = LibGRPP(PRODUCT_LIB)
    return _LIB


def full_grpp_batch(batch, radial_mode: int = 0):
    """(arep, so_x, so_y, so_z) per-task blocks of a BatchArrays, on the current CUDA device."""
    return load().full_grpp_batch(batch, radial_mode)

"""ctypes loader of the reference's own GPU scan kernel (oracle/_ref/
libbnref_gpu.so, built by `make -C oracle ref` from the reference source
scorer-bntm/src/gpu/kernels.cu:100-178 for sm_100a).

TEST AND MEASUREMENT INFRASTRUCTURE ONLY: the bar the product's scan is
timed against in bench.py, and checked against the oracle in tests/.  The
product never loads it."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libbnref_gpu.so")


def load():
    """The library, or None when it was not built (no reference checkout at
    build time)."""
    if not os.path.exists(LIB_PATH):
        return None
    lib = C.CDLL(LIB_PATH)
    lib.bnref_compute_products.restype = C.c_int
    lib.bnref_compute_products.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    return lib

"""Loading of the package's native libraries (built in-tree by build.py).

The numeric phase has no CPU fallback: when ``libsdsb200.so`` is missing or a
CUDA device is absent, every entry point raises instead of computing
elsewhere.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ANALYSIS_SO = os.path.join(PKG, "libsdsb200_analysis.so")
NUMERIC_SO = os.path.join(PKG, "libsdsb200.so")

_analysis = None
_numeric = None


class NativeLibraryMissing(RuntimeError):
    pass


def analysis_lib():
    global _analysis
    if _analysis is None:
        if not os.path.exists(ANALYSIS_SO):
            raise NativeLibraryMissing(f"{ANALYSIS_SO} is not built (run sparsedirectsolver.jl_b200/build.py)")
        lib = C.CDLL(ANALYSIS_SO)
        lib.sdsa_default_options.argtypes = [C.c_void_p, C.c_int]
        lib.sdsa_default_options.restype = None
        lib.sdsa_analyze.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.sdsa_analyze.restype = C.c_int
        lib.sdsa_len.argtypes = [C.c_void_p, C.c_char_p]
        lib.sdsa_len.restype = C.c_int64
        lib.sdsa_get.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        lib.sdsa_get.restype = C.c_int
        lib.sdsa_stat.argtypes = [C.c_void_p, C.c_char_p]
        lib.sdsa_stat.restype = C.c_double
        lib.sdsa_free.argtypes = [C.c_void_p]
        lib.sdsa_free.restype = None
        lib.sdsa_last_error.argtypes = []
        lib.sdsa_last_error.restype = C.c_char_p
        lib.sdsa_matching.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.sdsa_matching.restype = C.c_int
        lib.sdsa_matching_pairs.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_void_p,
                                            C.c_void_p]
        lib.sdsa_matching_pairs.restype = C.c_int
        _analysis = lib
    return _analysis


def numeric_lib():
    """The CUDA numeric phase; raises when it is not built (no fallback)."""
    global _numeric
    if _numeric is None:
        if not os.path.exists(NUMERIC_SO):
            raise NativeLibraryMissing(f"{NUMERIC_SO} is not built (run sparsedirectsolver.jl_b200/build.py)")
        from . import capi
        _numeric = capi.bind(C.CDLL(NUMERIC_SO))
    return _numeric

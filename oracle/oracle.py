"""ctypes binding of the CPU oracle (liboracle.so). TEST INFRASTRUCTURE ONLY.

The oracle restates the reference's CPU reference factorizations and solves
(SparseDirectSolver.jl src/reference/cholesky.jl, ldlt.jl, lu.jl); see
oracle.h. Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline leg import this module, as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "oracle.cpp")
    if force or not os.path.exists(LIB) or os.path.getmtime(src) > os.path.getmtime(LIB) or \
            os.path.getmtime(os.path.join(HERE, "oracle.h")) > os.path.getmtime(LIB):
        subprocess.check_call(["make", "-C", HERE, "-B" if force else "liboracle.so"])
    from .blas_port import build as build_blas_port   # the benchmark's CPU-baseline port

    build_blas_port(force)
    return LIB


class _Sym(C.Structure):
    _fields_ = [("n", C.c_int64), ("ns", C.c_int64), ("nnz", C.c_int64)] + [
        (nm, C.POINTER(C.c_int64)) for nm in (
            "perm", "super_ptr", "snparent", "snpost", "rowptr", "rowval", "front_ptr", "child_ptr", "child_list",
            "relind_ptr", "relind", "amap", "amap_ptr", "amap_src")] + [("schur", C.c_int64)]


def _load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(LIB)
        lib.oracle_factor.restype = C.c_int64
        lib.oracle_factor.argtypes = [C.POINTER(_Sym), C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double,
                                      C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p]
        lib.oracle_set_threads.restype = None
        lib.oracle_set_threads.argtypes = [C.c_int]
        lib.oracle_solve.restype = C.c_int
        lib.oracle_solve.argtypes = [C.POINTER(_Sym), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int]
        _lib = lib
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Oracle:
    """Factor and solve with the CPU oracle on the maps of one analysis.

    ``sym`` is an object with int64 numpy fields named as the reference's
    ``Symbolic`` maps (1-based), e.g. ``sdsb200.analysis.Symbolic``.
    """

    STRUCT = {"G": 0, "S": 1, "SPD": 3}

    def __init__(self, sym):
        self.sym = sym
        self._keep = {}
        fields = {}
        for nm in ("perm", "super_ptr", "snparent", "snpost", "rowptr", "rowval", "front_ptr", "child_ptr",
                   "child_list", "relind_ptr", "relind", "amap", "amap_ptr", "amap_src"):
            a = np.ascontiguousarray(getattr(sym, nm), dtype=np.int64)
            if a.size == 0:
                a = np.zeros(1, np.int64)
            self._keep[nm] = a
            fields[nm] = a.ctypes.data_as(C.POINTER(C.c_int64))
        self._s = _Sym(n=sym.n, ns=sym.ns, nnz=sym.nnz, schur=int(getattr(sym, "schur", 0)), **fields)
        self.factor = self.ufactor = self.d = self.piv = self.kind = self.stats = None
        self.structure = None

    def factorize(self, nzval, structure="SPD", pivot_type=0, pivot_threshold=0.01, pivot_epsilon=None,
                  eps_scaled=False, pivot_sign=None):
        lib = _load()
        sym = self.sym
        nz = np.ascontiguousarray(nzval, dtype=np.float64)
        assert nz.size == sym.nnz
        flen = int(sym.front_ptr[-1] - 1)
        self.factor = np.zeros(max(flen, 1))
        self.ufactor = np.zeros(max(flen, 1))
        self.d = np.zeros(max(2 * sym.n, 1))
        self.piv = np.zeros(max(sym.n, 1), np.int32)
        self.kind = np.zeros(max(sym.n, 1), np.int8)
        self.stats = np.zeros(max(6 * sym.ns, 1), np.int64)
        if pivot_epsilon is None:
            pivot_epsilon = 1e-13
        ps = None if pivot_sign is None else np.ascontiguousarray(pivot_sign, dtype=np.int8)
        info = lib.oracle_factor(C.byref(self._s), _ptr(nz), self.STRUCT[structure], int(pivot_type),
                                 float(pivot_threshold), float(pivot_epsilon), int(bool(eps_scaled)), _ptr(ps),
                                 _ptr(self.factor), _ptr(self.ufactor), _ptr(self.d), _ptr(self.piv),
                                 _ptr(self.kind), _ptr(self.stats))
        if info < 0:
            raise ValueError("oracle_factor rejected its input")
        self.structure = structure
        return int(info)

    def solve(self, B, transpose=False):
        lib = _load()
        B = np.asarray(B, dtype=np.float64)
        vec = B.ndim == 1
        Bm = np.asfortranarray(B.reshape(self.sym.n, -1))
        X = np.zeros_like(Bm, order="F")
        rc = lib.oracle_solve(C.byref(self._s), self.STRUCT[self.structure], _ptr(self.factor), _ptr(self.ufactor),
                              _ptr(self.d), _ptr(self.piv), _ptr(self.kind), _ptr(X), _ptr(Bm), Bm.shape[1],
                              int(bool(transpose)))
        if rc != 0:
            raise ValueError("oracle_solve rejected its input")
        return X.reshape(-1) if vec else X

    def stats_matrix(self):
        return self.stats[: 6 * self.sym.ns].reshape(self.sym.ns, 6)


def set_threads(n: int) -> None:
    """Host threads of the factorizations (1: the reference's serial postorder; more: the fronts of one
    elimination-tree level concurrently, with the same results)."""
    _load().oracle_set_threads(int(n))


"""The reference's CPU Cholesky path over threaded LAPACK/BLAS -- TEST INFRASTRUCTURE ONLY.

``ref_factorize!`` (SparseDirectSolver.jl src/reference/cholesky.jl:44-111) factors each front with
``LAPACK.potrf!``, ``BLAS.trsm!`` and ``BLAS.syrk!`` on dense column-major fronts, in postorder,
after assembling A and extend-adding the children's contribution blocks. Its solve
(src/reference/cholesky.jl:127-170) runs the supernodal forward and backward sweeps. This module
restates that path on scipy's LAPACK/BLAS (OpenBLAS, multithreaded), so that the benchmark's CPU
baseline runs the reference's CPU algorithm with all the host threads it can use.

Only the benchmark's CPU-baseline leg and its reference arm use it. The parity checks use the
bit-exact scalar oracle (oracle.cpp), whose loops follow the same order without BLAS blocking.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
EXT = os.path.join(HERE, "blas_port_ext" + sysconfig.get_config_var("EXT_SUFFIX"))


def build(force: bool = False) -> str:
    """Compile the front loop (blas_port_ext.pyx, Cython over scipy's BLAS/LAPACK) beside this file."""
    src = os.path.join(HERE, "blas_port_ext.pyx")
    if not force and os.path.exists(EXT) and os.path.getmtime(EXT) >= os.path.getmtime(src):
        return EXT
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    csrc = os.path.join(bdir, "blas_port_ext.c")
    subprocess.check_call([sys.executable, "-m", "cython", "-3", src, "-o", csrc])
    subprocess.check_call(["gcc", "-O2", "-shared", "-fPIC", "-I", sysconfig.get_paths()["include"], csrc,
                           "-o", EXT])
    return EXT


def _ext():
    if HERE not in sys.path:
        sys.path.insert(0, HERE)
    import blas_port_ext

    return blas_port_ext


def blas_threads() -> int:
    """The threads the BLAS library uses (threadpoolctl when present, else the host's CPUs)."""
    try:
        from threadpoolctl import threadpool_info

        n = [d.get("num_threads", 0) for d in threadpool_info() if d.get("user_api") == "blas"]
        if n:
            return int(max(n))
    except Exception:
        pass
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


class CholeskyPort:
    """Multifrontal Cholesky and solve of one analysis (the maps of ``sdsb200.analysis.Symbolic``,
    1-based as the reference's). The flat 0-based index arrays are built once, from the maps."""

    def __init__(self, sym):
        m = sym.maps
        i64 = np.int64
        self.n, self.ns = int(sym.n), int(sym.ns)
        self.perm0 = np.asarray(m["perm"], i64) - 1
        sp, rp = np.asarray(m["super_ptr"], i64), np.asarray(m["rowptr"], i64)
        self.c0 = np.ascontiguousarray(sp[:-1] - 1)
        self.w = np.ascontiguousarray(np.diff(sp))
        self.f = np.ascontiguousarray(np.diff(rp))
        self.base = np.ascontiguousarray(np.asarray(m["front_ptr"], i64)[:-1] - 1)
        self.flen = int(m["front_ptr"][-1] - 1)
        self.post = np.ascontiguousarray(np.asarray(m["snpost"], i64) - 1)
        self.parent = np.ascontiguousarray(np.asarray(m["snparent"], i64) - 1)
        self.rowptr = np.ascontiguousarray(rp - 1)
        self.rowval = np.ascontiguousarray(np.asarray(m["rowval"], i64) - 1)
        amap, aptr = np.asarray(m["amap"], i64), np.asarray(m["amap_ptr"], i64) - 1
        self.aptr = np.ascontiguousarray(aptr)
        self.asrc = np.ascontiguousarray(np.asarray(m["amap_src"], i64) - 1)
        fr_of = np.repeat(np.arange(self.ns), np.diff(aptr))
        loc = np.abs(amap[self.asrc]) - 1 - self.base[fr_of]
        self.ai = np.ascontiguousarray(loc % self.f[fr_of])
        self.aj = np.ascontiguousarray(loc // self.f[fr_of])
        self.cptr = np.ascontiguousarray(np.asarray(m["child_ptr"], i64) - 1)
        self.clist = np.ascontiguousarray(np.asarray(m["child_list"], i64) - 1)
        self.rptr = np.ascontiguousarray(np.asarray(m["relind_ptr"], i64) - 1)
        self.rind = np.ascontiguousarray(np.asarray(m["relind"], i64) - 1)
        self.factor = np.zeros(max(self.flen, 1))
        self._ext = _ext()

    def factorize(self, nzval) -> int:
        """Returns 0, or the original column (1-based) of the first failed pivot."""
        nz = np.ascontiguousarray(nzval, dtype=np.float64)
        r = self._ext.factorize(self.post, self.parent, self.f, self.w, self.base, self.aptr, self.ai, self.aj,
                                self.asrc, self.cptr, self.clist, self.rptr, self.rind, nz, self.factor)
        if r < 0:
            return 0
        s, col = r % self.ns, r // self.ns
        return int(self.perm0[self.c0[s] + col] + 1)

    def solve(self, B):
        """X = A^{-1} B with the last factorization (supernodal sweeps, src/reference/cholesky.jl:127-170)."""
        B = np.asarray(B, dtype=np.float64)
        vec = B.ndim == 1
        Y = np.asfortranarray(B.reshape(self.n, -1)[self.perm0])
        self._ext.solve(self.post, self.f, self.w, self.base, self.c0, self.rowptr, self.rowval, self.factor, Y)
        X = np.empty_like(Y)
        X[self.perm0] = Y
        return X[:, 0] if vec else X

"""Shared helpers of the tests: generators, oracle runs, comparisons."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from sdsb200 import analyze_csr
from sdsb200 import matrices as M


def oracle_for(A, structure, **kw):
    """Analysis + CPU oracle factorization on the same Symbolic."""
    from oracle.oracle import Oracle

    fkw = {k: kw.pop(k) for k in list(kw) if k in ("pivot_type", "pivot_threshold", "pivot_epsilon", "eps_scaled",
                                                   "pivot_sign")}
    S = analyze_csr(A, structure, **kw)
    O = Oracle(S)
    info = O.factorize(A.data, structure, **fkw)
    return S, O, info


def eigen_inertia(A):
    ev = np.linalg.eigvalsh(A.toarray())
    return int((ev > 0).sum()), int((ev < 0).sum())


def small_kkt(nx=20, ny=20, nj=150, seed=0, delta=0.0):
    return M.kkt(nx, ny, nj, delta=delta, seed=seed)


def dense_panels(S, factor):
    """The stored lower trapezoid of every panel, concatenated (the comparable part of the factor)."""
    out = []
    for s in range(S.ns):
        f, w, base = int(S.front_nrows[s]), int(S.front_ncols[s]), int(S.front_ptr[s]) - 1
        P = factor[base: base + f * w].reshape(w, f).T
        out.append(np.concatenate([P[j:, j] for j in range(w)]))
    return np.concatenate(out) if out else np.zeros(0)


def rel_max_diff(a, b):
    scale = max(1.0, float(np.abs(b).max(initial=0.0)))
    return float(np.abs(a - b).max(initial=0.0)) / scale

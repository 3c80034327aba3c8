"""Host analysis: CSR pattern -> the reference's ``Symbolic`` maps.

Thin ctypes layer over ``libsdsb200_analysis.so`` (include/sdsb200_analysis.h),
which restates the reference's ``symbolic_analysis``
(SparseDirectSolver.jl src/symbolic/maps.jl:255-268).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from ._native import analysis_lib

STRUCTURES = {"G": 0, "S": 1, "SPD": 3}
REORDERING = {"default": 0, "algo1": 1, "algo2": 1, "algo3": 1, "amd": 1, "algo4": 2, "nd": 2, "algo5": 3,
              "natural": 3}
PAIRS = {"none": 0, "default": 1, "all": 2}

MAP_NAMES = ("perm", "iperm", "super_ptr", "snparent", "snpost", "rowptr", "rowval", "front_ptr", "front_nrows",
             "front_ncols", "child_ptr", "child_list", "relind_ptr", "relind", "amap", "amap_ptr", "amap_src",
             "counts", "pairs", "full_rowptr", "full_colval", "full_srcptr", "full_src", "full_conj",
             "schur_rowptr", "schur_colval", "ordering")


class _Opts(C.Structure):
    _fields_ = [("structure", C.c_int), ("view", C.c_int), ("index_base", C.c_int), ("reordering", C.c_int),
                ("user_perm", C.POINTER(C.c_int64)), ("pivot_pairs", C.c_int),
                ("pivot_pair_tolerance", C.c_double), ("pivot_threshold", C.c_double),
                ("use_superpanels", C.c_int), ("amalg_max_width", C.c_int), ("amalg_zero_fraction", C.c_double),
                ("amalg_min_width", C.c_int), ("user_pairs", C.c_void_p), ("n_user_pairs", C.c_int64),
                ("user_schur_indices", C.c_void_p)]


@dataclass
class Symbolic:
    """The reference's ``Symbolic`` (src/symbolic/maps.jl:62-95): 1-based int64 maps.

    Field names follow ``DEVICE_MAPS`` (maps.jl:16-18); ``snpost``, ``counts``,
    ``pairs`` and the ``full_*`` residual map are the host-side extras. Schur
    complement mode: ``schur`` is the root supernode that is assembled and not
    factored (``schedule.schur``, 1-based; 0 = none), ``schur_n`` its order, and
    ``schur_rowptr``/``schur_colval`` the 1-based CSR pattern of S
    (``schur_pattern``, src/symbolic/ordering.jl:424-470).
    """

    n: int
    nnz: int
    ns: int
    structure: str
    view: str
    index_base: int
    nnz_stored: int
    nnz_L: int
    flops: float
    sdepth: int
    alg_used: int
    maps: dict = field(default_factory=dict)
    schur: int = 0
    schur_n: int = 0

    def __getattr__(self, name):
        maps = self.__dict__.get("maps")
        if maps is not None and name in maps:
            return maps[name]
        raise AttributeError(name)

    @property
    def factor_len(self) -> int:
        return int(self.front_ptr[-1] - 1) if self.ns > 0 else 0


def analyze(rowptr, colval, n, structure="SPD", nzval=None, view="F", index_base=0, reordering="default",
            user_perm=None, pivot_pairs="default", pivot_pair_tolerance=1e-6, pivot_threshold=0.01,
            use_superpanels=1, amalgamation=(32, 0.25, 8), user_pairs=None, user_schur_indices=None) -> Symbolic:
    """Analyse the pattern of an ``n x n`` CSR matrix (``index_base`` of its arrays).

    ``user_schur_indices`` (n flags 0/1, or None): Schur complement mode, the flagged rows and columns
    ordered last as one unfactored root supernode (compute_schur_ordering and
    schur_supernode_partition, src/symbolic/ordering.jl:386-415, src/symbolic/supernodes.jl:391-425)."""
    lib = analysis_lib()
    rp = np.ascontiguousarray(rowptr, dtype=np.int64)
    cv = np.ascontiguousarray(colval, dtype=np.int64)
    if rp.size != n + 1:
        raise ValueError(f"rowptr has {rp.size} entries, expected n + 1 = {n + 1}")
    nz = None if nzval is None else np.ascontiguousarray(np.asarray(nzval, dtype=np.float64).reshape(-1)[: cv.size])
    up = None if user_perm is None else np.ascontiguousarray(user_perm, dtype=np.int64)
    o = _Opts()
    lib.sdsa_default_options(C.byref(o), STRUCTURES[structure])
    o.view = ord(view)
    o.index_base = int(index_base)
    o.reordering = REORDERING[reordering]
    o.user_perm = up.ctypes.data_as(C.POINTER(C.c_int64)) if up is not None else None
    o.pivot_pairs = PAIRS[pivot_pairs]
    o.pivot_pair_tolerance = pivot_pair_tolerance
    o.pivot_threshold = pivot_threshold
    o.use_superpanels = int(use_superpanels)
    o.amalg_max_width, o.amalg_zero_fraction, o.amalg_min_width = amalgamation
    upairs = None
    if user_pairs is not None and len(user_pairs) > 0:
        upairs = np.ascontiguousarray(np.asarray(user_pairs, dtype=np.int64).reshape(-1, 2))
        o.user_pairs = upairs.ctypes.data
        o.n_user_pairs = upairs.shape[0]
    flags = None
    if user_schur_indices is not None:
        flags = np.ascontiguousarray(np.asarray(user_schur_indices).reshape(-1) != 0, dtype=np.int8)
        if flags.size != n:
            raise ValueError(f"user_schur_indices has {flags.size} entries, the matrix has {n} rows")
        o.user_schur_indices = flags.ctypes.data
    res = C.c_void_p()
    rc = lib.sdsa_analyze(C.c_int64(n), rp.ctypes.data_as(C.c_void_p), cv.ctypes.data_as(C.c_void_p),
                          nz.ctypes.data_as(C.c_void_p) if nz is not None else None, C.byref(o), C.byref(res))
    if rc != 0:
        raise ValueError("analysis failed: " + lib.sdsa_last_error().decode())
    try:
        maps = {}
        for nm in MAP_NAMES:
            ln = lib.sdsa_len(res, nm.encode())
            a = np.zeros(max(ln, 0), dtype=np.int64)
            if ln > 0:
                lib.sdsa_get(res, nm.encode(), a.ctypes.data_as(C.c_void_p))
            maps[nm] = a
        st = lambda k: lib.sdsa_stat(res, k.encode())  # noqa: E731
        return Symbolic(n=int(n), nnz=int(cv.size), ns=int(st("ns")), structure=structure, view=view,
                        index_base=int(index_base), nnz_stored=int(st("nnz_stored")), nnz_L=int(st("nnz_L")),
                        flops=float(st("flops")), sdepth=int(st("sdepth")), alg_used=int(st("alg_used")),
                        maps=maps, schur=int(st("schur")), schur_n=int(st("schur_n")))
    finally:
        lib.sdsa_free(res)


def analyze_csr(A, structure="SPD", **kw) -> Symbolic:
    """``analyze`` for a scipy CSR matrix (0-based arrays)."""
    return analyze(A.indptr, A.indices, A.shape[0], structure, nzval=A.data, index_base=0, **kw)


MATCHING_JOBS = {"algo1": 1, "algo2": 2, "algo3": 3, "algo4": 4, "algo5": 5, "algo6": 6}


@dataclass
class Matching:
    """Result of :func:`compute_matching`, the reference's ``Matching`` (src/matching/mc64.jl:18-45).

    ``perm[i]`` is the 1-based column matched to row ``i`` (``"perm_matching"``), ``matched[i]`` whether
    row ``i`` has a matched entry, ``rscale``/``cscale`` the row and column scalings (``"scale_row"``,
    ``"scale_col"``; ones for jobs 1-4, equal for the symmetric structures, whose factored matrix
    would be ``D A D``)."""

    job: int
    perm: np.ndarray
    matched: np.ndarray
    rscale: np.ndarray
    cscale: np.ndarray
    symmetric: bool


def compute_matching(rowptr, colval, nzval, n, structure="G", matching_alg="algo5", view="F",
                     index_base=0) -> Matching:
    """MC64 matching and scaling of an ``n x n`` CSR matrix from its values (``compute_matching``,
    src/matching/mc64.jl:378-398): ``matching_alg`` ``"algo1"``-``"algo6"`` (or 1-6) is the MC64 job.
    ``"G"`` matches the stored rows; ``"S"``/``"SPD"`` the full matrix read from ``view``'s triangle,
    with the symmetric scaling ``d = sqrt(r c)``."""
    lib = analysis_lib()
    job = MATCHING_JOBS[matching_alg] if isinstance(matching_alg, str) else int(matching_alg)
    rp = np.ascontiguousarray(rowptr, dtype=np.int64)
    cv = np.ascontiguousarray(colval, dtype=np.int64)
    if rp.size != n + 1:
        raise ValueError(f"rowptr has {rp.size} entries, expected n + 1 = {n + 1}")
    nz = np.ascontiguousarray(np.asarray(nzval, dtype=np.float64).reshape(-1)[: cv.size])
    perm = np.zeros(max(n, 1), np.int64)
    matched = np.zeros(max(n, 1), np.int8)
    rs = np.ones(max(n, 1))
    cs = np.ones(max(n, 1))
    rc = lib.sdsa_matching(C.c_int64(n), rp.ctypes.data_as(C.c_void_p), cv.ctypes.data_as(C.c_void_p),
                           nz.ctypes.data_as(C.c_void_p), STRUCTURES[structure], ord(view), int(index_base), job,
                           perm.ctypes.data_as(C.c_void_p), matched.ctypes.data_as(C.c_void_p),
                           rs.ctypes.data_as(C.c_void_p), cs.ctypes.data_as(C.c_void_p))
    if rc != 0:
        raise ValueError("matching failed: " + lib.sdsa_last_error().decode())
    return Matching(job=5 if job == 6 else job, perm=perm[:n], matched=matched[:n].astype(bool), rscale=rs[:n],
                    cscale=cs[:n], symmetric=structure != "G")


def matching_pairs(rowptr, colval, nzval, n, m: Matching, pivot_pairs="default", pivot_pair_tolerance=1e-6,
                   view="F", index_base=0) -> np.ndarray:
    """The 2x2 pivot pairs of ``"S"`` from the cycles of the symmetric matching ``m`` (the reference's
    ``matching_pairs``, src/matching/mc64.jl:380-441): an array of 1-based (partner, candidate) rows,
    sorted by candidate, for ``analyze(..., user_pairs=...)``."""
    lib = analysis_lib()
    rp = np.ascontiguousarray(rowptr, dtype=np.int64)
    cv = np.ascontiguousarray(colval, dtype=np.int64)
    nz = np.ascontiguousarray(np.asarray(nzval, dtype=np.float64).reshape(-1)[: cv.size])
    perm = np.ascontiguousarray(m.perm, dtype=np.int64)
    matched = np.ascontiguousarray(m.matched, dtype=np.int8)
    d = np.ascontiguousarray(m.rscale, dtype=np.float64)
    out = np.zeros(max(n, 2), np.int64)
    cnt = C.c_int64(0)
    rc = lib.sdsa_matching_pairs(C.c_int64(n), rp.ctypes.data_as(C.c_void_p), cv.ctypes.data_as(C.c_void_p),
                                 nz.ctypes.data_as(C.c_void_p), ord(view), int(index_base),
                                 perm.ctypes.data_as(C.c_void_p), matched.ctypes.data_as(C.c_void_p),
                                 d.ctypes.data_as(C.c_void_p), PAIRS[pivot_pairs], float(pivot_pair_tolerance),
                                 out.ctypes.data_as(C.c_void_p), C.byref(cnt))
    if rc != 0:
        raise ValueError("matching pairs failed: " + lib.sdsa_last_error().decode())
    return out[: 2 * cnt.value].reshape(-1, 2).copy()


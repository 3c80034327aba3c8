"""Host analysis invariants (CPU): the Symbolic maps restated from the reference.

Mirrors the reference's symbolic tests (test/test_symbolic_*.jl, brute-force
symbolic factorization test/utils.jl:182-207): the supernodal row structure
holds the filled pattern, the assembly map puts every entry of A at its place
in the panels, the extend-add maps are consistent, and 2x2 pairs are
eliminated together.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from sdsb200 import analyze_csr
from sdsb200 import matrices as M


def filled_pattern(A, p):
    """Brute-force symbolic Cholesky of A[p, p] (boolean elimination)."""
    B = (A.toarray()[np.ix_(p, p)] != 0) | np.eye(A.shape[0], dtype=bool)
    B = B | B.T
    n = B.shape[0]
    L = np.tril(B)
    for k in range(n):
        rows = np.nonzero(L[k + 1:, k])[0] + k + 1
        for i in rows:
            L[rows[rows >= i], i] = True
    return L


@pytest.mark.parametrize("structure,gen", [("SPD", lambda: M.lap2d_shifted(9, 7)),
                                           ("G", lambda: M.convection_diffusion3d(4, 5, 3)),
                                           ("S", lambda: M.kkt(6, 6, 15, seed=1))])
@pytest.mark.parametrize("reordering", ["amd", "nd", "natural"])
def test_supernodal_structure_holds_fill(structure, gen, reordering):
    A = gen()
    S = analyze_csr(A, structure, reordering=reordering)
    n = S.n
    assert sorted(S.perm) == list(range(1, n + 1))
    p = S.perm - 1
    pat = A if structure != "G" else (abs(A) + abs(A.T)).tocsr()
    if structure == "S" and S.pairs.size:
        # pair_pattern (src/symbolic/pairs.jl:450-466): the expansion of the graph compressed by the pairs
        group = np.arange(n)
        for a, c in S.pairs.reshape(-1, 2):
            group[c - 1] = group[a - 1]
        D = (pat.toarray() != 0)
        G = np.zeros((n, n), dtype=bool)
        G[np.ix_(group, group)] |= False
        gi, gj = np.nonzero(D)
        Gc = np.zeros((n, n), dtype=bool)
        Gc[group[gi], group[gj]] = True
        pat = sp.csr_matrix(Gc[np.ix_(group, group)].astype(float))
    Lf = filled_pattern(pat, p)
    stored = np.zeros_like(Lf)
    for s in range(S.ns):
        rows = S.rowval[S.rowptr[s] - 1: S.rowptr[s + 1] - 1] - 1
        cols = range(S.super_ptr[s] - 1, S.super_ptr[s + 1] - 1)
        assert list(rows[: len(cols)]) == list(cols)
        assert np.all(np.diff(rows) > 0)
        for j, c in enumerate(cols):
            stored[rows[j:], c] = True
    assert not np.any(Lf & ~stored)
    assert S.nnz_L == int(Lf.sum())
    assert S.nnz_stored >= S.nnz_L


@pytest.mark.parametrize("structure", ["SPD", "G"])
def test_assembly_map_places_every_entry(structure):
    A = M.lap2d_shifted(8, 8) if structure == "SPD" else M.convection_diffusion3d(4, 4, 4)
    S = analyze_csr(A, structure)
    n = S.n
    iperm = np.empty(n, np.int64)
    iperm[S.perm - 1] = np.arange(n)
    Lbuf = np.zeros(S.factor_len)
    Ubuf = np.zeros(S.factor_len)
    for p, off in enumerate(S.amap):
        if off > 0:
            Lbuf[off - 1] += A.data[p]
        elif off < 0:
            Ubuf[-off - 1] += A.data[p]
    Ap = A.toarray()[np.ix_(S.perm - 1, S.perm - 1)]
    for s in range(S.ns):
        f, w, base = int(S.front_nrows[s]), int(S.front_ncols[s]), int(S.front_ptr[s]) - 1
        rows = S.rowval[S.rowptr[s] - 1: S.rowptr[s + 1] - 1] - 1
        c0 = int(S.super_ptr[s]) - 1
        for j in range(w):
            for i in range(j, f):
                assert Lbuf[base + j * f + i] == Ap[rows[i], c0 + j]
                if structure == "G" and i > j:
                    assert Ubuf[base + j * f + i] == Ap[c0 + j, rows[i]]
    # grouping: sorted by destination, grouped by supernode
    for s in range(S.ns):
        src = S.amap_src[S.amap_ptr[s] - 1: S.amap_ptr[s + 1] - 1] - 1
        offs = np.abs(S.amap[src])
        assert np.all(np.diff(offs) >= 0)
        assert np.all((offs >= S.front_ptr[s]) & (offs < S.front_ptr[s + 1]))


def test_relind_and_children():
    A = M.lap3d(6, 6, 6)
    S = analyze_csr(A, "SPD", reordering="nd")
    for c in range(S.ns):
        par = S.snparent[c]
        ri = S.relind[S.relind_ptr[c] - 1: S.relind_ptr[c + 1] - 1]
        if par == 0:
            assert ri.size == 0
            continue
        assert par - 1 > c
        rows_c = S.rowval[S.rowptr[c] - 1: S.rowptr[c + 1] - 1]
        rows_p = S.rowval[S.rowptr[par - 1] - 1: S.rowptr[par] - 1]
        w = S.super_ptr[c + 1] - S.super_ptr[c]
        assert np.array_equal(rows_p[ri - 1], rows_c[w:])
        kids = S.child_list[S.child_ptr[par - 1] - 1: S.child_ptr[par] - 1]
        assert c + 1 in kids and np.all(np.diff(kids) > 0)


def test_orderings_reduce_fill():
    A = M.lap2d_shifted(30, 30)
    nat = analyze_csr(A, "SPD", reordering="natural")
    amd = analyze_csr(A, "SPD", reordering="amd")
    nd = analyze_csr(A, "SPD", reordering="nd")
    assert amd.nnz_L < 0.5 * nat.nnz_L and nd.nnz_L < 0.5 * nat.nnz_L
    auto = analyze_csr(A, "SPD")
    cost = lambda S: S.flops + 1e8 * S.sdepth  # noqa: E731
    assert cost(auto) <= min(cost(amd), cost(nd)) + 1e-6


def test_pairs_eliminated_together():
    A = M.kkt(10, 10, 40, seed=2)
    S = analyze_csr(A, "S")
    assert S.pairs.size > 0
    pos = np.empty(S.n, np.int64)
    pos[S.perm - 1] = np.arange(S.n)
    col2sn = np.repeat(np.arange(S.ns), np.diff(S.super_ptr))
    for a, c in S.pairs.reshape(-1, 2):
        assert pos[c - 1] == pos[a - 1] + 1
        assert col2sn[pos[a - 1]] == col2sn[pos[c - 1]]


def test_user_perm_and_errors():
    A = M.lap2d_shifted(5, 5)
    up = np.arange(25)[::-1].copy()
    S = analyze_csr(A, "SPD", user_perm=up)
    assert S.alg_used == 4
    with pytest.raises(ValueError):
        analyze_csr(A, "SPD", user_perm=np.zeros(25, np.int64))
    with pytest.raises(ValueError):
        from sdsb200 import analyze
        analyze(A.indptr[:-1], A.indices, 25, "SPD")

"""The CPU oracle against independent references (CPU only).

The reference ships no golden vectors for the numeric phase; its tests pin the
CPU oracle through invariants (test/test_reference_ldlt.jl, test/utils.jl):
residuals, A[p,p] = L D L^T, eigenvalue inertia, perturbation counts. The same
invariants are checked here against numpy/scipy, plus the known-answer
fixtures of tests/golden/ (dense factors computed by LAPACK through numpy).
"""
import json
import os

import numpy as np
import pytest
import scipy.linalg as sla
import scipy.sparse as sp

from helpers import eigen_inertia, oracle_for, small_kkt
from sdsb200 import matrices as M

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _reconstruct_ldlt(S, O):
    """A[p, p] = L D L^T with p = perm[piv] (extract_ldlt, src/reference/ldlt.jl:550-580)."""
    n = S.n
    piv = O.piv[:n].astype(np.int64)
    pos = np.empty(n, np.int64)
    pos[piv - 1] = np.arange(n)
    L = np.zeros((n, n))
    for s in range(S.ns):
        f, w, base = int(S.front_nrows[s]), int(S.front_ncols[s]), int(S.front_ptr[s]) - 1
        rows = S.rowval[S.rowptr[s] - 1: S.rowptr[s + 1] - 1] - 1
        c0 = int(S.super_ptr[s]) - 1
        for j in range(w):
            for i in range(j, f):
                r = c0 + i if i < w else pos[rows[i]]
                L[r, c0 + j] = O.factor[base + j * f + i]
    D = np.diag(O.d[:n])
    for k in range(n):
        if O.kind[k] == 2:
            D[k + 1, k] = D[k, k + 1] = O.d[n + k]
    p = S.perm[piv - 1] - 1
    return L, D, p


@pytest.mark.parametrize("reordering", ["amd", "nd", "natural"])
def test_cholesky_oracle_vs_lapack(reordering):
    A = M.lap2d_shifted(12, 12, seed=1)
    S, O, info = oracle_for(A, "SPD", reordering=reordering)
    assert info == 0
    p = S.perm - 1
    Lref = np.linalg.cholesky(A.toarray()[np.ix_(p, p)])
    L = np.zeros_like(Lref)
    for s in range(S.ns):
        f, w, base = int(S.front_nrows[s]), int(S.front_ncols[s]), int(S.front_ptr[s]) - 1
        rows = S.rowval[S.rowptr[s] - 1: S.rowptr[s + 1] - 1] - 1
        c0 = int(S.super_ptr[s]) - 1
        for j in range(w):
            for i in range(j, f):
                L[rows[i], c0 + j] = O.factor[base + j * f + i]
    assert np.abs(L - Lref).max() <= 1e-13 * np.abs(Lref).max()
    b = M.rhs(S.n, 3, seed=2)
    assert M.scaled_backward_error(A, O.solve(b), b) <= 1e-15


@pytest.mark.parametrize("case", ["kkt", "kkt_onefront", "kkt_nopairs"])
def test_ldlt_oracle_invariants(case):
    # without pairs the dual rows are 1x1 leaf pivots of size delta: the reference
    # (test_reference_ldlt.jl) uses delta = 1e-8 there and the backward error relative
    # to |L| |D| |L|^T, since the growth is ~1/delta
    nopairs = case == "kkt_nopairs"
    A = small_kkt(12, 12, 60, seed=3, delta=1e-8 if nopairs else 0.0)
    kw = {}
    if case == "kkt_onefront":
        kw["amalgamation"] = (10_000, 100.0, 10_000)
    if nopairs:
        kw["pivot_pairs"] = "none"
    S, O, info = oracle_for(A, "S", **kw)
    assert info == 0
    st = O.stats_matrix().sum(0)
    assert (st[0], st[1]) == eigen_inertia(A) == (144, 60)
    assert st[4] == (O.kind[: S.n] == 2).sum() == (O.kind[: S.n] == 3).sum()
    L, D, p = _reconstruct_ldlt(S, O)
    Ap = A.toarray()[np.ix_(p, p)]
    E = np.abs(Ap - L @ D @ L.T)
    if nopairs:
        assert E.max() <= 1e-12 * (np.abs(L) @ np.abs(D) @ np.abs(L).T).max()
        return
    assert E.max() <= 1e-12 * np.abs(Ap).max()
    b = M.rhs(S.n, 2, seed=4)
    assert M.scaled_backward_error(A, O.solve(b), b) <= 1e-13


def test_ldlt_oracle_bk_2x2_known_answer():
    # [[0, 1], [1, 0]] as one front: a 2x2 pivot, D equal to the block, unit L
    A = sp.csr_matrix(np.array([[0.0, 1.0], [1.0, 0.0]]))
    A = A + sp.csr_matrix((np.zeros(2), ([0, 1], [0, 1])), shape=(2, 2))
    A.sort_indices()
    S, O, info = oracle_for(A, "S", pivot_pairs="none", reordering="natural")
    assert info == 0
    assert list(O.kind[:2]) == [2, 3]
    assert O.d[0] == 0.0 and O.d[1] == 0.0 and O.d[2] == 1.0
    assert tuple(O.stats_matrix().sum(0)[:2]) == (1, 1)


def test_ldlt_zero_pivot_info_and_perturbation():
    A = sp.csr_matrix(np.diag([2.0, 0.0, 3.0]))
    A = A + sp.csr_matrix((np.zeros(3), (np.arange(3), np.arange(3))), shape=(3, 3))
    A.sort_indices()
    S, O, info = oracle_for(A, "S", pivot_epsilon=0.0, pivot_pairs="none", reordering="natural")
    assert info == S.perm[1] or info == 2
    S, O, info = oracle_for(A, "S", pivot_epsilon=1e-10, pivot_pairs="none", reordering="natural")
    assert info == 0
    st = O.stats_matrix().sum(0)
    assert st[2] == 1 and st[3] == 1   # nzero, nperturbed


@pytest.mark.parametrize("u", [0.1, 1.0])
def test_lu_oracle_vs_dense(u):
    A = M.convection_diffusion3d(6, 6, 6, seed=5)
    S, O, info = oracle_for(A, "G", pivot_threshold=u)
    assert info == 0
    b = M.rhs(S.n, 2, seed=6)
    assert M.scaled_backward_error(A, O.solve(b), b) <= 1e-14
    assert M.scaled_backward_error(A.T.tocsr(), O.solve(b, transpose=True), b) <= 1e-14
    x = np.linalg.solve(A.toarray(), b)
    assert np.abs(O.solve(b) - x).max() <= 1e-10 * np.abs(x).max()


def test_cholesky_oracle_failure_info():
    A = M.lap2d_shifted(6, 6).tolil()
    A[10, 10] = -1.0
    A = A.tocsr()
    S, O, info = oracle_for(A, "SPD", pivot_epsilon=0.0)
    assert info > 0
    # the failing original column is one whose elimination meets a non-positive pivot
    assert 1 <= info <= S.n


def test_golden_fixtures():
    with open(os.path.join(GOLDEN, "dense_fronts.json")) as fh:
        cases = json.load(fh)
    assert len(cases) >= 3
    for c in cases:
        A = sp.csr_matrix((np.array(c["data"]), np.array(c["indices"]), np.array(c["indptr"])),
                          shape=(c["n"], c["n"]))
        S, O, info = oracle_for(A, c["structure"], reordering="natural", pivot_pairs="none",
                                amalgamation=(10_000, 100.0, 10_000), pivot_threshold=c.get("u", 0.01))
        assert S.ns == 1 and info == 0
        n = c["n"]
        if c["structure"] == "SPD":
            L = O.factor[: n * n].reshape(n, n).T
            assert np.allclose(np.tril(L), np.array(c["L"]), rtol=1e-13, atol=1e-14)
        elif c["structure"] == "G":
            assert list(O.piv[:n]) == c["piv"]
            L = np.tril(O.factor[: n * n].reshape(n, n).T, -1) + np.eye(n)
            U = np.tril(O.ufactor[: n * n].reshape(n, n).T, -1).T + np.eye(n)
            assert np.allclose(L, np.array(c["L"]), rtol=1e-13, atol=1e-14)
            assert np.allclose(np.diag(O.d[:n]) @ U, np.array(c["DU"]), rtol=1e-13, atol=1e-14)
        else:
            assert list(O.kind[:n]) == c["kind"]
            assert np.allclose(O.d[: 2 * n], np.array(c["d"]), rtol=1e-13, atol=1e-14)


@pytest.mark.parametrize("structure", ["SPD", "S", "G"])
def test_edge_cases_small_and_empty(structure):
    """The smallest inputs the reference's tests use: n = 0, n = 1, a diagonal matrix (every front a
    single column), and a structurally empty row. The empty row meets the static pivot of the SPD clamp
    (0 <= a_jj accepted as eps = 1e-13, src/numeric/front.jl:38-53) and the LDLT/LU perturbation to
    eps, so its unknown is b / eps."""
    from sdsb200 import analyze_csr

    S = analyze_csr(sp.csr_matrix((0, 0)), structure)
    assert S.n == 0 and S.ns == 0
    for A, x_expected in ((sp.csr_matrix(np.array([[4.0]])), [0.25]),
                          (sp.diags(np.arange(1.0, 6.0)).tocsr(), 1.0 / np.arange(1.0, 6.0)),
                          (sp.csr_matrix(np.array([[2.0, 0.0], [0.0, 0.0]])), [0.5, 1e13])):
        S, O, info = oracle_for(A, structure)
        assert info == 0
        assert S.ns == A.shape[0]
        x = O.solve(np.ones(A.shape[0]))
        assert np.allclose(x, x_expected, rtol=1e-12)

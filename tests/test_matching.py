"""MC64 matching and scaling of the analysis library (CPU).

The reference's matching (src/matching/mc64.jl) has no golden outputs, and Julia cannot run here, so
the checks are the properties its docstrings state and the reference's own matching tests assert
(optimality of the assignment, the scaling bounds, the completion rule), against scipy's
independent assignment and bipartite-matching solvers.
"""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.optimize import linear_sum_assignment
from scipy.sparse.csgraph import maximum_bipartite_matching

from sdsb200.analysis import compute_matching


def _random_nonsingular(n, density, seed):
    """Sparse n x n with a full structural matching hidden behind a random column permutation."""
    rng = np.random.default_rng(seed)
    A = sp.random(n, n, density=density, random_state=seed, format="coo")
    P = sp.coo_matrix((rng.uniform(0.1, 10.0, n) * rng.choice([-1, 1], n), (np.arange(n), rng.permutation(n))),
                      shape=(n, n))
    A = (A + P).tocsr()
    A.data *= np.exp(rng.normal(0, 3, A.nnz))          # values spread over many orders of magnitude
    return A


def _matched_values(A, perm):
    D = np.abs(A.toarray())
    return D[np.arange(A.shape[0]), perm - 1]


def _optimum(A, objective):
    D = np.abs(A.toarray())
    if objective == "product":
        cost = np.where(D > 0, -np.log(np.where(D > 0, D, 1.0)), 1e6)
    else:
        cost = np.where(D > 0, -D, 1e12)
    r, c = linear_sum_assignment(cost)
    return D[r, c]


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_job5_maximizes_product_and_scales(seed):
    A = _random_nonsingular(60, 0.08, seed)
    m = compute_matching(A.indptr, A.indices, A.data, 60, "G", "algo5")
    assert m.matched.all()
    assert sorted(m.perm) == list(range(1, 61))
    got = np.log(_matched_values(A, m.perm)).sum()
    best = np.log(_optimum(A, "product")).sum()
    assert got == pytest.approx(best, rel=0, abs=1e-9 * max(1.0, abs(best)))
    # |r_i a_ij c_j| <= 1 on every stored entry, = 1 on the matched ones
    S = sp.diags(m.rscale) @ abs(A) @ sp.diags(m.cscale)
    assert S.max() <= 1 + 1e-12
    assert np.allclose(S.toarray()[np.arange(60), m.perm - 1], 1.0, rtol=1e-12)


def test_job4_maximizes_sum():
    A = _random_nonsingular(50, 0.1, 7)
    m = compute_matching(A.indptr, A.indices, A.data, 50, "G", 4)
    assert _matched_values(A, m.perm).sum() == pytest.approx(_optimum(A, "sum").sum(), rel=1e-12)
    assert np.all(m.rscale == 1.0) and np.all(m.cscale == 1.0)


@pytest.mark.parametrize("job", [2, 3])
def test_bottleneck_jobs(job):
    A = _random_nonsingular(40, 0.1, 11)
    m = compute_matching(A.indptr, A.indices, A.data, 40, "G", job)
    assert m.matched.all()
    got = _matched_values(A, m.perm).min()
    # the largest threshold that still admits a perfect matching
    vals = np.unique(np.abs(A.data[A.data != 0]))
    best = 0.0
    for t in vals:
        B = A.copy()
        B.data = (np.abs(B.data) >= t).astype(float)
        B.eliminate_zeros()
        if (maximum_bipartite_matching(B, perm_type="column") >= 0).sum() == 40:
            best = t
    assert got == best


def test_job1_structurally_singular_completion():
    # rows 2 and 5 share their only columns with others: structural rank n - 1
    rows = [0, 0, 1, 2, 3, 3, 4, 5, 6]
    cols = [0, 1, 1, 2, 3, 4, 4, 2, 6]
    A = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(7, 7))
    m = compute_matching(A.indptr, A.indices, A.data, 7, "G", "algo1")
    rank = (maximum_bipartite_matching(A, perm_type="column") >= 0).sum()
    assert m.matched.sum() == rank == 6
    assert sorted(m.perm) == list(range(1, 8))
    for i in np.nonzero(m.matched)[0]:
        assert A[i, m.perm[i] - 1] != 0
    # the unmatched row takes the unmatched column (here column 6, 1-based)
    (u,) = np.nonzero(~m.matched)
    assert m.perm[u[0]] == 6


def test_explicit_zero_counts_for_job1_only():
    A = sp.csr_matrix((np.array([1.0, 0.0, 1.0]), (np.array([0, 1, 1]), np.array([1, 0, 1]))), shape=(2, 2))
    assert compute_matching(A.indptr, A.indices, A.data, 2, "G", 1).matched.all()
    assert not compute_matching(A.indptr, A.indices, A.data, 2, "G", 5).matched.all()


@pytest.mark.parametrize("structure", ["S", "SPD"])
def test_symmetric_scaling_from_either_triangle(structure):
    rng = np.random.default_rng(3)
    B = sp.random(80, 80, density=0.05, random_state=3, format="csr")
    A = (B + B.T).tocsr()
    A.setdiag(rng.uniform(0.01, 100.0, 80) * (1 if structure == "SPD" else rng.choice([-1, 1], 80)))
    A = A.tocsr()
    A.sort_indices()
    full = compute_matching(A.indptr, A.indices, A.data, 80, structure, "algo5", view="F")
    L = sp.tril(A).tocsr()
    low = compute_matching(L.indptr, L.indices, L.data, 80, structure, "algo5", view="L")
    U = sp.triu(A).tocsr()
    up = compute_matching(U.indptr, U.indices, U.data, 80, structure, "algo5", view="U")
    assert full.symmetric
    assert np.array_equal(full.rscale, full.cscale)
    assert np.array_equal(full.rscale, low.rscale) and np.array_equal(full.rscale, up.rscale)
    assert np.array_equal(full.perm, low.perm)
    d = full.rscale
    S = sp.diags(d) @ abs(A) @ sp.diags(d)
    assert S.max() <= 1 + 1e-12


def test_index_base_one_and_errors():
    A = _random_nonsingular(20, 0.2, 5)
    m0 = compute_matching(A.indptr, A.indices, A.data, 20, "G", 5)
    m1 = compute_matching(A.indptr + 1, A.indices + 1, A.data, 20, "G", 5, index_base=1)
    assert np.array_equal(m0.perm, m1.perm) and np.array_equal(m0.rscale, m1.rscale)
    assert compute_matching(A.indptr, A.indices, A.data, 20, "G", "algo6").job == 5
    with pytest.raises(ValueError, match="unknown matching job"):
        compute_matching(A.indptr, A.indices, A.data, 20, "G", 7)
    with pytest.raises(ValueError, match="column index out of range"):
        compute_matching(A.indptr, A.indices + 30, A.data, 20, "G", 5)


def _host_solver(A, structure, alg="algo5"):
    """A DirectSolver's host side only (CPU tensors, no plan): enough for the matching algebra."""
    import torch

    from sdsb200.solver import _DEFAULTS, DirectSolver

    ds = DirectSolver.__new__(DirectSolver)
    ds._torch = torch
    ds.device = torch.device("cpu")
    ds.rowptr, ds.colval, ds.n, ds.nnz = A.indptr.astype(np.int64), A.indices.astype(np.int64), A.shape[0], A.nnz
    ds.structure, ds.view, ds.index_base, ds.nbatch = structure, "F", 0, 1
    ds.params = dict(_DEFAULTS)
    ds.params["matching_alg"] = alg
    ds.nzval = torch.from_numpy(A.data.astype(np.float64))
    ds._matching = ds._mdev = None
    return ds


@pytest.mark.parametrize("structure", ["G", "S", "SPD"])
@pytest.mark.parametrize("mode", [0, 1])
def test_matched_system_algebra(structure, mode):
    """The matched system the numeric phase would factor, solved here by scipy, maps back to A x = b
    (or A^T x = b): the relabeled analysis columns, the entry weights, the right-hand-side scaling and
    the solution's unscaling of DirectSolver."""
    import torch
    from scipy.sparse.linalg import spsolve

    rng = np.random.default_rng(5)
    n = 50
    if structure == "G":
        A = _random_nonsingular(n, 0.1, 9)
    else:
        B = sp.random(n, n, density=0.08, random_state=9, format="csr")
        A = (B + B.T).tocsr()
        A.setdiag(rng.uniform(1.0, 5.0, n) * (1 if structure == "SPD" else rng.choice([-1, 1], n)) + 0.0)
        if structure == "SPD":
            A = A + sp.eye(n) * (abs(A).sum(1).max() + 1.0)
        D = sp.diags(np.exp(rng.normal(0, 4, n)))
        A = (D @ A @ D).tocsr()
    A.sort_indices()
    ds = _host_solver(A, structure)
    colval = ds._prepare_matching()
    w = ds._mdev["w_host"]
    # M: the stored entries with the analysis' column indices and the factored values
    rows = np.repeat(np.arange(n), np.diff(A.indptr))
    M = sp.csr_matrix((A.data * w, (rows, np.asarray(colval) - 0)), shape=(n, n))
    if structure == "G":
        # the matched entries are on M's diagonal, of modulus 1 (job 5)
        assert np.allclose(np.abs(M.diagonal()), 1.0, rtol=1e-12)
    b = rng.uniform(-1, 1, (n, 2))
    Bcm = torch.from_numpy(np.ascontiguousarray(b.T))
    rhs = ds._scaled_rhs(Bcm, mode).numpy().T
    Y = spsolve((M if mode == 0 else M.T).tocsc(), rhs)
    X = ds._unscaled_solution(torch.from_numpy(np.ascontiguousarray(Y.T)), mode).numpy().T
    AA = A if mode == 0 else A.T
    res = np.abs(AA @ X - b).max() / (np.abs(AA).max() * np.abs(X).max() + np.abs(b).max())
    assert res <= 1e-12


def test_matching_pairs_from_cycles():
    """The 2x2 pairs of "S" from a job-5 matching's cycles (matching_pairs, src/matching/mc64.jl:380-441),
    and the analysis keeping each pair adjacent when they are passed as user_pairs."""
    from helpers import small_kkt
    from sdsb200.analysis import analyze, matching_pairs

    A = small_kkt(8, 8, 20, seed=1).tocsr()
    A.sort_indices()
    n = A.shape[0]
    m = compute_matching(A.indptr, A.indices, A.data, n, "S", "algo5")
    pr = matching_pairs(A.indptr, A.indices, A.data, n, m)
    assert len(pr) == 20                                    # one per constraint row of [H J^T; J 0]
    flat = pr.ravel()
    assert len(set(flat.tolist())) == flat.size             # disjoint
    assert np.all(np.diff(pr[:, 1]) > 0)                    # sorted by candidate
    D = A.toarray()
    for partner, cand in pr:
        assert D[partner - 1, cand - 1] != 0                # consecutive in a cycle: adjacent in A
        assert D[cand - 1, cand - 1] == 0                   # the candidate is the zero-diagonal row
    assert len(matching_pairs(A.indptr, A.indices, A.data, n, m, pivot_pairs="none")) == 0
    assert len(matching_pairs(A.indptr, A.indices, A.data, n, m, pivot_pairs="all")) >= len(pr)
    S = analyze(A.indptr, A.indices, n, "S", nzval=A.data, user_pairs=pr)
    assert np.array_equal(S.maps["pairs"], pr.ravel())
    pos = np.empty(n, int)
    pos[S.perm - 1] = np.arange(n)
    assert all(abs(pos[a - 1] - pos[b - 1]) == 1 for a, b in pr)
    with pytest.raises(ValueError, match="user_pairs out of range"):
        analyze(A.indptr, A.indices, n, "S", nzval=A.data, user_pairs=[[1, n + 5]])

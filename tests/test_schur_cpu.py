"""Schur complement mode on the host (CPU): the analysis and the oracle.

The reference orders the flagged rows and columns of ``user_schur_indices`` last, in increasing
order, as one dense root supernode (compute_schur_ordering, src/symbolic/ordering.jl:386-415;
schur_supernode_partition, src/symbolic/supernodes.jl:391-425), exports the pattern of
S = A22 - A21 A11^{-1} A12 (schur_pattern, ordering.jl:424-470), and the numeric phase assembles
that root without factoring it (assemble_schur!, src/numeric/schur.jl:65-98). The checks: the
ordering and partition invariants, the pattern against the nonzeros of a dense Schur complement,
and the oracle's assembled root against the dense S (the pin of the oracle's Schur semantics),
with the root's unit pivots and zero statistics.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from helpers import oracle_for
from sdsb200 import analyze_csr
from sdsb200 import matrices as M


def _flags(n, k, seed):
    fl = np.zeros(n, np.int8)
    fl[np.random.default_rng(seed).choice(n, k, replace=False)] = 1
    return fl


def dense_schur(A, fl):
    Ad = A.toarray()
    idx, rest = np.flatnonzero(fl), np.flatnonzero(fl == 0)
    if rest.size == 0:
        return Ad
    return Ad[np.ix_(idx, idx)] - Ad[np.ix_(idx, rest)] @ np.linalg.solve(Ad[np.ix_(rest, rest)], Ad[np.ix_(rest, idx)])


def oracle_schur(S, O, structure):
    """The oracle's assembled root as a dense matrix: the lower triangle of L's panel, the strict upper one
    mirrored ("SPD", "S") or from the U^T panel ("G")."""
    ns = S.schur_n
    p0 = int(S.front_ptr[S.schur - 1]) - 1
    P = O.factor[p0:p0 + ns * ns].reshape(ns, ns, order="F")
    if structure == "G":
        U = O.ufactor[p0:p0 + ns * ns].reshape(ns, ns, order="F")
        return np.tril(P) + np.triu(U.T, 1)
    return np.tril(P) + np.tril(P, -1).T


def _indefinite(nx, ny):
    """A symmetric indefinite matrix with a nonzero diagonal: no zero pivot, so no perturbation changes S."""
    return (M.lap2d_shifted(nx, ny) - 2.5 * sp.eye(nx * ny)).tocsr()


CASES = {
    "SPD": lambda: M.lap2d_shifted(10, 10),
    "S": lambda: _indefinite(10, 10),
    "G": lambda: M.convection_diffusion3d(5, 5, 5, seed=2),
}


@pytest.mark.parametrize("structure", ["SPD", "S", "G"])
@pytest.mark.parametrize("k", [1, 12])
def test_schur_ordering_and_partition(structure, k):
    A = CASES[structure]()
    A.sort_indices()
    n = A.shape[0]
    fl = _flags(n, k, seed=k)
    S = analyze_csr(A, structure, user_schur_indices=fl)
    assert S.schur == S.ns and S.schur_n == k
    # the flagged indices last, in increasing original order (1-based perm)
    assert np.array_equal(S.perm[-k:], np.flatnonzero(fl) + 1)
    assert sorted(S.perm) == list(range(1, n + 1))
    # one dense root: its rows are its columns, no 2x2 pairs
    assert S.snparent[-1] == 0
    assert S.super_ptr[-1] - S.super_ptr[-2] == k
    assert S.rowptr[-1] - S.rowptr[-2] == k
    assert S.front_ptr[-1] - S.front_ptr[-2] == k * k
    assert S.pairs.size == 0
    # every other supernode reaches the root or is a root of a part that never touches the Schur block
    for s in range(S.ns - 1):
        assert S.snparent[s] == 0 or S.snparent[s] > s + 1


def test_schur_pattern_matches_dense():
    rng = np.random.default_rng(3)
    for A, fl in ((M.lap2d_shifted(12, 9), _flags(108, 15, 1)), (M.lap3d(6, 5, 4, shift=0.1), _flags(120, 20, 2))):
        A = A.tocsr()
        A.sort_indices()
        A.data = A.data * (1 + 0.1 * rng.random(A.nnz))   # generic values: no cancellation in S
        A = ((A + A.T) * 0.5).tocsr()
        A.sort_indices()
        S = analyze_csr(A, "SPD", user_schur_indices=fl)
        ns = S.schur_n
        pat = np.zeros((ns, ns), bool)
        for i in range(ns):
            pat[i, S.schur_colval[S.schur_rowptr[i] - 1:S.schur_rowptr[i + 1] - 1] - 1] = True
        assert np.array_equal(pat, np.abs(dense_schur(A, fl)) > 1e-13)
        assert np.array_equal(pat, pat.T) and pat.diagonal().all()


def test_schur_user_perm():
    """With a user permutation the other indices come first (in the supernodal postorder of the partition
    built from the user's relative order), the Schur indices last in increasing order."""
    A = M.lap2d_shifted(8, 8)
    n = A.shape[0]
    fl = _flags(n, 6, seed=4)
    up = np.random.default_rng(5).permutation(n) + 1
    S = analyze_csr(A, "SPD", user_schur_indices=fl, user_perm=up)
    assert S.alg_used == 4
    assert sorted(S.perm[: n - 6]) == sorted(v for v in up if not fl[v - 1])
    assert np.array_equal(S.perm[n - 6:], np.flatnonzero(fl) + 1)


def test_schur_rejects_bad_flags():
    A = M.lap2d_shifted(6, 6)
    with pytest.raises(ValueError, match="selects no row"):
        analyze_csr(A, "SPD", user_schur_indices=np.zeros(36, np.int8))
    with pytest.raises(ValueError, match="entries"):
        analyze_csr(A, "SPD", user_schur_indices=np.ones(35, np.int8))


@pytest.mark.parametrize("structure", ["SPD", "S", "G"])
@pytest.mark.parametrize("k", [1, 12, "all"])
def test_oracle_schur_complement(structure, k):
    A = CASES[structure]()
    A.sort_indices()
    n = A.shape[0]
    fl = np.ones(n, np.int8) if k == "all" else _flags(n, k, seed=7)
    kw = dict(pivot_threshold=0.1) if structure == "G" else {}
    S, O, info = oracle_for(A, structure, user_schur_indices=fl, **kw)
    assert info == 0
    Sd = dense_schur(A, fl)
    So = oracle_schur(S, O, structure)
    assert np.abs(So - Sd).max() <= 1e-12 * np.abs(Sd).max()
    # the root: zero statistics; unit 1x1 pivots in identity order for LDLT and LU
    st = O.stats_matrix()
    assert not st[-1].any()
    ns = S.schur_n
    if structure != "SPD":
        assert np.array_equal(O.piv[n - ns:n], np.arange(n - ns + 1, n + 1))
        assert np.all(O.kind[n - ns:n] == 1)
        assert np.all(O.d[n - ns:n] == 1.0) and not O.d[2 * n - ns:2 * n].any()
    if structure == "S" and k != "all":
        # the inertia counts the factored block A11 only
        rest = np.flatnonzero(fl == 0)
        ev = np.linalg.eigvalsh(A.toarray()[np.ix_(rest, rest)])
        tot = st.sum(0)
        assert (tot[0], tot[1]) == (int((ev > 0).sum()), int((ev < 0).sum()))


@pytest.mark.parametrize("variant", ["amd", "nd", "natural", "user_perm", "no_amalgamation"])
def test_schur_forest_of_two_blocks(variant):
    """As the reference's Schur edge-case test (test/test_schur.jl:186-210): two disconnected blocks with the
    Schur indices in the second one only, so the first block is a tree of its own."""
    A = sp.block_diag([M.laplacian2d(6, 6), M.laplacian2d(7, 5)]).tocsr()
    A.sort_indices()
    n = A.shape[0]
    fl = np.zeros(n, np.int8)
    fl[np.array([40, 45, 50, 55, 60, 70]) - 1] = 1
    kw = {"amd": dict(reordering="amd"), "nd": dict(reordering="nd"), "natural": dict(reordering="natural"),
          "user_perm": dict(user_perm=np.random.default_rng(1).permutation(n) + 1),
          "no_amalgamation": dict(use_superpanels=0)}[variant]
    S, O, info = oracle_for(A, "SPD", user_schur_indices=fl, **kw)
    assert info == 0
    assert np.array_equal(S.perm[n - 6:], np.flatnonzero(fl) + 1)
    assert (S.snparent == 0).sum() >= 2                       # the first block's root besides the Schur root
    Sd = dense_schur(A, fl)
    assert np.abs(oracle_schur(S, O, "SPD") - Sd).max() <= 1e-12 * np.abs(Sd).max()
    rows = np.repeat(np.arange(6), np.diff(S.schur_rowptr))
    lower = int(np.count_nonzero(S.schur_colval - 1 <= rows))
    assert lower == int(np.count_nonzero(np.tril(np.abs(Sd) > 1e-13)))


def test_schur_shape_of_a_corner():
    """The first four indices of a 6 x 6 Laplacian: S is dense, 4 x 4 with 10 lower entries
    (test/test_schur.jl:238)."""
    A = sp.tril(M.laplacian2d(6, 6)).tocsr()
    fl = np.zeros(36, np.int8)
    fl[:4] = 1
    S = analyze_csr(A, "SPD", view="L", user_schur_indices=fl)
    rows = np.repeat(np.arange(4), np.diff(S.schur_rowptr))
    assert S.schur_n == 4 and int(np.count_nonzero(S.schur_colval - 1 <= rows)) == 10


def test_schur_directsolver_errors():
    """DirectSolver refuses Schur mode without indices, with an empty set, and for a uniform batch, before
    any device work (device="cpu": these checks precede the analysis)."""
    torch = pytest.importorskip("torch")  # noqa: F841
    from sdsb200.solver import DirectSolver, InvalidValueError, NotSupportedError

    A = M.lap2d_shifted(6, 6)
    for ind in (None, np.zeros(36)):
        ds = DirectSolver(A, "SPD", device="cpu", schur_mode=1)
        if ind is not None:
            ds.setparam("user_schur_indices", ind)
        with pytest.raises(InvalidValueError):
            ds.execute("analysis")
    with pytest.raises(InvalidValueError):
        DirectSolver(A, "SPD", device="cpu", user_schur_indices=np.ones(35))
    vals = np.concatenate([A.data, 2 * A.data])
    batch = DirectSolver((A.indptr, A.indices, vals, 36), "SPD", device="cpu", schur_mode=1,
                         user_schur_indices=np.eye(1, 36, 0).ravel())
    with pytest.raises(NotSupportedError):
        batch.execute("analysis")

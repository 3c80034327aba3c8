"""Schur complement mode and the solve sub-phases on the GPU, through DirectSolver and the C ABI.

Schur complement mode (src/solver.jl:395-418, 876-900; src/numeric/schur.jl): the factorization
factors A11 and assembles S = A22 - A21 A11^{-1} A12 in the unfactored root; "solve_fwd_schur",
"solve_diag" and "solve_bwd_schur" then solve A x = b around the user's solve of the condensed
system. The checks: S against the oracle's assembled root (same Symbolic) and against a dense
Schur complement; pivots, kinds and statistics of the factored part exactly the oracle's; the
condensed right-hand side against b2 - A21 A11^{-1} b1; the whole route to a scaled backward error
<= 1e-12 (A and, for "G", A^T); the CSR export; the phase errors.

The sub-phases (src/solver.jl:856-867): "solve_fwd_perm", "solve_fwd", "solve_diag", "solve_bwd",
"solve_bwd_perm" in a row give the complete solve's X bit for bit when the complete solve runs the
same per-level launches (persistent engine off), and within rounding of the persistent engine.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from helpers import small_kkt
from sdsb200 import matrices as M
from test_schur_cpu import CASES, _flags, dense_schur, oracle_schur

pytestmark = pytest.mark.gpu

BERR = 1e-12
S_TOL = 1e-12     # S of the GPU (DMMA updates, their own summation order) against the oracle's


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def _schur_solver(structure, k=12, **params):
    from sdsb200.solver import DirectSolver

    A = CASES[structure]()
    A.sort_indices()
    fl = _flags(A.shape[0], k, seed=7)
    if structure == "G":
        params.setdefault("pivot_threshold", 0.1)
    ds = DirectSolver(A, structure, schur_mode=1, user_schur_indices=fl, **params)
    ds.execute("analysis")
    return A, fl, ds


@pytest.mark.parametrize("structure", ["SPD", "S", "G"])
def test_schur_complement_against_oracle(torch_cuda, structure):
    from oracle.oracle import Oracle

    A, fl, ds = _schur_solver(structure)
    n, ns = A.shape[0], 12
    lower = structure != "G"
    shape = ds.getparam("schur_shape")
    assert shape[:2] == (ns, ns)
    assert ds.execute("factorization") == 0
    Sg = ds.getparam("schur_matrix").cpu().numpy()
    O = Oracle(ds.symbolic)
    assert O.factorize(A.data, structure, pivot_threshold=0.1 if structure == "G" else 0.01) == 0
    So = oracle_schur(ds.symbolic, O, structure)
    assert np.abs(Sg - So).max() <= S_TOL * np.abs(So).max()
    Sd = dense_schur(A, fl)
    assert np.abs(Sg - Sd).max() <= 1e-11 * np.abs(Sd).max()
    if lower:
        assert np.array_equal(Sg, Sg.T)
    # the factored part is the oracle's; the root has unit pivots and zero statistics
    assert np.array_equal(ds.stats_host(), O.stats_matrix())
    assert not ds.stats_host()[-1].any()
    if structure != "SPD":
        piv, kind, d = ds.pivots_host()
        assert np.array_equal(piv[:n], O.piv[:n])
        assert np.array_equal(kind[:n], O.kind[:n])
        assert np.array_equal(d[n - ns:n], np.ones(ns))


@pytest.mark.parametrize("case", ["SPD", "S", "G", "G_T"])
def test_schur_solve_route(torch_cuda, case):
    """solve_fwd_schur -> solve_diag -> (x2 = S^{-1} b_s on the host) -> solve_bwd_schur solves A x = b."""
    structure = case[0] if case != "SPD" else "SPD"
    A, fl, ds = _schur_solver(structure)
    transpose = case == "G_T"
    if transpose:
        ds.setparam("solve_mode", 1)
    n, ns = A.shape[0], 12
    ds.execute("factorization")
    Sg = ds.getparam("schur_matrix").cpu().numpy()
    b = M.rhs(n, 2, seed=11)
    Z = ds.execute("solve_fwd_schur", None, b).cpu().numpy()
    # the condensed right-hand side b2 - A21 A11^{-1} b1 (with A^T for the transposed solve)
    AA = A.T.tocsr() if transpose else A
    Ad = AA.toarray()
    idx, rest = np.flatnonzero(fl), np.flatnonzero(fl == 0)
    bs = b[idx] - Ad[np.ix_(idx, rest)] @ np.linalg.solve(Ad[np.ix_(rest, rest)], b[rest])
    assert np.abs(Z[n - ns:] - bs).max() <= 1e-12 * np.abs(bs).max()
    Z = ds.execute("solve_diag", None, Z).cpu().numpy()
    Z[n - ns:] = np.linalg.solve(Sg.T if transpose else Sg, Z[n - ns:])
    x = ds.execute("solve_bwd_schur", None, Z).cpu().numpy()
    assert M.scaled_backward_error(AA, x, b) <= BERR
    # X is B allowed: in place on a device tensor, one right-hand side
    bt = torch_cuda.from_numpy(b[:, 0].copy()).cuda()
    ds.execute("solve_fwd_schur", bt, bt)
    ds.execute("solve_diag", bt, bt)
    zt = bt.cpu().numpy()
    zt[n - ns:] = np.linalg.solve(Sg.T if transpose else Sg, zt[n - ns:])
    bt.copy_(torch_cuda.from_numpy(zt))
    ds.execute("solve_bwd_schur", bt, bt)
    assert M.scaled_backward_error(AA, bt.cpu().numpy().reshape(n, 1), b[:, :1]) <= BERR


def test_schur_csr_export_and_errors(torch_cuda):
    from sdsb200.solver import DirectSolver, FactorizationError, InvalidValueError, NotSupportedError

    torch = torch_cuda
    A, fl, ds = _schur_solver("S")
    ns, _, nnz = ds.getparam("schur_shape")
    with pytest.raises(FactorizationError):
        ds.execute("solve_fwd_schur", None, np.ones(A.shape[0]))
    ds.execute("factorization")
    S = ds.symbolic
    rows = np.repeat(np.arange(ns), np.diff(S.schur_rowptr))
    keep = S.schur_colval - 1 <= rows                   # the lower triangle with the diagonal
    assert int(keep.sum()) == nnz
    rp = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=ns))])
    rowptr = torch.from_numpy(rp.astype(np.int64)).cuda()
    colval = torch.from_numpy((S.schur_colval[keep] - 1).astype(np.int64)).cuda()
    nzval = torch.zeros(nnz, dtype=torch.float64, device="cuda")
    ds.setparam("schur_matrix", (rowptr, colval, nzval, "L"))
    out = ds.getparam("schur_matrix")
    assert out.data_ptr() == nzval.data_ptr()
    ds.setparam("schur_matrix", None)
    D = ds.getparam("schur_matrix").cpu().numpy()
    assert np.array_equal(nzval.cpu().numpy(), D[rows[keep], S.schur_colval[keep] - 1])
    # the complete solve and the ordinary sub-phases need the full factorization
    for phase in ("solve", "solve_fwd", "solve_bwd_perm"):
        with pytest.raises(NotSupportedError):
            ds.execute(phase, None, np.ones(A.shape[0]))
    # a Schur phase without schur_mode = 1
    B = M.lap2d_shifted(6, 6)
    plain = DirectSolver(B, "SPD")
    plain.execute("analysis")
    plain.execute("factorization")
    with pytest.raises(FactorizationError):
        plain.execute("solve_fwd_schur", None, np.ones(36))
    with pytest.raises(InvalidValueError):
        plain.getparam("schur_matrix")
    bad = DirectSolver(B, "SPD", schur_mode=1)
    with pytest.raises(InvalidValueError):
        bad.execute("analysis")


@pytest.mark.parametrize("case", ["SPD", "S", "G", "G_T"])
def test_solve_sub_phases_match_solve(torch_cuda, case):
    from sdsb200._native import numeric_lib
    from sdsb200.solver import DirectSolver

    lib = numeric_lib()
    structure = "SPD" if case == "SPD" else case[0]
    A = {"SPD": lambda: M.lap3d(12, 12, 12, seed=3), "S": lambda: small_kkt(16, 16, 90, seed=3),
         "G": lambda: M.convection_diffusion3d(10, 10, 10, seed=3)}[structure]()
    ds = DirectSolver(A, structure, reordering_alg="nd", max_nrhs=4)
    ds.execute("analysis")
    ds.execute("factorization")
    if case == "G_T":
        ds.setparam("solve_mode", 1)
    b = M.rhs(A.shape[0], 3, seed=5)
    X = np.zeros_like(b)
    assert ds.execute("solve_fwd_perm", None, b) is None
    for phase in ("solve_fwd", "solve_diag", "solve_bwd"):
        ds.execute(phase, None, b)
    ds.execute("solve_bwd_perm", X, b)
    AA = A.T.tocsr() if case == "G_T" else A
    assert M.scaled_backward_error(AA, X, b) <= BERR
    x_persistent = ds.execute("solve", None, b).cpu().numpy()
    assert np.abs(X - x_persistent).max() <= 1e-10 * np.abs(x_persistent).max()
    lib.sdsb200_set_persistent(ds._plan, 0)
    x_levels = ds.execute("solve", None, b).cpu().numpy()
    assert np.array_equal(X, x_levels)

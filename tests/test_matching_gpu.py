"""Matching and scaling through the numeric phase (GPU): DirectSolver with ``matching_alg``.

The reference factors M = (Dr A Dc)[:, q] ("G") or D A D (symmetric structures) and maps the solve
back (src/solver.jl:545-604, src/solve/permute.jl:155-183). The checks: the GPU factorization of M
against the oracle's on the same Symbolic and scaled values (pivots, kinds, statistics exact), and
solves of the original system (A and A^T) to a scaled backward error <= 1e-12.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from helpers import small_kkt
from sdsb200 import matrices as M

pytestmark = pytest.mark.gpu

BERR = 1e-12


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def test_matching_lu_scrambled_rows(torch_cuda):
    from oracle.oracle import Oracle
    from sdsb200.solver import DirectSolver

    rng = np.random.default_rng(2)
    A0 = M.convection_diffusion3d(10, 10, 10, seed=2)
    n = A0.shape[0]
    P = sp.csr_matrix((np.ones(n), (np.arange(n), rng.permutation(n))), shape=(n, n))
    Dr = sp.diags(np.exp(rng.normal(0, 3, n)))
    A = (Dr @ P @ A0).tocsr()          # rows scrambled and badly scaled: the diagonal is mostly zero
    A.sort_indices()
    ds = DirectSolver(A, "G", matching_alg="algo5", pivot_threshold=0.1, ir_n_steps=5, ir_tol=1e-14)
    ds.execute("analysis")
    assert ds.execute("factorization") == 0
    perm = ds.getparam("perm_matching")
    assert sorted(perm) == list(range(1, n + 1))
    assert np.all(np.asarray(A[np.arange(n), perm - 1]).ravel() != 0)
    r, c = ds.getparam("scale_row"), ds.getparam("scale_col")
    assert np.all(r > 0) and np.all(c > 0)
    # the factorization of M against the oracle's on the same Symbolic and values
    O = Oracle(ds.symbolic)
    assert O.factorize(A.data * ds._mdev["w_host"], "G", pivot_threshold=0.1) == 0
    piv, kind, _ = ds.pivots_host()
    assert np.array_equal(piv[:n], O.piv[:n])
    assert np.array_equal(kind[:n], O.kind[:n])
    assert np.array_equal(ds.stats_host(), O.stats_matrix())
    b = M.rhs(n, 2, seed=3)
    x = ds.execute("solve", None, b).cpu().numpy()
    assert M.scaled_backward_error(A, x, b) <= BERR
    ds.setparam("solve_mode", 1)
    xt = ds.execute("solve", None, b).cpu().numpy()
    assert M.scaled_backward_error(A.T.tocsr(), xt, b) <= BERR


def test_matching_ldlt_keeps_inertia(torch_cuda):
    from sdsb200.solver import DirectSolver

    rng = np.random.default_rng(4)
    A0 = small_kkt(12, 12, 40, seed=4)
    n = A0.shape[0]
    D = sp.diags(np.exp(rng.normal(0, 3, n)))
    A = (D @ A0 @ D).tocsr()
    A.sort_indices()
    ds = DirectSolver(A, "S", matching_alg="algo5", ir_n_steps=10, ir_tol=1e-14)
    ds.execute("analysis")
    ds.execute("factorization")
    assert ds.getparam("inertia") == (144, 40)
    d = ds.getparam("scale_row")
    assert np.array_equal(d, ds.getparam("scale_col"))
    b = M.rhs(n, 1, seed=5)
    x = ds.execute("solve", None, b[:, 0]).cpu().numpy()
    assert M.scaled_backward_error(A, x.reshape(n, 1), b) <= BERR


def test_matching_outputs_need_matching(torch_cuda):
    from sdsb200.solver import DirectSolver, InvalidValueError

    A = M.lap3d(6, 6, 6)
    ds = DirectSolver(A, "SPD")
    ds.execute("analysis")
    with pytest.raises(InvalidValueError):
        ds.getparam("perm_matching")


def test_matching_fgmres_and_adjoint(torch_cuda):
    """FGMRES-IR on the matched system, and the solve's adjoint with matching against the host's
    (the matching changes how A is factored, not x, b-bar or A-bar): b-bar = A^-T x-bar and
    A-bar_ij = -b-bar_i x_j on the stored entries."""
    from scipy.sparse.linalg import spsolve

    from sdsb200 import adjoint
    from sdsb200.solver import DirectSolver

    torch = torch_cuda
    rng = np.random.default_rng(6)
    A0 = M.convection_diffusion3d(8, 8, 8, seed=6)
    n = A0.shape[0]
    P = sp.csr_matrix((np.ones(n), (np.arange(n), rng.permutation(n))), shape=(n, n))
    A = (sp.diags(np.exp(rng.normal(0, 2, n))) @ P @ A0).tocsr()
    A.sort_indices()
    ds = DirectSolver(A, "G", matching_alg="algo5", pivot_threshold=0.1, ir_mode="fgmres", ir_n_steps=10,
                      ir_tol=1e-14)
    ds.execute("analysis")
    ds.execute("factorization")
    b = M.rhs(n, 2, seed=7)
    x = ds.execute("solve", None, b).cpu().numpy()
    assert M.scaled_backward_error(A, x, b) <= BERR
    s = DirectSolver(A, "G", matching_alg="algo5", pivot_threshold=0.1)
    nz = torch.from_numpy(A.data.copy()).cuda().requires_grad_(True)
    bt = torch.from_numpy(b[:, 0].copy()).cuda().requires_grad_(True)
    xbar = np.linspace(-1.0, 1.0, n)
    xt = adjoint.solve(s, nz, bt)
    (xt * torch.from_numpy(xbar).cuda()).sum().backward()
    xh = spsolve(A.tocsc(), b[:, 0])
    bbar = spsolve(A.T.tocsc(), xbar)
    rows = np.repeat(np.arange(n), np.diff(A.indptr))
    abar = -bbar[rows] * xh[A.indices]
    assert np.abs(bt.grad.cpu().numpy() - bbar).max() <= 1e-8 * np.abs(bbar).max()
    assert np.abs(nz.grad.cpu().numpy() - abar).max() <= 1e-8 * np.abs(abar).max()

"""KKTSolver through the numeric phase (GPU): the interior-point loop of src/kkt.jl (factorize with new
values, inertia, solve) on a KKT matrix [H J^T; J 0] stored as its lower triangle."""
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


def _kkt_lower(nx, nj, seed):
    A = small_kkt(nx, nx, nj, seed=seed)
    L = sp.tril(A).tocsr()
    L.sort_indices()
    return A, L


def test_ipm_loop_static_pivoting(torch_cuda):
    from sdsb200.kkt import KKTSolver

    torch = torch_cuda
    nx, nj = 14, 60
    A, L = _kkt_lower(nx, nj, 3)
    n, nh = A.shape[0], nx * nx
    nz = torch.from_numpy(L.data.copy()).cuda()          # aliased: new values are written into it
    K = KKTSolver((L.indptr, L.indices, nz, n), "L", factorization="ldl", pivoting="none",
                  pivot_sign=[1] * nh + [-1] * nj, ir_n_steps=10)
    assert K.pipeline() == "stock" and K.getparam("info") == 0
    assert K.inertia() == (nh, 0, nj)
    b = M.rhs(n, 1, seed=1)[:, 0]
    x = np.zeros(n)
    K.solve(x, b)
    assert M.scaled_backward_error(A, x.reshape(n, 1), b.reshape(n, 1)) <= BERR
    # the next iterate: H scaled by 3, the same pattern, written into the aliased values
    rows = np.repeat(np.arange(n), np.diff(L.indptr))
    scale = np.where(rows < nh, 3.0, 1.0)
    nz.mul_(torch.from_numpy(scale).cuda())
    K.factorize()
    A2 = sp.tril(sp.csr_matrix((L.data * scale, L.indices, L.indptr), shape=(n, n)))
    A2 = (A2 + sp.tril(A2, -1).T).tocsr()
    assert K.inertia() == (nh, 0, nj)
    xb = torch.from_numpy(b.copy()).cuda()
    K.solve(xb)                                          # one vector: b in, x out
    assert M.scaled_backward_error(A2, xb.cpu().numpy().reshape(n, 1), b.reshape(n, 1)) <= BERR
    # explicit new values
    K.factorize(L.data)
    K.solve(x, b)
    assert M.scaled_backward_error(A, x.reshape(n, 1), b.reshape(n, 1)) <= BERR


def test_bunch_kaufman_with_matching(torch_cuda):
    from sdsb200.kkt import KKTSolver

    A, L = _kkt_lower(10, 30, 5)
    n = A.shape[0]
    K = KKTSolver(L, "L", factorization="ldl", pivoting="bk", matching="algo5", ir_n_steps=5)
    assert K.inertia() == (100, 0, 30)
    b = M.rhs(n, 1, seed=2)[:, 0]
    x = np.zeros(n)
    K.solve(x, b)
    assert M.scaled_backward_error(A, x.reshape(n, 1), b.reshape(n, 1)) <= BERR


def test_cholesky_and_deferred_analysis(torch_cuda):
    from sdsb200.kkt import KKTSolver
    from sdsb200.solver import FactorizationError

    A = M.lap3d(8, 8, 8, shift=0.1, seed=1)
    n = A.shape[0]
    L = sp.tril(A).tocsr()
    K = KKTSolver(L, "L", deferred_analysis=True)
    with pytest.raises(FactorizationError):
        K.inertia()
    K.factorize()
    assert K.inertia() == (n, 0, 0)
    b = M.rhs(n, 1, seed=3)[:, 0]
    x = np.zeros(n)
    K.solve(x, b)
    assert M.scaled_backward_error(A, x.reshape(n, 1), b.reshape(n, 1)) <= BERR

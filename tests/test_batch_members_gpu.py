"""Active members of a uniform batch on the GPU: ``ubatch_index`` and ``ubatch_mask`` restrict the
factorization and the solve to a subset of the members (src/solver.jl:145-148, 694-705;
set_members!, src/numeric/storage.jl:290-306), and the other members' factors and solutions are left
as they are.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from sdsb200 import matrices as M

pytestmark = pytest.mark.gpu

BERR = 1e-12


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def test_ubatch_mask_refactor_and_solve(torch_cuda):
    from sdsb200.solver import DirectSolver, InvalidValueError

    A = M.lap2d_shifted(12, 12, seed=1)
    n, nb = A.shape[0], 5
    vals = M.batch_members(A, nb, spread=0.1, seed=2)
    ds = DirectSolver((A.indptr, A.indices, vals.reshape(-1), n), "SPD")
    ds.execute("analysis")
    assert list(ds.execute("factorization")) == [0] * nb
    b = M.rhs(n * nb, 1, seed=3).reshape(nb, n)
    x_all = ds.execute("solve", None, b).cpu().numpy()
    # new values for every member; refactor members 0, 2 and 4 only
    vals2 = M.batch_members(A, nb, spread=0.1, seed=9)
    ds.update(vals2.reshape(-1))
    mask = [1, 0, 1, 0, 1]
    ds.setparam("ubatch_mask", mask)
    ds.execute("refactorization")
    X = np.full((nb, n), 7.0)
    ds.execute("solve", X, b)
    for k in range(nb):
        if mask[k]:
            Ak = sp.csr_matrix((vals2[k], A.indices, A.indptr), shape=A.shape)
            assert M.scaled_backward_error(Ak, X[k].reshape(n, 1), b[k].reshape(n, 1)) <= BERR
        else:
            assert np.all(X[k] == 7.0)                     # an inactive member's solution: untouched
    # ubatch_index and ubatch_mask together: their intersection (member 4)
    ds.setparam("ubatch_index", 4)
    X = np.full((nb, n), 7.0)
    ds.execute("solve", X, b)
    assert np.all(X[:4] == 7.0) and not np.any(X[4] == 7.0)
    ds.setparam("ubatch_index", -1)
    # all members again: the inactive ones kept their old factors
    ds.setparam("ubatch_mask", None)
    x = ds.execute("solve", None, b).cpu().numpy()
    for k in (1, 3):
        assert np.array_equal(x[k], x_all[k])
    # a mask or an index outside the batch, or an empty selection: an error at the next phase
    ds.setparam("ubatch_mask", [1, 0, 1])
    with pytest.raises(InvalidValueError):
        ds.execute("refactorization")
    ds.setparam("ubatch_mask", [0] * nb)
    with pytest.raises(InvalidValueError):
        ds.execute("solve", None, b)
    ds.setparam("ubatch_mask", None)
    ds.setparam("ubatch_index", nb)
    with pytest.raises(InvalidValueError):
        ds.execute("refactorization")
    ds.setparam("ubatch_index", -1)
    assert ds.getparam("ubatch_mask") is None
    # memory_estimates: the plan's buffers in the reference's slots (every member's panels in slot 7)
    est = ds.getparam("memory_estimates")
    assert len(est) == 16 and est[1] >= est[0] > 0 and est[6] >= nb * 8 * A.nnz // 2
    # a vector right-hand side of a batch is member after member
    xv = ds.execute("solve", None, b.reshape(-1)).cpu().numpy()
    assert np.array_equal(xv.reshape(nb, n), x)

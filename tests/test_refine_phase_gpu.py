"""The "solve_refinement" phase on the GPU (_refine_phase!, src/solver.jl:902-926): a solution X from
the FP32 factor without refinement is refined in place against B, ir_n_steps steps of plain
refinement or FGMRES-IR, to a scaled backward error <= 1e-12; ir_n_steps = 0 leaves X as it is; X
and B must not alias. Cases: "SPD", "G" with A^T (solve_mode 1), and "G" with a matching (the
refinement runs on the matched system and X comes back in A's unknowns).
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


def _case(case):
    if case == "SPD":
        return M.lap2d_shifted(24, 24), "SPD", {}
    A = M.convection_diffusion3d(8, 8, 8, seed=4)
    if case == "G_match":
        rng = np.random.default_rng(5)
        n = A.shape[0]
        P = sp.csr_matrix((np.ones(n), (np.arange(n), rng.permutation(n))), shape=(n, n))
        A = (sp.diags(np.exp(rng.normal(0, 2, n))) @ P @ A).tocsr()
        A.sort_indices()
        return A, "G", dict(matching_alg="algo5", pivot_threshold=0.1)
    return A, "G", dict(pivot_threshold=0.1, solve_mode=1)


@pytest.mark.parametrize("case", ["SPD", "G_T", "G_match"])
@pytest.mark.parametrize("mode", ["ir", "fgmres"])
def test_solve_refinement_phase(torch_cuda, case, mode):
    from sdsb200.solver import DirectSolver, InvalidValueError

    A, structure, kw = _case(case)
    ds = DirectSolver(A, structure, factor_precision="fp32", ir_mode=mode, **kw)
    ds.execute("analysis")
    assert ds.execute("factorization") == 0
    AA = A.T.tocsr() if kw.get("solve_mode") == 1 else A
    b = M.rhs(A.shape[0], 2, seed=3)
    x0 = ds.execute("solve", None, b).cpu().numpy()
    assert M.scaled_backward_error(AA, x0, b) > 1e-13          # the FP32 factor alone
    X = x0.copy()
    assert ds.execute("solve_refinement", X, b) is X            # ir_n_steps = 0: X as it is
    assert np.array_equal(X, x0)
    ds.setparam("ir_n_steps", 6)
    ds.execute("solve_refinement", X, b)
    assert M.scaled_backward_error(AA, X, b) <= BERR
    assert 1 <= ds.getparam("ir_n_steps") <= 6
    # a device X refined in place, stopping at ir_tol
    ds.setparam("ir_tol", 1e-12)
    Xt = torch_cuda.from_numpy(x0.copy()).cuda()
    ds.execute("solve_refinement", Xt, b)
    assert M.scaled_backward_error(AA, Xt.cpu().numpy(), b) <= BERR
    with pytest.raises(InvalidValueError):
        ds.execute("solve_refinement", Xt, Xt)

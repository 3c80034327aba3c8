"""The "solve_refinement" loop on the host (CPU): plain iterative refinement of a given X
(refine!, src/solve/refinement.jl:359-397) with stand-ins for the residual and the factor solve.

The factor solve is an FP32 inverse of A, so each correction gains about six digits, as the FP32
factor does on the GPU. Checks: convergence to the FP64 accuracy, the early stop at ir_tol (checked
before each correction, so the steps counted are the corrections applied), nsteps = 0 leaving X as
it is, and an interrupt leaving the last completed iterate.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from sdsb200.refinement import ir_iterate  # noqa: E402


def _system(n=60, nrhs=3, seed=0):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) + n * np.eye(n)
    B = rng.uniform(-1, 1, (n, nrhs))
    inv32 = np.linalg.inv(A.astype(np.float32)).astype(np.float64)
    At = torch.from_numpy(A)
    Inv = torch.from_numpy(inv32)
    # column-major per right-hand side: (nrhs, n), as the C ABI's buffers
    residual = lambda X, Bc: Bc - X @ At.T           # noqa: E731  (row k of X is column k of X)
    solve = lambda R: R @ Inv.T                      # noqa: E731
    return A, B, residual, solve


def _rel(A, X, B):
    R = B - A @ X
    return max(np.linalg.norm(R[:, k]) / np.linalg.norm(B[:, k]) for k in range(B.shape[1]))


def test_plain_refinement_converges_and_counts():
    A, B, residual, solve = _system()
    Bc = torch.from_numpy(np.ascontiguousarray(B.T))
    X = solve(Bc).clone()
    assert _rel(A, X.numpy().T, B) > 1e-9
    steps, stopped = ir_iterate(residual, solve, X, Bc, A.shape[0], nsteps=5, tol=0.0)
    assert (steps, stopped) == (5, False)          # tol = 0 never stops early
    assert _rel(A, X.numpy().T, B) <= 1e-14
    # with a tolerance: stop as soon as the residual before a correction meets it
    X = solve(Bc).clone()
    steps, _ = ir_iterate(residual, solve, X, Bc, A.shape[0], nsteps=20, tol=1e-12)
    assert 1 <= steps <= 3
    assert _rel(A, X.numpy().T, B) <= 1e-12
    X2 = X.clone()
    steps, _ = ir_iterate(residual, solve, X2, Bc, A.shape[0], nsteps=20, tol=1e-12)
    assert steps == 0 and torch.equal(X, X2)       # already refined: no correction applied


def test_zero_steps_and_interrupt():
    A, B, residual, solve = _system(seed=1)
    Bc = torch.from_numpy(np.ascontiguousarray(B.T))
    X = solve(Bc).clone()
    X0 = X.clone()
    assert ir_iterate(residual, solve, X, Bc, A.shape[0], nsteps=0, tol=0.0) == (0, False)
    assert torch.equal(X, X0)
    polls = []

    def interrupted():
        polls.append(1)
        return len(polls) > 2                          # the third poll sees the flag

    steps, stopped = ir_iterate(residual, solve, X, Bc, A.shape[0], nsteps=10, tol=0.0, interrupted=interrupted)
    assert (steps, stopped) == (2, True)
    X2 = X0.clone()
    ir_iterate(residual, solve, X2, Bc, A.shape[0], nsteps=2, tol=0.0)
    assert torch.equal(X, X2)                          # X holds the last completed iterate

"""Uneven batches (GPU): many systems of different sizes and patterns in one plan.

The batch is one block-diagonal system. Its factorization is one level-batched launch sequence,
and its solve is one persistent launch. Every system must reach a scaled backward error <= 1e-12
on its own, and must match the same system solved alone.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from sdsb200 import matrices as M

pytestmark = pytest.mark.gpu

BERR = 1e-12
TOL = 1e-10


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def _systems(count, smin, smax, seed):
    return M.uneven_batch(count, smin, smax, 0.1, seed)


def _solve_batch(torch, systems, structure="SPD", **params):
    from sdsb200.batch import UnevenBatch

    ub = UnevenBatch(systems, structure, **params)
    ub.execute("analysis")
    assert np.all(np.asarray(ub.execute("factorization")) == 0)
    rng = np.random.default_rng(3)
    b = rng.uniform(-1, 1, ub.A.shape[0])
    x = ub.execute("solve", None, b).cpu().numpy()
    return ub, b, x


def test_uneven_batch_fp64_one_launch_solve(torch_cuda):
    systems = _systems(40, 8, 28, seed=1)
    ub, b, x = _solve_batch(torch_cuda, systems)
    assert ub.solver.plan_stat("launches_done") == 1          # the whole batch in one persistent launch
    errs = ub.backward_errors(x, b)
    assert errs.max() <= BERR
    from sdsb200.solver import DirectSolver

    for i in (0, 7, 39):
        one = DirectSolver(systems[i], "SPD")
        one.execute("analysis")
        one.execute("factorization")
        bi = b[ub.offsets[i]:ub.offsets[i + 1]]
        xi = one.execute("solve", None, bi).cpu().numpy()
        assert np.abs(xi - ub.split(x)[i]).max() <= TOL * max(1.0, np.abs(xi).max())


def test_uneven_batch_mixed_refinement(torch_cuda):
    systems = _systems(32, 10, 30, seed=2)
    ub, b, x = _solve_batch(torch_cuda, systems, factor_precision="fp32", ir_n_steps=3, ir_tol=0.0)
    assert ub.backward_errors(x, b).max() <= BERR


@pytest.mark.parametrize("structure", ["S", "G"])
def test_uneven_batch_indefinite_and_general(torch_cuda, structure):
    rng = np.random.default_rng(4)
    if structure == "S":
        systems = [M.kkt(int(s), int(s), int(s) * 2, seed=int(k)) for k, s in enumerate(rng.integers(5, 10, 12))]
        params = {}
    else:
        systems = [M.convection_diffusion3d(int(s), int(s), int(s), seed=int(k))
                   for k, s in enumerate(rng.integers(3, 7, 12))]
        params = dict(pivot_threshold=0.1)
    ub, b, x = _solve_batch(torch_cuda, systems, structure, **params)
    assert ub.backward_errors(x, b).max() <= BERR


def test_autotune_uneven_batch(torch_cuda):
    from sdsb200.autotune import autotune

    systems = _systems(64, 16, 48, seed=5)
    from sdsb200.batch import UnevenBatch

    ub = UnevenBatch(systems, "SPD")
    ub.execute("analysis")
    b = np.random.default_rng(6).uniform(-1, 1, ub.A.shape[0])
    times = autotune(ub.solver, b, reps=2, use_cache=False)
    assert len(times) >= 4
    best = min(times, key=times.get)
    assert ub.solver.params["tuning"] == best
    x = ub.execute("solve", None, b).cpu().numpy()
    assert ub.backward_errors(x, b).max() <= BERR

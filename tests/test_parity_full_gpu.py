"""Parity at the benchmark configurations' full sizes, and of the mixed (FP32-factor) form (GPU).

Same pattern as the reference's device tests (test/utils.jl:357-369): analyse once, factor with the
CPU oracle and on the device from the same Symbolic, and compare what must be exact (pivot order
and kinds, per-front statistics, inertia, perm_row / perm_col) and the values within a tolerance.

* The FP64 form: Cholesky panels within 1e-10 of the oracle (relative to max(1, max |entry|)); LDL^T
  and LU factors and D equal to the oracle's bit for bit (their updates are summed in its order).
* The mixed form (FP32 assembly, FP32 Schur updates as 3xTF32 on the tensor cores, FP32 panel steps):
  its factor against the FP64 oracle within 1e-5 relative, an FP32 bound. A factor with a broken
  hi/lo split (one TF32 term) or a wrong accumulator read-back is off by 1e-3 or more and fails it,
  even though refinement would still converge from it. LDL^T inertia must equal the FP64 oracle's.
* Full sizes: the lap3d 48^3 SPD workload (n = 110 592), the 40^3 LU convection-diffusion (n = 64 000)
  with perm_row / perm_col, the KKT on a 100 x 100 grid (n = 13 750) and the 1024-system uneven
  batch, against the threaded oracle (bit-identical to the serial one).
"""
import numpy as np
import pytest
import scipy.sparse as sp

from helpers import dense_panels, rel_max_diff, small_kkt
from sdsb200 import matrices as M

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10    # panels / D of the FP64 form, relative to max(1, max |entry|)
FP32_TOL = 1e-5     # panels / D of the FP32 factor against the FP64 oracle
BERR = 1e-12        # scaled backward error of every solve (FP64 form directly, mixed form after refinement)


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


@pytest.fixture(scope="module", autouse=True)
def oracle_threads():
    import os

    from oracle.oracle import set_threads

    set_threads(max(1, min(32, os.cpu_count() or 1)))
    yield
    set_threads(1)


def _oracle(ds, A, structure, **okw):
    from oracle.oracle import Oracle

    O = Oracle(ds.symbolic)
    info = O.factorize(A.data, structure, **okw)
    return O, info


def _inertia(O):
    st = O.stats_matrix()
    return int(st[:, 0].sum()), int(st[:, 1].sum())


def _solver(A, structure, **params):
    from sdsb200.solver import DirectSolver

    ds = DirectSolver(A, structure, **params)
    ds.execute("analysis")
    return ds


def _pair(A, structure, **params):
    """The FP64 and the mixed-form solver on one analysis."""
    d64 = _solver(A, structure, **params)
    d32 = _solver(A, structure, factor_precision="fp32", **params)
    assert np.array_equal(d32.symbolic.perm, d64.symbolic.perm)
    return d64, d32


def _check_panels(ds, S, O, tol, lu=False):
    fac, ufac = ds.factor_host()
    err = rel_max_diff(dense_panels(S, fac), dense_panels(S, O.factor))
    assert err <= tol, err
    if lu:
        uerr = rel_max_diff(dense_panels(S, ufac), dense_panels(S, O.ufactor))
        assert uerr <= tol, uerr
        err = max(err, uerr)
    return err


def _berr(ds, A, b, transpose=False):
    ds.setparam("solve_mode", int(transpose))
    x = ds.execute("solve", None, b).cpu().numpy().reshape(A.shape[0], -1)
    ds.setparam("solve_mode", 0)
    AA = A.T.tocsr() if transpose else A
    return M.scaled_backward_error(AA, x, b), x


# ---------------------------------------------------------------------------------------------------
# the mixed form's factor against the FP64 oracle


def test_mixed_spd_factor_wide_fronts(torch_cuda):
    # lap3d 24^3 with ND: fronts wider than 32 columns run the FP32 32-column steps and the 3xTF32
    # tensor-core Schur updates; the small fronts run the FP32 shared-memory kernel
    A = M.lap3d(24, 24, 24, seed=5)
    d32 = _solver(A, "SPD", reordering_alg="nd", factor_precision="fp32", ir_n_steps=10, ir_tol=1e-14)
    S = d32.symbolic
    assert int(S.front_ncols.max()) > 64 and int(S.front_nrows.max()) > 512
    assert d32.execute("factorization") == 0
    O, info = _oracle(d32, A, "SPD")
    assert info == 0
    err = _check_panels(d32, S, O, FP32_TOL)
    assert err > 1e-12          # the factor is FP32 arithmetic, not an FP64 copy
    assert np.array_equal(d32.stats_host(), O.stats_matrix())
    b = M.rhs(A.shape[0], 4, seed=6)
    e, _ = _berr(d32, A, b)
    assert e <= BERR


@pytest.mark.parametrize("case", ["kkt20", "kkt40_coop"])
def test_mixed_ldlt_inertia(torch_cuda, case):
    # Bunch-Kaufman LDL^T with an FP32 factor: the inertia must equal the FP64 oracle's. kkt40_coop
    # has fronts above 512 rows and 32 columns (the cooperative wide-front kernel).
    A = small_kkt(20, 20, 150, seed=2) if case == "kkt20" else small_kkt(40, 40, 600, seed=3)
    nh = 400 if case == "kkt20" else 1600
    nj = A.shape[0] - nh
    d32 = _solver(A, "S", factor_precision="fp32", ir_n_steps=10, ir_tol=1e-14)
    S = d32.symbolic
    O, info = _oracle(d32, A, "S")
    assert d32.execute("factorization") == info
    assert _inertia(O) == (nh, nj)
    assert d32.getparam("inertia") == _inertia(O)
    if case == "kkt40_coop":
        f, w = S.front_nrows.astype(int), S.front_ncols.astype(int)
        assert ((f > 512) & (w > 32)).any()
    piv, kind, d = d32.pivots_host()
    if np.array_equal(piv[: S.n], O.piv[: S.n]) and np.array_equal(kind[: S.n], O.kind[: S.n]):
        # same pivot sequence: D and the panels agree to FP32 accuracy, scaled by the growth of the
        # perturbed KKT pivots
        st = O.stats_matrix()
        if st[:, 3].sum() == 0:
            _check_panels(d32, S, O, FP32_TOL)
            assert rel_max_diff(d[: 2 * S.n], O.d[: 2 * S.n]) <= FP32_TOL
    if O.stats_matrix()[:, 3].sum() == 0:
        b = M.rhs(A.shape[0], 1, seed=4)
        e, _ = _berr(d32, A, b)
        assert e <= BERR


def test_mixed_lu_factor(torch_cuda):
    A = M.convection_diffusion3d(16, 16, 16, seed=16)
    d32 = _solver(A, "G", factor_precision="fp32", pivot_threshold=0.1, reordering_alg="nd", ir_n_steps=10,
                  ir_tol=1e-14)
    S = d32.symbolic
    O, info = _oracle(d32, A, "G", pivot_threshold=0.1)
    assert d32.execute("factorization") == info == 0
    piv, kind, d = d32.pivots_host()
    # diagonally dominant: threshold pivoting keeps every diagonal in both precisions
    assert np.array_equal(piv[: S.n], O.piv[: S.n])
    _check_panels(d32, S, O, FP32_TOL, lu=True)
    assert rel_max_diff(d[: S.n], O.d[: S.n]) <= FP32_TOL
    b = M.rhs(A.shape[0], 2, seed=5)
    for tr in (False, True):
        e, _ = _berr(d32, A, b, transpose=tr)
        assert e <= BERR


# ---------------------------------------------------------------------------------------------------
# the benchmark configurations at full size


def test_c2_lap3d48_full_size(torch_cuda):
    # lap3d 48^3 (n = 110 592), ND, 4 right-hand sides: both forms against the FP64 oracle
    A = M.lap3d(48, 48, 48, seed=0)
    d64, d32 = _pair(A, "SPD", reordering_alg="nd", max_nrhs=4, ir_n_steps=10, ir_tol=1e-14)
    S = d64.symbolic
    assert S.n == 110592
    assert d64.execute("factorization") == 0
    assert d32.execute("factorization") == 0
    O, info = _oracle(d64, A, "SPD")
    assert info == 0
    _check_panels(d64, S, O, FP64_TOL)
    _check_panels(d32, S, O, FP32_TOL)
    assert np.array_equal(d64.stats_host(), O.stats_matrix())
    b = M.rhs(A.shape[0], 4, seed=0)
    e64, x64 = _berr(d64, A, b)
    e32, x32 = _berr(d32, A, b)
    assert e64 <= BERR and e32 <= BERR
    # the refined solution against the FP64 one, per right-hand side
    for r in range(4):
        assert np.abs(x32[:, r] - x64[:, r]).max() <= 1e-10 * np.abs(x64[:, r]).max()


def test_c5_lu40_full_size(torch_cuda):
    # convection-diffusion 40^3 (n = 64 000), threshold 0.1: pivots, perm_row and perm_col bit-exact
    A = M.convection_diffusion3d(40, 40, 40, seed=0)
    ds = _solver(A, "G", pivot_threshold=0.1, reordering_alg="nd", max_nrhs=8)
    S = ds.symbolic
    assert S.n == 64000
    O, info = _oracle(ds, A, "G", pivot_threshold=0.1)
    assert ds.execute("factorization") == info == 0
    piv, kind, d = ds.pivots_host()
    assert np.array_equal(piv[: S.n], O.piv[: S.n])
    assert np.array_equal(kind[: S.n], O.kind[: S.n])
    assert np.array_equal(ds.stats_host(), O.stats_matrix())
    assert np.array_equal(ds.getparam("perm_row"), S.perm[O.piv[: S.n] - 1])
    assert np.array_equal(ds.getparam("perm_col"), S.perm)
    # every update summed in the oracle's order: L, U^T and D are the oracle's bit for bit
    fac, ufac = ds.factor_host()
    assert np.array_equal(fac, O.factor) and np.array_equal(ufac, O.ufactor)
    assert np.array_equal(d[: S.n], O.d[: S.n])
    b = M.rhs(A.shape[0], 8, seed=0)
    for tr in (False, True):
        e, _ = _berr(ds, A, b, transpose=tr)
        assert e <= BERR


def test_c3_kkt_grid100(torch_cuda):
    # the KKT of the benchmark's generator on a 100 x 100 grid (n = 13 750, 3 750 constraints): pivots,
    # kinds and statistics bit-exact, exact inertia in both forms
    A = M.kkt(100, 100, 3750, seed=0)
    d64, d32 = _pair(A, "S", ir_n_steps=20, ir_tol=1e-14)
    S = d64.symbolic
    O, info = _oracle(d64, A, "S")
    assert d64.execute("factorization") == info
    piv, kind, d = d64.pivots_host()
    assert np.array_equal(piv[: S.n], O.piv[: S.n])
    assert np.array_equal(kind[: S.n], O.kind[: S.n])
    assert np.array_equal(d64.stats_host(), O.stats_matrix())
    # the FP64 LDL^T sums every update in the oracle's order: factor and D are the oracle's bit for bit
    fac, _ = d64.factor_host()
    assert np.array_equal(fac, O.factor)
    assert np.array_equal(d[: 2 * S.n], O.d[: 2 * S.n])
    assert _inertia(O) == (10000, 3750)
    assert d64.getparam("inertia") == (10000, 3750)
    assert d32.execute("factorization") == info
    assert d32.getparam("inertia") == _inertia(O)
    b = M.rhs(A.shape[0], 1, seed=0)
    e64, _ = _berr(d64, A, b)
    e32, _ = _berr(d32, A, b)
    assert e64 <= BERR and e32 <= BERR


def test_c4_uneven_batch_1024(torch_cuda):
    # 1024 systems (2-D Laplacians on s x s grids, s ~ U[16, 48]) as one block-diagonal plan: every
    # system's panels against the oracle on the same analysis, in both forms, and every system's
    # backward error
    from sdsb200.batch import UnevenBatch

    systems = M.uneven_batch(1024, 16, 48, 0.1, 0)
    ub64 = UnevenBatch(systems, "SPD")
    ub64.execute("analysis")
    ub32 = UnevenBatch(systems, "SPD", factor_precision="fp32", ir_n_steps=4, ir_tol=0.0)
    ub32.solver.symbolic = ub64.solver.symbolic
    ub32.solver._stage = 1
    ub32.solver.replan()
    S = ub64.solver.symbolic
    A = ub64.A
    O, info = _oracle(ub64.solver, A, "SPD")
    assert info == 0
    assert np.all(np.asarray(ub64.execute("factorization")) == 0)
    assert np.all(np.asarray(ub32.execute("factorization")) == 0)
    # per system: the fronts of system k are those whose first column (1-based perm) lies in its block
    c0 = S.super_ptr[:-1].astype(np.int64) - 1
    owner = np.searchsorted(ub64.offsets, S.perm[c0].astype(np.int64) - 1, side="right") - 1
    assert owner.min() == 0 and owner.max() == 1023
    base = S.front_ptr[:-1].astype(np.int64) - 1
    size = S.front_nrows.astype(np.int64) * S.front_ncols.astype(np.int64)
    for ub, tol in ((ub64, FP64_TOL), (ub32, FP32_TOL)):
        fac, _ = ub.solver.factor_host()
        diff = np.abs(fac - O.factor)
        worst = np.zeros(1024)
        scale = np.ones(1024)
        for s in range(S.ns):
            seg = slice(base[s], base[s] + size[s])
            k = owner[s]
            worst[k] = max(worst[k], float(diff[seg].max(initial=0.0)))
            scale[k] = max(scale[k], float(np.abs(O.factor[seg]).max(initial=0.0)))
        assert (worst / scale).max() <= tol
    b = np.random.default_rng(3).uniform(-1, 1, A.shape[0])
    for ub in (ub64, ub32):
        x = ub.execute("solve", None, b).cpu().numpy()
        errs = ub.backward_errors(x, b)
        assert errs.shape == (1024,) and errs.max() <= BERR

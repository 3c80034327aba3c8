"""Parity of the B200 numeric phase with the CPU oracle (GPU).

Pattern of the reference's own device tests (test/utils.jl:357-369, 620-630,
797-808): analyse once, factor with the CPU oracle and on the device from the
same Symbolic, then compare exactly what must be exact (pivot order, pivot
kinds, per-front statistics, inertia, info) and the values within a growth
tolerance; solves must reach a scaled backward error <= 1e-12.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from helpers import dense_panels, eigen_inertia, oracle_for, rel_max_diff, small_kkt
from sdsb200 import matrices as M

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10   # panels / D relative to max(1, max|entry|)
BERR = 1e-12       # scaled backward error of every FP64 solve


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def _solver(A, structure, **params):
    from sdsb200.solver import DirectSolver

    return DirectSolver(A, structure, **params)


def _check_factor(A, structure, torch_cuda, okw=None, **params):
    okw = okw or {}
    S, O, info = oracle_for(A, structure, reordering=params.get("reordering_alg", "default"), **okw)
    ds = _solver(A, structure, **params)
    ds.execute("analysis")
    assert np.array_equal(ds.symbolic.perm, S.perm)
    dinfo = ds.execute("factorization")
    assert dinfo == info
    fac, ufac = ds.factor_host()
    assert rel_max_diff(dense_panels(S, fac), dense_panels(S, O.factor)) <= FP64_TOL
    if structure == "G":
        assert rel_max_diff(dense_panels(S, ufac), dense_panels(S, O.ufactor)) <= FP64_TOL
    if structure != "SPD":
        piv, kind, d = ds.pivots_host()
        assert np.array_equal(piv[: S.n], O.piv[: S.n])
        assert np.array_equal(kind[: S.n], O.kind[: S.n])
        assert rel_max_diff(d[: 2 * S.n], O.d[: 2 * S.n]) <= FP64_TOL
    st = ds.stats_host()
    assert np.array_equal(st, O.stats_matrix())
    return ds, S, O


def _check_solve(ds, A, nrhs=1, transpose=False):
    b = M.rhs(A.shape[0], nrhs, seed=1)
    if transpose:
        ds.setparam("solve_mode", 1)
    x = ds.execute("solve", None, b if nrhs > 1 else b[:, 0]).cpu().numpy()
    AA = A.T.tocsr() if transpose else A
    err = M.scaled_backward_error(AA, x.reshape(A.shape[0], -1), b)
    if transpose:
        ds.setparam("solve_mode", 0)
    return err


@pytest.mark.parametrize("reordering", ["amd", "nd"])
def test_cholesky_lap2d_64(torch_cuda, reordering):
    A = M.lap2d_shifted(64, 64, seed=0)
    ds, S, O = _check_factor(A, "SPD", torch_cuda, reordering_alg=reordering)
    assert _check_solve(ds, A, 1) <= BERR
    assert _check_solve(ds, A, 3) <= BERR


def test_cholesky_large_fronts(torch_cuda):
    # 3-D grid: the top separators exceed the shared-memory fronts (large-front dense path)
    A = M.lap3d(18, 18, 18, shift=0.05, seed=3)
    ds, S, O = _check_factor(A, "SPD", torch_cuda, reordering_alg="nd")
    assert int(S.front_nrows.max()) > 160
    assert _check_solve(ds, A, 4) <= BERR


def test_cholesky_refactorization_bitwise(torch_cuda):
    A = M.lap3d(14, 14, 14, seed=1)
    ds = _solver(A, "SPD", reordering_alg="nd")
    ds.execute("analysis")
    ds.execute("factorization")
    f1, _ = ds.factor_host()
    ds.execute("refactorization")
    f2, _ = ds.factor_host()
    assert np.array_equal(f1, f2)
    b = M.rhs(A.shape[0], 2, seed=4)
    x1 = ds.execute("solve", None, b).cpu().numpy()
    x2 = ds.execute("solve", None, b).cpu().numpy()
    assert np.array_equal(x1, x2)


def test_cholesky_failure_info(torch_cuda):
    A = M.lap2d_shifted(20, 20, seed=0).tolil()
    A[57, 57] = -5.0
    A = A.tocsr()
    S, O, info = oracle_for(A, "SPD", pivot_epsilon=0.0)
    assert info > 0
    ds = _solver(A, "SPD", pivot_epsilon=0.0)
    ds.execute("analysis")
    assert ds.execute("factorization") == info


@pytest.mark.parametrize("nx,nj", [(20, 150), (30, 400)])
def test_ldlt_kkt(torch_cuda, nx, nj):
    A = small_kkt(nx, nx, nj, seed=2)
    ds, S, O = _check_factor(A, "S", torch_cuda)
    inertia = ds.getparam("inertia")
    assert inertia == (nx * nx, nj)
    if A.shape[0] <= 2000:
        assert inertia == eigen_inertia(A)
    assert _check_solve(ds, A, 1) <= BERR


def test_ldlt_large_fronts_and_2x2(torch_cuda):
    # one dense front: BK with 2x2 pivots on the global-memory path
    A = small_kkt(14, 14, 90, seed=5)
    big = dict(amalgamation=(10_000, 100.0, 10_000))
    S, O, info = oracle_for(A, "S", amalgamation=big["amalgamation"])
    ds = _solver(A, "S", **big)
    ds.execute("analysis")
    assert ds.execute("factorization") == info
    piv, kind, d = ds.pivots_host()
    assert np.array_equal(piv[: S.n], O.piv[: S.n])
    assert np.array_equal(kind[: S.n], O.kind[: S.n])
    assert np.array_equal(ds.stats_host(), O.stats_matrix())
    fac, _ = ds.factor_host()
    assert rel_max_diff(dense_panels(S, fac), dense_panels(S, O.factor)) <= FP64_TOL
    assert ds.getparam("inertia") == eigen_inertia(A)
    assert _check_solve(ds, A, 2) <= BERR


def test_ldlt_pivot_sign_and_zero_pivot(torch_cuda):
    # a structurally singular diagonal block with epsilon = 0: info of the failed pivot
    A = sp.csr_matrix(np.array([[4.0, 1, 0, 0], [1, 3, 0, 0], [0, 0, 0, 0], [0, 0, 0, 2]]))
    A = A + sp.csr_matrix((np.zeros(1), ([2], [2])), shape=(4, 4))
    A.sort_indices()
    S, O, info = oracle_for(A, "S", pivot_epsilon=0.0, pivot_pairs="none")
    ds = _solver(A, "S", pivot_epsilon=0.0, pivot_pairs="none")
    ds.execute("analysis")
    assert ds.execute("factorization") == info != 0
    # with epsilon > 0 and a requested sign the pivot is perturbed to -eps
    psign = np.zeros(4, np.int8)
    psign[2] = -1
    S2, O2, info2 = oracle_for(A, "S", pivot_epsilon=1e-8, pivot_sign=psign, pivot_pairs="none")
    ds2 = _solver(A, "S", pivot_epsilon=1e-8, pivot_sign=psign, pivot_pairs="none")
    ds2.execute("analysis")
    assert ds2.execute("factorization") == info2 == 0
    assert ds2.getparam("npivots") == 1
    piv, kind, d = ds2.pivots_host()
    assert np.array_equal(kind[:4], O2.kind[:4])
    assert np.allclose(d[:8], O2.d[:8])


@pytest.mark.parametrize("g", [10, 16])
def test_lu_convection_diffusion(torch_cuda, g):
    A = M.convection_diffusion3d(g, g, g, seed=g)
    ds, S, O = _check_factor(A, "G", torch_cuda, okw=dict(pivot_threshold=0.1), pivot_threshold=0.1,
                             reordering_alg="nd")
    perm_row = ds.getparam("perm_row")
    assert np.array_equal(perm_row, S.perm[O.piv[: S.n] - 1])
    assert np.array_equal(ds.getparam("perm_col"), S.perm)
    assert _check_solve(ds, A, 2) <= BERR
    assert _check_solve(ds, A, 2, transpose=True) <= BERR


@pytest.mark.parametrize("case", ["kkt_ldlt", "cd_lu", "kkt_lu"])
def test_wide_fronts_many_chunks(torch_cuda, case):
    # fronts of more than two 256-row chunks, and (kkt_ldlt, cd_lu) of more than one 32-column group:
    # the chunked large-front assembly, and the cooperative kernel's per-chunk column maxima, update
    # items and deferred multiplier writes; kkt_lu also interchanges hundreds of rows
    if case == "kkt_ldlt":
        A, st, kw = small_kkt(40, 40, 600, seed=3), "S", {}
    elif case == "cd_lu":
        A, st, kw = M.convection_diffusion3d(28, 28, 28, seed=1), "G", dict(pivot_threshold=0.1, reordering_alg="nd")
    else:
        A, st, kw = small_kkt(40, 40, 600, seed=3), "G", dict(pivot_threshold=0.1)
    okw = {"pivot_threshold": kw["pivot_threshold"]} if st == "G" else {}
    if case == "kkt_lu":
        # LU of the KKT perturbs 189 zero pivots to +-eps, which grows entries to ~1e13. The FP64
        # contribution-block updates sum in the oracle's order, so the factors are still the oracle's
        # bit for bit.
        S, O, info = oracle_for(A, st, **okw)
        ds = _solver(A, st, **kw)
        ds.execute("analysis")
        assert np.array_equal(ds.symbolic.perm, S.perm)
        assert ds.execute("factorization") == info
        piv, kind, d = ds.pivots_host()
        assert np.array_equal(piv[: S.n], O.piv[: S.n])
        assert np.array_equal(kind[: S.n], O.kind[: S.n])
        assert np.array_equal(ds.stats_host(), O.stats_matrix())
        fac, ufac = ds.factor_host()
        assert np.array_equal(fac, O.factor)
        assert np.array_equal(ufac, O.ufactor)
    else:
        ds, S, O = _check_factor(A, st, torch_cuda, okw=okw, **kw)
    f, w = S.front_nrows.astype(int), S.front_ncols.astype(int)
    assert f.max() > 512
    if case != "kkt_lu":
        assert ((f > 512) & (w > 32)).any()
    else:
        assert (O.piv[: S.n] != np.arange(1, S.n + 1)).sum() > 100
    # a plain FP64 solve reaches the bound only without statically perturbed pivots (the KKT cases
    # perturb some: their parity is the factor's)
    exact = O.stats_matrix()[:, 3].sum() == 0
    if st == "G":
        assert np.array_equal(ds.getparam("perm_row"), S.perm[O.piv[: S.n] - 1])
        if exact:
            assert _check_solve(ds, A, 2) <= BERR
            assert _check_solve(ds, A, 2, transpose=True) <= BERR
    else:
        assert ds.getparam("inertia") == (1600, 600)
        if exact:
            assert _check_solve(ds, A, 2) <= BERR


def test_lu_row_swaps(torch_cuda):
    # weak diagonal: threshold pivoting must swap rows inside the fully-summed block
    rng = np.random.default_rng(7)
    A = M.convection_diffusion3d(8, 8, 8, seed=7).tolil()
    for i in range(0, A.shape[0], 5):
        A[i, i] = 0.05 * rng.uniform()
    A = A.tocsr()
    A.sort_indices()
    ds, S, O = _check_factor(A, "G", torch_cuda, okw=dict(pivot_threshold=0.5), pivot_threshold=0.5)
    piv = O.piv[: S.n]
    assert (piv != np.arange(1, S.n + 1)).any()
    assert _check_solve(ds, A, 1) <= BERR


def test_refinement_fp32_factor(torch_cuda):
    A = M.lap3d(16, 16, 16, seed=2)
    ds = _solver(A, "SPD", reordering_alg="nd", factor_precision="fp32", ir_n_steps=10, ir_tol=1e-14)
    ds.execute("analysis")
    assert ds.execute("factorization") == 0
    b = M.rhs(A.shape[0], 4, seed=3)
    x = ds.execute("solve", None, b).cpu().numpy()
    assert M.scaled_backward_error(A, x, b) <= BERR
    assert 1 <= ds.getparam("ir_n_steps") <= 10


def test_uniform_batch(torch_cuda):
    A = M.lap2d_shifted(24, 24, seed=0)
    nb = 6
    vals = M.batch_members(A, nb, spread=0.1, seed=1)
    ds = _solver((A.indptr, A.indices, vals.reshape(-1), A.shape[0]), "SPD")
    ds.execute("analysis")
    info = ds.execute("factorization")
    assert list(info) == [0] * nb
    b = M.rhs(A.shape[0] * nb, 1, seed=2).reshape(nb, A.shape[0], 1)
    x = ds.execute("solve", None, b).cpu().numpy().reshape(nb, A.shape[0], 1)
    for k in range(nb):
        Ak = sp.csr_matrix((vals[k], A.indices, A.indptr), shape=A.shape)
        assert M.scaled_backward_error(Ak, x[k], b[k]) <= BERR
    # ubatch_index: refactor one member only
    ds.setparam("ubatch_index", 3)
    ds.execute("refactorization")
    ds.setparam("ubatch_index", -1)


def test_phase_order_errors(torch_cuda):
    from sdsb200.solver import FactorizationError, InvalidValueError

    A = M.lap2d_shifted(8, 8)
    ds = _solver(A, "SPD")
    with pytest.raises(FactorizationError):
        ds.execute("factorization")
    ds.execute("analysis")
    with pytest.raises(FactorizationError):
        ds.execute("solve", None, np.ones(64))
    with pytest.raises(InvalidValueError):
        ds.setparam("pivot_threshold", -1.0)


@pytest.mark.parametrize("structure", ["SPD", "S", "G"])
def test_graph_replay_matches_eager(torch_cuda, structure):
    from sdsb200._native import numeric_lib

    A = {"SPD": lambda: M.lap3d(16, 16, 16, seed=4), "S": lambda: small_kkt(16, 16, 100, seed=4),
         "G": lambda: M.convection_diffusion3d(12, 12, 12, seed=4)}[structure]()
    b = M.rhs(A.shape[0], 2, seed=5)
    out = []
    for graphs in (0, 1):
        ds = _solver(A, structure, reordering_alg="nd", ir_n_steps=2)
        ds.execute("analysis")
        numeric_lib().sdsb200_set_graphs(ds._plan, graphs)
        for _ in range(2):  # second call replays the captured graph
            ds.execute("factorization")
            x = ds.execute("solve", None, b).cpu().numpy()
        out.append((ds.factor_host()[0], x, ds.stats_host()))
        assert M.scaled_backward_error(A, x, b) <= BERR
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])


@pytest.mark.parametrize("structure", ["SPD", "S", "G"])
def test_persistent_solve_matches_level_launches(torch_cuda, structure):
    from sdsb200._native import numeric_lib

    lib = numeric_lib()
    A = {"SPD": lambda: M.lap3d(20, 20, 20, seed=6), "S": lambda: small_kkt(22, 22, 200, seed=6),
         "G": lambda: M.convection_diffusion3d(14, 14, 14, seed=6)}[structure]()
    ds = _solver(A, structure, reordering_alg="nd", max_nrhs=4)
    ds.execute("analysis")
    ds.execute("factorization")
    b = M.rhs(A.shape[0], 3, seed=7)
    xs = []
    for mode in (1, 0):
        lib.sdsb200_set_persistent(ds._plan, mode)
        for tr in ((False, True) if structure == "G" else (False,)):
            ds.setparam("solve_mode", int(tr))
            x = ds.execute("solve", None, b).cpu().numpy()
            AA = A.T.tocsr() if tr else A
            assert M.scaled_backward_error(AA, x, b) <= BERR
            xs.append(x)
    assert lib.sdsb200_plan_stat(ds._plan, b"solve_status") == 0
    k = len(xs) // 2
    for x1, x0 in zip(xs[:k], xs[k:]):
        assert np.abs(x1 - x0).max() <= 1e-10 * np.abs(x0).max()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_dataflow_cholesky_steps_match_step_launches(torch_cuda, precision):
    # the large fronts' 32-column steps as dataflow tasks in one persistent launch per batch (tuning
    # steps = 1) against one launch per step and kernel: the same factor to rounding, the same statistics,
    # on several streams; and against the oracle
    from sdsb200.capi import tuning

    A = M.lap3d(20, 20, 20, seed=6)
    S, O, info = oracle_for(A, "SPD", reordering="nd")
    out = {}
    for steps in (0, 1):
        ds = _solver(A, "SPD", reordering_alg="nd", max_nrhs=4, factor_precision=precision,
                     tuning=tuning(0, 0, 0, 0, steps))
        ds.execute("analysis")
        assert ds.execute("factorization") == 0
        fac, _ = ds.factor_host()
        out[steps] = (dense_panels(S, fac), ds.stats_host())
        b = M.rhs(A.shape[0], 3, seed=7)
        x = ds.execute("solve", None, b).cpu().numpy()
        assert M.scaled_backward_error(A, x, b) <= (BERR if precision == "fp64" else 1e-5)
    tol = FP64_TOL if precision == "fp64" else 1e-5
    assert rel_max_diff(out[1][0], out[0][0]) <= tol
    assert np.array_equal(out[1][1], out[0][1])
    assert rel_max_diff(out[1][0], dense_panels(S, O.factor)) <= tol
    assert S.front_ncols.max() > 96   # several steps per front


@pytest.mark.parametrize("structure,precision", [("SPD", "fp64"), ("S", "fp64"), ("G", "fp64"), ("SPD", "fp32")])
def test_inverse_panels_match_block_chains(torch_cuda, structure, precision):
    # the dataflow solve's two forms for tiled fronts: inverse panels [L11^-1; L21 L11^-1] built after the
    # factorization (the default) and 64-column block chains; fronts wider than 64 and taller than 128
    # (several doubling levels, partial last blocks, partial-product chunks in both sweeps)
    from sdsb200.capi import tuning

    A = {"SPD": lambda: M.lap3d(20, 20, 20, seed=6),
         "S": lambda: small_kkt(30, 30, 400, seed=2),   # the well-conditioned KKT of test_ldlt_kkt
         "G": lambda: M.convection_diffusion3d(16, 16, 16, seed=6)}[structure]()
    b = M.rhs(A.shape[0], 3, seed=7)
    xs = {}
    for chains in (0, 1):
        ds = _solver(A, structure, reordering_alg="nd", max_nrhs=4, factor_precision=precision,
                     tuning=tuning(0, 0, chains))
        ds.execute("analysis")
        assert ds.execute("factorization") == 0
        if chains == 0:
            assert ds.symbolic.front_ncols.max() > 128 and ds.symbolic.front_nrows.max() > 256
        for tr in ((False, True) if structure == "G" else (False,)):
            ds.setparam("solve_mode", int(tr))
            x = ds.execute("solve", None, b).cpu().numpy()
            AA = A.T.tocsr() if tr else A
            berr = M.scaled_backward_error(AA, x, b)
            assert berr <= (BERR if precision == "fp64" else 1e-5), (chains, tr, berr)
            xs[chains, tr] = x
        assert ds.plan_stat("solve_status") == 0
    tol = 1e-10 if precision == "fp64" else 1e-4
    for tr in ((False, True) if structure == "G" else (False,)):
        assert rel_max_diff(xs[0, tr], xs[1, tr]) <= tol


@pytest.mark.parametrize("case", ["SPD", "G", "G_T", "S"])
def test_fgmres_refinement(torch_cuda, case):
    # FGMRES-IR with the FP32 factor as right preconditioner reaches the FP64 accuracy target, and
    # needs no more iterations than plain refinement
    if case == "SPD":
        A, st, kw = M.lap3d(16, 16, 16, seed=2), "SPD", dict(reordering_alg="nd")
    elif case.startswith("G"):
        A, st, kw = M.convection_diffusion3d(10, 10, 10, seed=2), "G", dict(pivot_threshold=0.1)
    else:
        A, st, kw = small_kkt(20, 20, 150, seed=2), "S", {}
    transpose = case == "G_T"
    b = M.rhs(A.shape[0], 2, seed=3)
    its = {}
    for mode in ("ir", "fgmres"):
        ds = _solver(A, st, factor_precision="fp32", ir_mode=mode, ir_n_steps=10, ir_tol=1e-13, **kw)
        ds.execute("analysis")
        ds.execute("factorization")
        if transpose:
            ds.setparam("solve_mode", 1)
        x = ds.execute("solve", None, b).cpu().numpy()
        AA = A.T.tocsr() if transpose else A
        assert M.scaled_backward_error(AA, x, b) <= BERR
        its[mode] = ds.getparam("ir_n_steps")
    assert 1 <= its["fgmres"] <= its["ir"]


def test_user_host_interrupt(torch_cuda):
    # user_host_interrupt (src/logging.jl:60-63): a set host flag stops a factorization and a
    # refinement loop with InterruptedError; cleared, the same plan factors and solves normally
    import ctypes as C

    from sdsb200.solver import InterruptedError_

    flag = C.c_int32(0)
    A = M.lap3d(12, 12, 12, seed=1)
    ds = _solver(A, "SPD", user_host_interrupt=flag, ir_n_steps=3, ir_tol=0.0)
    ds.execute("analysis")
    flag.value = 1
    with pytest.raises(InterruptedError_):
        ds.execute("factorization")
    flag.value = 0
    assert ds.execute("factorization") == 0
    b = M.rhs(A.shape[0], 1, seed=2)[:, 0]
    flag.value = 1
    with pytest.raises(InterruptedError_):
        ds.execute("solve", None, b)
    flag.value = 0
    x = ds.execute("solve", None, b).cpu().numpy()
    assert M.scaled_backward_error(A, x, b) <= BERR


@pytest.mark.parametrize("structure,precision", [("SPD", "fp64"), ("SPD", "fp32"), ("S", "fp64"), ("S", "fp32"),
                                                 ("G", "fp64")])
def test_fused_subtrees_match_level_launches(torch_cuda, structure, precision):
    # fused subtrees (one CTA factors a whole subtree of shared-memory fronts in postorder; at most 16
    # fronts each, and at most 4) against one launch per level and size class (tuning subtree = 15): the
    # same panels, pivots, kinds, D and statistics bit for bit; the oracle's pivots and statistics in
    # FP64, and its inertia in FP32. The default (subtree = 0) fuses none.
    from sdsb200.capi import tuning

    A, reordering = {"SPD": lambda: (M.lap2d_shifted(40, 40, seed=3), "amd"),
                     "S": lambda: (small_kkt(30, 30, 400, seed=2), "nd"),
                     "G": lambda: (M.convection_diffusion3d(12, 12, 12, seed=6), "nd")}[structure]()
    S, O, info = oracle_for(A, structure, reordering=reordering)
    out = {}
    for sub in (15, 4, 2, 0):
        ir = {} if precision == "fp64" else dict(ir_n_steps=10, ir_tol=1e-14)
        ds = _solver(A, structure, reordering_alg=reordering, max_nrhs=1, factor_precision=precision,
                     tuning=tuning(subtree=sub), **ir)
        ds.execute("analysis")
        assert ds.execute("factorization") == info
        fac, ufac = ds.factor_host()
        piv, kind, d = ds.pivots_host()
        out[sub] = dict(fac=fac, ufac=ufac, piv=piv, kind=kind, d=d, st=ds.stats_host(),
                        nsub=ds.plan_stat("subtrees"), nfr=ds.plan_stat("subtree_fronts"))
        b = M.rhs(A.shape[0], 1, seed=7)
        x = ds.execute("solve", None, b[:, 0]).cpu().numpy()
        assert M.scaled_backward_error(A, x.reshape(-1, 1), b) <= BERR
    assert out[15]["nsub"] == 0 and out[0]["nsub"] == 0
    assert out[4]["nsub"] > 0 and out[2]["nsub"] > out[4]["nsub"]
    assert out[4]["nfr"] > out[4]["nsub"]   # subtrees of several fronts
    for sub in (4, 2, 0):
        for k in ("fac", "piv", "kind", "d", "st"):
            assert np.array_equal(out[sub][k], out[15][k]), (sub, k)
        if structure == "G":
            assert np.array_equal(out[sub]["ufac"], out[15]["ufac"])
    n = S.n
    if precision == "fp64":
        assert rel_max_diff(dense_panels(S, out[4]["fac"]), dense_panels(S, O.factor)) <= FP64_TOL
        assert np.array_equal(out[4]["st"], O.stats_matrix())
        if structure != "SPD":
            assert np.array_equal(out[4]["piv"][:n], O.piv[:n])
            assert np.array_equal(out[4]["kind"][:n], O.kind[:n])
    else:
        assert np.array_equal(out[4]["st"][:, :2].sum(0), O.stats_matrix()[:, :2].sum(0))


@pytest.mark.parametrize("structure,precision", [("SPD", "fp64"), ("S", "fp64"), ("G", "fp64"), ("SPD", "fp32")])
def test_batch_dataflow_solve_matches_level_sweeps(torch_cuda, structure, precision):
    # a uniform batch solved by the one-launch dataflow solve (every active member's tasks in one launch,
    # block chains for the tiled fronts) against the per-level sweeps: all members, 10 right-hand sides
    # (two groups of the launch), A^T for LU, and a subset of the members
    from sdsb200._native import numeric_lib

    lib = numeric_lib()
    A = {"SPD": lambda: M.lap3d(12, 12, 12, seed=6), "S": lambda: small_kkt(16, 16, 100, seed=2),
         "G": lambda: M.convection_diffusion3d(10, 10, 10, seed=6)}[structure]()
    nb, n, nrhs = 5, A.shape[0], 10
    vals = M.batch_members(A, nb, spread=0.1, seed=3)
    ir = {} if precision == "fp64" else dict(ir_n_steps=10, ir_tol=1e-14)
    ds = _solver((A.indptr, A.indices, vals.reshape(-1), n), structure, reordering_alg="nd", max_nrhs=nrhs,
                 factor_precision=precision, **ir)
    ds.execute("analysis")
    assert list(ds.execute("factorization")) == [0] * nb
    b = np.random.default_rng(4).uniform(-1, 1, (nb, n, nrhs))
    out = {}
    for mode in (1, 0):
        lib.sdsb200_set_persistent(ds._plan, mode)
        for tr in ((False, True) if structure == "G" else (False,)):
            ds.setparam("solve_mode", int(tr))
            x = ds.execute("solve", None, b).cpu().numpy().reshape(nb, n, nrhs)
            for k in range(nb):
                Ak = sp.csr_matrix((vals[k], A.indices, A.indptr), shape=A.shape)
                assert M.scaled_backward_error(Ak.T.tocsr() if tr else Ak, x[k], b[k]) <= BERR
            out[mode, tr] = x
    ds.setparam("solve_mode", 0)
    assert lib.sdsb200_plan_stat(ds._plan, b"solve_status") == 0
    for key in out:
        if key[0] == 1:
            x1, x0 = out[key], out[0, key[1]]
            assert np.abs(x1 - x0).max() <= (1e-10 if precision == "fp64" else 1e-9) * np.abs(x0).max()
    # a subset of the members: the others' X is kept
    lib.sdsb200_set_persistent(ds._plan, 1)
    ds.setparam("ubatch_index", 2)
    x0 = np.zeros((nb, n, nrhs))
    xs = ds.execute("solve", x0, b)
    xs = (xs.cpu().numpy() if hasattr(xs, "cpu") else np.asarray(xs)).reshape(nb, n, nrhs)
    ds.setparam("ubatch_index", -1)
    assert np.abs(xs[2] - out[1, False][2]).max() <= 1e-12 * np.abs(out[1, False][2]).max() + 1e-300
    assert not np.any(xs[[0, 1, 3, 4]])


"""Host-side plumbing of DirectSolver (CPU, device="cpu"; no numeric library call): the layouts of
right-hand sides (a batch's are member after member, whatever the shape), the inactive members' part
of X kept by a subset solve, and the checks of the Schur and batch parameters."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from sdsb200 import matrices as M  # noqa: E402
from sdsb200.solver import DirectSolver, InvalidValueError  # noqa: E402


def _batch(nb):
    A = M.lap2d_shifted(4, 4)
    vals = M.batch_members(A, nb, spread=0.1, seed=1)
    return DirectSolver((A.indptr, A.indices, vals.reshape(-1), A.shape[0]), "SPD", device="cpu"), A.shape[0]


def test_colmajor_layouts():
    ds, n = _batch(1)
    b = np.arange(n * 2, dtype=np.float64).reshape(n, 2)
    cm, nrhs, back = ds._colmajor(b)
    assert nrhs == 2 and tuple(cm.shape) == (2, n) and cm.is_contiguous()
    assert np.array_equal(cm[1].numpy(), b[:, 1])
    assert np.array_equal(back(cm).numpy(), b)
    cm, nrhs, back = ds._colmajor(b[:, 0].copy())
    assert nrhs == 1 and np.array_equal(back(cm).numpy(), b[:, 0])
    ds3, n = _batch(3)
    v = np.arange(3 * n, dtype=np.float64)                    # member after member
    cm, nrhs, back = ds3._colmajor(v)
    assert nrhs == 1 and tuple(cm.shape) == (3, 1, n)
    assert np.array_equal(cm[2, 0].numpy(), v[2 * n:3 * n])
    assert np.array_equal(back(cm).numpy(), v)
    B = np.arange(3 * n * 2, dtype=np.float64).reshape(3, n, 2)
    cm, nrhs, back = ds3._colmajor(B)
    assert nrhs == 2 and np.array_equal(cm[1, 0].numpy(), B[1, :, 0])
    assert np.array_equal(back(cm).numpy(), B)


def test_subset_keeps_inactive_members():
    ds, n = _batch(4)
    ds.setparam("ubatch_mask", [1, 0, 0, 1])                   # no plan yet: stored, applied at analysis
    assert ds._members() == [0, 3]
    X = np.full((4, n), 7.0)
    out = torch.arange(4 * n, dtype=torch.float64).reshape(4, n)
    kept = ds._keep_inactive(X, out).numpy()
    assert np.array_equal(kept[[0, 3]], out.numpy()[[0, 3]])
    assert np.all(kept[[1, 2]] == 7.0)
    ds.setparam("ubatch_mask", None)
    ds.setparam("ubatch_index", 2)
    assert ds._members() == [2]
    with pytest.raises(InvalidValueError):
        ds.setparam("ubatch_mask", [1, 2, 0, 1])


def test_schur_parameter_checks():
    A = M.lap2d_shifted(4, 4)
    with pytest.raises(InvalidValueError):
        DirectSolver(A, "SPD", device="cpu", schur_mode=2)
    with pytest.raises(InvalidValueError):
        DirectSolver(A, "SPD", device="cpu", user_schur_indices=np.ones(5))
    with pytest.raises(InvalidValueError):
        DirectSolver(A, "SPD", device="cpu", user_schur_indices=np.full(16, 2))
    ds = DirectSolver(A, "SPD", device="cpu", schur_mode=1, user_schur_indices=np.eye(1, 16, 3).ravel())
    assert ds.getparam("schur_mode") == 1
    with pytest.raises(InvalidValueError):
        ds.setparam("schur_matrix", None)                       # no analysis with schur_mode = 1 yet


def test_member_selection_checked_at_the_next_phase():
    """As the reference's _set_members!: setparam stores ubatch_index / ubatch_mask as given, and the next
    factorization or solve raises InvalidValueError for a selection outside the batch or an empty one.
    A stand-in plan handle is enough here: the selection is checked before any call into the library."""
    import ctypes

    ds, n = _batch(4)
    ds.setparam("ubatch_index", 4)                              # outside 0:3, stored
    assert ds.getparam("ubatch_index") == 4
    ds._plan = ctypes.c_void_p(1)
    try:
        with pytest.raises(InvalidValueError):
            ds._sync_members()
        ds.setparam("ubatch_index", -1)
        ds.setparam("ubatch_mask", [0, 0, 0, 0])
        with pytest.raises(InvalidValueError):
            ds._sync_members()
        ds.setparam("ubatch_mask", [1, 0])
        with pytest.raises(InvalidValueError):
            ds._sync_members()
    finally:
        ds._plan = None


def test_reordering_then_symbolic_factorization():
    """The analysis phases as the reference splits them (src/solver.jl:444-452, 609-612, 1082-1085):
    "reordering" alone gives the ordering algorithm's permutation as perm_reorder_row, and
    "symbolic_factorization" without it is a FactorizationError. ("reordering" is host work only: no
    device is needed.)"""
    from sdsb200.analysis import analyze_csr
    from sdsb200.solver import FactorizationError

    A = M.lap2d_shifted(8, 8)
    ds = DirectSolver(A, "SPD", device="cpu", reordering_alg="nd")
    with pytest.raises(FactorizationError):
        ds.execute("symbolic_factorization")
    assert ds.execute("reordering") is None
    S = analyze_csr(A, "SPD", reordering="nd")
    assert np.array_equal(ds.getparam("perm_reorder_row"), S.ordering)
    assert sorted(ds.getparam("perm_reorder_col")) == list(range(1, 65))

"""The oracle's level-parallel factorization (oracle_set_threads) equals its serial postorder (CPU)."""
import numpy as np
import pytest

from helpers import oracle_for, small_kkt
from oracle import oracle as orc
from sdsb200 import matrices as M


@pytest.fixture
def threads():
    yield orc.set_threads
    orc.set_threads(1)


@pytest.mark.parametrize("structure", ["SPD", "S", "G"])
def test_threads_equal_serial(threads, structure):
    A, kw, okw = {
        "SPD": (M.lap3d(12, 12, 12, shift=0.05, seed=1), {"reordering": "nd"}, {}),
        "S": (small_kkt(16, 16, 100, seed=2), {}, {}),
        "G": (M.convection_diffusion3d(10, 10, 10, seed=3), {"reordering": "nd"}, {"pivot_threshold": 0.1}),
    }[structure]
    threads(1)
    S, O1, info1 = oracle_for(A, structure, **kw, **okw)
    out1 = (O1.factor.copy(), O1.ufactor.copy(), O1.d.copy(), O1.piv.copy(), O1.kind.copy(), O1.stats.copy())
    threads(8)
    O8 = orc.Oracle(S)
    info8 = O8.factorize(A.data, structure, **okw)
    out8 = (O8.factor, O8.ufactor, O8.d, O8.piv, O8.kind, O8.stats)
    assert info8 == info1
    for a, b in zip(out1, out8):
        assert np.array_equal(a, b)


def test_threads_first_failed_pivot(threads):
    # an indefinite matrix given to Cholesky: the first failed column in postorder, as the serial order
    A = M.lap3d(8, 8, 8, shift=0.05, seed=4).tolil()
    A[100, 100] = -1.0
    A[300, 300] = -1.0
    A = A.tocsr()
    threads(1)
    S, O1, info1 = oracle_for(A, "SPD")
    threads(8)
    info8 = orc.Oracle(S).factorize(A.data, "SPD")
    assert info1 != 0 and info8 == info1


def test_threads_dense_front(threads):
    # one dense 1200 x 1200 front with 300 rows below: the threaded potrf, trsm and syrk loops
    rng = np.random.default_rng(5)
    G = rng.normal(size=(1200, 1200))
    D = G @ G.T / 1200 + np.eye(1200)
    import scipy.sparse as sp

    B = sp.random(300, 1200, density=0.05, random_state=5) * 0.1
    A = sp.bmat([[sp.csr_matrix(D), B.T], [B, sp.eye(300) * 50.0]], format="csr")
    threads(1)
    S, O1, info1 = oracle_for(A, "SPD", reordering="natural")
    f1 = O1.factor.copy()
    threads(8)
    O8 = orc.Oracle(S)
    assert O8.factorize(A.data, "SPD") == info1 == 0
    assert np.array_equal(O8.factor, f1)


def test_blas_port_matches_oracle():
    """The benchmark's CPU baseline (the reference's CPU Cholesky over threaded LAPACK/BLAS) agrees
    with the bit-exact scalar oracle to rounding, and solves to a backward error <= 1e-12."""
    from oracle.blas_port import CholeskyPort
    from sdsb200 import analyze_csr

    A = M.lap3d(16, 16, 16, shift=0.02, seed=6)
    S = analyze_csr(A, "SPD", reordering="nd")
    O = orc.Oracle(S)
    assert O.factorize(A.data, "SPD") == 0
    P = CholeskyPort(S)
    assert P.factorize(A.data) == 0
    assert np.abs(P.factor - O.factor).max() <= 1e-13 * np.abs(O.factor).max()
    b = M.rhs(A.shape[0], 3, seed=7)
    assert M.scaled_backward_error(A, P.solve(b), b) <= 1e-12
    # an indefinite matrix: the same first failed pivot as the oracle
    B = A.tolil()
    B[50, 50] = -1.0
    B = B.tocsr()
    S2 = analyze_csr(B, "SPD", reordering="nd")
    assert CholeskyPort(S2).factorize(B.data) == orc.Oracle(S2).factorize(B.data, "SPD") != 0

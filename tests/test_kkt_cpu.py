"""KKTSolver option checks (CPU): the errors of the reference's constructor (src/kkt.jl:162-183),
raised before any device work."""
import pytest
import scipy.sparse as sp

from sdsb200.kkt import KKTSolver
from sdsb200.solver import InvalidValueError, NotSupportedError

A = sp.eye(4, format="csr")


@pytest.mark.parametrize("kw,err", [
    (dict(factorization="qr"), InvalidValueError),
    (dict(pivoting="full"), InvalidValueError),
    (dict(pivoting="bk"), InvalidValueError),                                  # needs 'ldl'
    (dict(factorization="ldl", pivoting="bk", fused=True), InvalidValueError),
    (dict(factorization="ldl", pivot_threshold=0.1), InvalidValueError),       # needs 'diagonal' or 'bk'
    (dict(pivot_sign=[1, 1, 1, 1]), InvalidValueError),                        # needs 'ldl'
    (dict(factorization="ldl", matching="algo9"), InvalidValueError),
    (dict(matching="algo5"), InvalidValueError),                               # needs 'ldl'
    (dict(factorization="ldl", fused=True), NotSupportedError),                # no fused pipeline here
])
def test_option_errors(kw, err):
    with pytest.raises(err):
        KKTSolver(A, "L", **kw)

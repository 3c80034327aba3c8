"""Generate tests/golden/dense_fronts.json: known-answer single-front factorizations.

The answers come from LAPACK through numpy/scipy (dense Cholesky, partial-
pivoting LU, LDL^T without interchanges), independently of the oracle, for
matrices whose analysis is one dense front in natural order (the oracle then
performs exactly the dense factorization of the reference's in-front code).
Run: python tests/golden/make_golden.py
"""
import json
import os

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp


def csr(A):
    S = sp.csr_matrix(A)
    S.sort_indices()
    # keep every position of the dense matrix (explicit zeros included)
    full = np.ones_like(A, dtype=bool)
    r, c = np.nonzero(full)
    S = sp.csr_matrix((A[r, c], (r, c)), shape=A.shape)
    S.sort_indices()
    return dict(n=A.shape[0], data=S.data.tolist(), indices=S.indices.tolist(), indptr=S.indptr.tolist())


def main():
    rng = np.random.default_rng(20261203)
    cases = []
    # SPD 6x6
    B = rng.standard_normal((6, 6))
    A = B @ B.T + 6 * np.eye(6)
    cases.append(dict(structure="SPD", L=np.linalg.cholesky(A).tolist(), **csr(A)))
    # LU with partial pivoting (u = 1 is LAPACK's rule), 5x5 with a weak diagonal
    A = rng.standard_normal((5, 5))
    A[np.diag_indices(5)] *= 0.05
    lu, ipiv = sla.lu_factor(A)
    order = list(range(5))
    for k, p in enumerate(ipiv):
        order[k], order[p] = order[p], order[k]
    L = np.tril(lu, -1) + np.eye(5)
    U = np.triu(lu)
    assert np.allclose(L @ U, A[order])
    cases.append(dict(structure="G", u=1.0, piv=[k + 1 for k in order], L=L.tolist(), DU=U.tolist(), **csr(A)))
    # LDL^T without interchanges (diagonally dominant indefinite)
    A = rng.standard_normal((5, 5))
    A = A + A.T
    A[np.diag_indices(5)] = np.array([9.0, -8.0, 10.0, -9.0, 8.0])
    Lf, D, perm = sla.ldl(A, lower=True)
    assert list(perm) == list(range(5)) and np.count_nonzero(D - np.diag(np.diag(D))) == 0
    d = np.concatenate([np.diag(D), np.zeros(5)])
    cases.append(dict(structure="S", kind=[1] * 5, d=d.tolist(), **csr(A)))
    # 2x2 pivot: [[0, 1], [1, 0]]
    A = np.array([[0.0, 1.0], [1.0, 0.0]])
    cases.append(dict(structure="S", kind=[2, 3], d=[0.0, 0.0, 1.0, 0.0], **csr(A)))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dense_fronts.json")
    with open(out, "w") as fh:
        json.dump(cases, fh, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main()

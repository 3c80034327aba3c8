"""Seeded synthetic matrices of the benchmark configurations and tests.

Generator semantics follow the reference's test generators
(SparseDirectSolver.jl test/matrices.jl: laplacian2d/3d :40-55, kkt_matrix
:143-160, batch_members :403-411); sizes and value distributions follow the
workloads the numeric phase is measured on. All return scipy CSR matrices
(0-based, sorted indices, full storage).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _lap1d(n):
    return sp.diags([-np.ones(n - 1), 2 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1], format="csr")


def laplacian2d(nx, ny):
    """5-point Laplacian, Dirichlet, row-major grid numbering (diag 4, off-diagonals -1)."""
    return (sp.kron(sp.eye(ny), _lap1d(nx)) + sp.kron(_lap1d(ny), sp.eye(nx))).tocsr()


def laplacian3d(nx, ny, nz):
    """7-point Laplacian, Dirichlet (diag 6, off-diagonals -1)."""
    Ix, Iy, Iz = sp.eye(nx), sp.eye(ny), sp.eye(nz)
    Lx, Ly, Lz = _lap1d(nx), _lap1d(ny), _lap1d(nz)
    A = sp.kron(Iz, sp.kron(Iy, Lx)) + sp.kron(Iz, sp.kron(Ly, Ix)) + sp.kron(Lz, sp.kron(Iy, Ix))
    return A.tocsr()


def _sorted(A):
    A = sp.csr_matrix(A)
    A.sum_duplicates()
    A.sort_indices()
    return A


def lap2d_shifted(nx, ny, shift=0.1, seed=0):
    """Laplacian plus a seeded diagonal shift U[0, shift]."""
    rng = np.random.default_rng(seed)
    A = laplacian2d(nx, ny) + sp.diags(rng.uniform(0.0, shift, nx * ny))
    return _sorted(A)


def lap3d(nx, ny, nz, shift=0.0, seed=0):
    rng = np.random.default_rng(seed)
    A = laplacian3d(nx, ny, nz)
    if shift > 0:
        A = A + sp.diags(rng.uniform(0.0, shift, nx * ny * nz))
    return _sorted(A)


def kkt(nx=200, ny=200, nj=15000, nnz_per_row=3, delta=0.0, seed=0):
    """[H J^T; J -delta I], H = 2-D Laplacian + U[0,1] diagonal, J random (3 N(0,1) entries per row).

    The (2,2) block is stored (explicit zeros when delta = 0), as the KKT
    systems of an interior-point solver store it.
    """
    rng = np.random.default_rng(seed)
    nh = nx * ny
    H = laplacian2d(nx, ny) + sp.diags(rng.uniform(0.0, 1.0, nh))
    rows = np.repeat(np.arange(nj), nnz_per_row)
    cols = np.empty(nj * nnz_per_row, dtype=np.int64)
    for i in range(nj):
        cols[i * nnz_per_row:(i + 1) * nnz_per_row] = rng.choice(nh, nnz_per_row, replace=False)
    vals = rng.standard_normal(nj * nnz_per_row)
    J = sp.csr_matrix((vals, (rows, cols)), shape=(nj, nh))
    D = sp.diags(np.full(nj, -float(delta)))
    K = sp.bmat([[H, J.T], [J, D]], format="csr")
    # keep the explicit zero diagonal of the dual block in the pattern
    K = K + sp.csr_matrix((np.zeros(nj), (np.arange(nh, nh + nj), np.arange(nh, nh + nj))), shape=K.shape)
    K = sp.csr_matrix(K)
    K.sort_indices()
    return K


def convection_diffusion3d(nx, ny, nz, beta=0.4, seed=0):
    """7-point convection-diffusion: diag 6 + U[0, 0.5], off-diagonals -1 +/- beta * (unit wind component)."""
    rng = np.random.default_rng(seed)
    wind = rng.standard_normal(3)
    wind /= np.linalg.norm(wind)
    n = nx * ny * nz
    idx = np.arange(n).reshape(nz, ny, nx)
    rows, cols, vals = [np.arange(n)], [np.arange(n)], [6.0 + rng.uniform(0.0, 0.5, n)]
    for axis, wa in zip((2, 1, 0), wind):
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[axis] = slice(0, -1)
        hi[axis] = slice(1, None)
        a, b = idx[tuple(lo)].ravel(), idx[tuple(hi)].ravel()
        rows += [a, b]
        cols += [b, a]
        vals += [np.full(a.size, -1.0 + beta * wa), np.full(a.size, -1.0 - beta * wa)]
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    return _sorted(A)


def batch_members(A, nb, spread=0.1, seed=0):
    """Uniform batch: member 0 is A, member k the congruence D A D, D in [1 - spread, 1 + spread]."""
    rng = np.random.default_rng(seed)
    A = _sorted(A)
    r = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    out = [A.data.copy()]
    for _ in range(1, nb):
        d = rng.uniform(1.0 - spread, 1.0 + spread, A.shape[0])
        out.append(A.data * d[r] * d[A.indices])
    return np.stack(out)


def uneven_batch(count=1024, smin=16, smax=48, shift=0.1, seed=0):
    """Distinct 2-D Laplacians on s x s grids, s ~ U[smin, smax], each + U[0, shift] diagonal."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(smin, smax + 1, count)
    return [lap2d_shifted(int(s), int(s), shift, seed=seed + 1 + k) for k, s in enumerate(sizes)]


def rhs(n, nrhs=1, seed=0):
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1.0, 1.0, (n, nrhs))
    return np.asfortranarray(b)


def scaled_backward_error(A, x, b):
    """max over columns of ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf)."""
    x = np.asarray(x).reshape(A.shape[0], -1)
    b = np.asarray(b).reshape(A.shape[0], -1)
    r = b - A @ x
    anorm = abs(A).sum(axis=1).max()
    err = np.abs(r).max(axis=0) / (anorm * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))
    return float(err.max())

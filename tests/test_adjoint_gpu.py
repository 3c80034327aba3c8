"""Differentiation of the solve (GPU): x = A^{-1} b, gradients of a scalar loss c^T x.

The reference has no automatic differentiation. The checks follow the pins for this form:
* central finite differences, h = 1e-6, on seeded entries of the values and of b, agreeing to 1e-6
  relative (to the largest gradient entry);
* a gradient built from the reference-semantics transposed solve: b_bar = A^{-T} c from the CPU
  oracle (ref_solve_lu! with transpose for "G", the symmetric solve otherwise) and A_bar = -b_bar x^T
  on the entries the factorization reads.
"""
import numpy as np
import pytest

from helpers import oracle_for, small_kkt
from sdsb200 import matrices as M

pytestmark = pytest.mark.gpu

FD_H = 1e-6
FD_TOL = 1e-6      # relative to max |gradient|
ORACLE_TOL = 1e-10


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


CASES = {
    "SPD": (lambda: M.lap2d_shifted(10, 10, seed=3), dict()),
    # a KKT whose factorization perturbs no pivot: with a perturbed pivot the solve is of a nearby
    # matrix and finite differences of A^{-1} b no longer apply
    "S": (lambda: small_kkt(10, 10, 30, seed=3), dict()),
    "G": (lambda: M.convection_diffusion3d(5, 5, 5, seed=3), dict(pivot_threshold=0.1)),
}


def _setup(torch, structure):
    from sdsb200.solver import DirectSolver

    make, params = CASES[structure]
    A = make()
    ds = DirectSolver(A, structure, **params)
    ds.execute("analysis")
    rng = np.random.default_rng(7)
    nz = torch.tensor(A.data, dtype=torch.float64, device="cuda")
    b = torch.tensor(rng.uniform(-1, 1, A.shape[0]), dtype=torch.float64, device="cuda")
    c = torch.tensor(rng.standard_normal(A.shape[0]), dtype=torch.float64, device="cuda")
    return A, ds, nz, b, c


def _grads(torch, ds, nz, b, c, **kw):
    from sdsb200 import adjoint

    nz = nz.clone().requires_grad_(True)
    b = b.clone().requires_grad_(True)
    x = adjoint.solve(ds, nz, b, **kw)
    (c * x).sum().backward()
    return x.detach(), nz.grad.detach(), b.grad.detach()


def _loss(ds, nz, b, c):
    from sdsb200 import adjoint

    return float((c * adjoint.solve(ds, nz, b)).sum())


@pytest.mark.parametrize("structure", ["SPD", "S", "G"])
def test_adjoint_matches_finite_differences(torch_cuda, structure):
    torch = torch_cuda
    A, ds, nz, b, c = _setup(torch, structure)
    x, gA, gb = _grads(torch, ds, nz, b, c)
    assert ds.getparam("npivots") == 0
    scale_a = float(gA.abs().max())
    scale_b = float(gb.abs().max())
    rng = np.random.default_rng(11)
    ks = rng.choice(A.nnz, 40, replace=False)
    for k in ks:
        e = torch.zeros_like(nz)
        e[k] = FD_H
        fd = (_loss(ds, nz + e, b, c) - _loss(ds, nz - e, b, c)) / (2 * FD_H)
        assert abs(fd - float(gA[k])) <= FD_TOL * scale_a, (k, fd, float(gA[k]))
    for i in rng.choice(A.shape[0], 8, replace=False):
        e = torch.zeros_like(b)
        e[i] = FD_H
        fd = (_loss(ds, nz, b + e, c) - _loss(ds, nz, b - e, c)) / (2 * FD_H)
        assert abs(fd - float(gb[i])) <= FD_TOL * scale_b, (i, fd, float(gb[i]))


@pytest.mark.parametrize("structure", ["SPD", "S", "G"])
def test_adjoint_matches_oracle_transposed_solve(torch_cuda, structure):
    torch = torch_cuda
    A, ds, nz, b, c = _setup(torch, structure)
    x, gA, gb = _grads(torch, ds, nz, b, c)
    okw = dict(pivot_threshold=0.1) if structure == "G" else {}
    S, O, info = oracle_for(A, structure, **okw)
    assert info == 0
    cc = c.cpu().numpy()
    bbar = O.solve(cc.reshape(-1, 1), transpose=structure == "G").reshape(-1)
    xs = x.cpu().numpy()
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    cols = A.indices
    if structure == "G":
        ref = -bbar[rows] * xs[cols]
    else:
        keep = cols <= rows                      # view "F": the lower triangle is what the factorization reads
        ref = np.where(keep, -(bbar[rows] * xs[cols] + np.where(rows != cols, bbar[cols] * xs[rows], 0.0)), 0.0)
    scale = max(1.0, np.abs(ref).max())
    assert np.abs(gA.cpu().numpy() - ref).max() <= ORACLE_TOL * scale
    assert np.abs(gb.cpu().numpy() - bbar).max() <= ORACLE_TOL * max(1.0, np.abs(bbar).max())


def test_adjoint_refactorizes_when_the_factor_changed(torch_cuda):
    torch = torch_cuda
    A, ds, nz, b, c = _setup(torch, "G")
    _, gA0, gb0 = _grads(torch, ds, nz, b, c)
    from sdsb200 import adjoint

    nz1 = nz.clone().requires_grad_(True)
    x1 = adjoint.solve(ds, nz1, b)
    adjoint.solve(ds, nz * 1.5, b)               # the plan now holds another factor
    (c * x1).sum().backward()
    assert torch.allclose(nz1.grad, gA0, rtol=0, atol=1e-12 * float(gA0.abs().max()))
    _, gA2, _ = _grads(torch, ds, nz, b, c, refactorize=True)
    assert torch.allclose(gA2, gA0, rtol=0, atol=1e-12 * float(gA0.abs().max()))


def test_adjoint_kkt_200_entries(torch_cuda):
    # the KKT form of the indefinite workload at reduced size: 2x2 pivots through pivot pairs
    from sdsb200.solver import DirectSolver

    torch = torch_cuda
    A = small_kkt(24, 24, 300, seed=11)   # no perturbed pivot (checked below)
    ds = DirectSolver(A, "S")
    ds.execute("analysis")
    rng = np.random.default_rng(13)
    nz = torch.tensor(A.data, dtype=torch.float64, device="cuda")
    b = torch.tensor(rng.uniform(-1, 1, A.shape[0]), dtype=torch.float64, device="cuda")
    c = torch.tensor(rng.standard_normal(A.shape[0]), dtype=torch.float64, device="cuda")
    _, gA, _ = _grads(torch, ds, nz, b, c)
    assert ds.getparam("inertia") == (24 * 24, 300)
    assert ds.getparam("npivots") == 0
    scale = float(gA.abs().max())
    for k in rng.choice(A.nnz, 200, replace=False):
        e = torch.zeros_like(nz)
        e[k] = FD_H
        fd = (_loss(ds, nz + e, b, c) - _loss(ds, nz - e, b, c)) / (2 * FD_H)
        assert abs(fd - float(gA[k])) <= FD_TOL * scale, (k, fd, float(gA[k]))


def test_adjoint_uniform_batch(torch_cuda):
    from sdsb200.solver import DirectSolver

    torch = torch_cuda
    A = M.lap2d_shifted(9, 9, seed=5)
    vals = M.batch_members(A, 3, spread=0.1, seed=5)
    rng = np.random.default_rng(17)
    n = A.shape[0]
    b = torch.tensor(rng.uniform(-1, 1, (3, n)), dtype=torch.float64, device="cuda")
    c = torch.tensor(rng.standard_normal((3, n)), dtype=torch.float64, device="cuda")
    nz = torch.tensor(vals.reshape(-1), dtype=torch.float64, device="cuda")
    ds = DirectSolver((A.indptr, A.indices, vals.reshape(-1), n), "SPD")
    ds.execute("analysis")
    _, gA, gb = _grads(torch, ds, nz, b, c)
    for m in range(3):
        one = DirectSolver(A, "SPD")
        one.execute("analysis")
        _, gA1, gb1 = _grads(torch, one, nz[m * A.nnz:(m + 1) * A.nnz], b[m], c[m])
        assert torch.allclose(gA[m * A.nnz:(m + 1) * A.nnz], gA1, rtol=0, atol=1e-12 * float(gA1.abs().max()))
        assert torch.allclose(gb[m], gb1, rtol=0, atol=1e-12 * float(gb1.abs().max()))

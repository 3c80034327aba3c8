"""Refinement of a given X on the host above the C ABI: plain iterative refinement (the reference's
``refine!``, src/solve/refinement.jl:359-397) for the "solve_refinement" phase, and FGMRES-IR
(``fgmres_refine!``, src/solve/refinement.jl:577-614).

Plain refinement, at most nsteps steps of

    R = B - op(A) X                        sdsb200_residual
    stop if tol > 0 and max_k ||R_k|| / ||B_k|| <= tol
    X += op(A)^{-1} R                      sdsb200_solve without refinement

FGMRES-IR:

On the stacked compact columns (all right-hand sides of all members as one vector of length
n * ncols):

    R0 = B - op(A) X                       sdsb200_residual
    stop if tol > 0 and max_k ||R0_k|| / ||B_k|| <= tol
    D  = FGMRES(op(A), R0; right preconditioner op(A)^{-1} through the factor (sdsb200_solve without
         refinement), at most nsteps iterations, ||R0 - op(A) D|| <= tol min_k ||B_k||)
    X += D

The operator op(A) z is one residual launch with B = 0 (R = -op(A) z, the reference's
RefinementOperator, refinement.jl:428-482) and the preconditioner one solve (FactorPreconditioner,
refinement.jl:484-541). As in the reference, every iteration synchronizes with the host for its
inner products. The Arnoldi basis is orthogonalized by classical Gram-Schmidt applied twice, and
the Hessenberg least-squares problem by Givens rotations.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np


def _max_relative(R, B, n):
    """max over the columns of ||R_k|| / ||B_k|| (||R_k|| where B_k = 0), as the reference's
    _max_relative_residual."""
    import torch

    rn = R.reshape(-1, n).norm(dim=1)
    bn = B.reshape(-1, n).norm(dim=1)
    rel = torch.where(bn > 0, rn / torch.where(bn > 0, bn, torch.ones_like(bn)), rn)
    return float(rel.max()) if rel.numel() else 0.0


def ir_iterate(residual, solve, Xcm, Bcm, n, nsteps, tol, interrupted=None):
    """Plain iterative refinement of Xcm in place (refine!, src/solve/refinement.jl:359-397) with the
    callables residual(X, B) -> B - op(A) X and solve(R) -> op(A)^{-1} R. tol = 0 never stops early.
    interrupted() is polled before every step; when it returns True the refinement stops and
    (steps done, True) is returned, X holding the last completed iterate. Returns (steps, False)
    otherwise."""
    steps = 0
    for _ in range(int(nsteps)):
        if interrupted is not None and interrupted():
            return steps, True
        R = residual(Xcm, Bcm)
        if tol > 0 and _max_relative(R, Bcm, n) <= tol:
            break
        Xcm += solve(R)
        steps += 1
    return steps, False


def _capi_ops(solver, nrhs, solve_mode, nzval):
    """residual(X, B) and solve(R) through the C ABI on the solver's plan and current stream."""
    import torch

    from ._native import numeric_lib
    from .solver import _check

    lib = numeric_lib()
    n = solver.n
    stream = C.c_void_p(torch.cuda.current_stream(solver.device).cuda_stream)
    nz = C.c_void_p((solver.nzval if nzval is None else nzval).data_ptr())
    opts = solver._opts()
    opts.ir_n_steps = 0
    opts.solve_mode = solve_mode
    steps = C.c_int32(0)

    def residual(X, B):
        X = X.contiguous()
        R = torch.empty_like(B)
        _check(lib.sdsb200_residual(solver._plan, C.c_void_p(R.data_ptr()), C.c_void_p(X.data_ptr()), n,
                                    C.c_void_p(B.data_ptr()), n, nrhs, nz, solve_mode, stream), lib)
        return R

    def solve(R):
        out = torch.empty_like(R)
        _check(lib.sdsb200_solve(solver._plan, C.c_void_p(out.data_ptr()), n, C.c_void_p(R.data_ptr()), n, nrhs,
                                 nz, C.byref(opts), C.byref(steps), stream), lib)
        return out

    return residual, solve


def ir_refine(solver, Xcm, Bcm, nrhs, solve_mode, nsteps, tol, nzval=None, interrupted=None):
    """Plain refinement of Xcm (device, column-major per member) in place through the C ABI; returns
    (steps, interrupted) as ir_iterate."""
    residual, solve = _capi_ops(solver, nrhs, solve_mode, nzval)
    return ir_iterate(residual, solve, Xcm, Bcm, solver.n, nsteps, tol, interrupted)


def fgmres_refine(solver, Xcm, Bcm, nrhs, solve_mode, nsteps, tol, nzval=None):
    """Refine Xcm (device, column-major per member: (nbatch, nrhs, n) or (nrhs, n)) in place, for the
    matrix with values ``nzval`` (default: the solver's; with a matching, the matched system's).

    Returns the FGMRES iterations performed."""
    import torch

    from ._native import numeric_lib
    from .solver import _check

    lib = numeric_lib()
    n = solver.n
    if nsteps <= 0 or n == 0:
        return 0
    stream = C.c_void_p(torch.cuda.current_stream(solver.device).cuda_stream)
    vals = solver.nzval if nzval is None else nzval
    nz = C.c_void_p(vals.data_ptr())
    shape = Xcm.shape
    zeros = torch.zeros_like(Bcm)

    def residual(X, B):
        R = torch.empty_like(B)
        _check(lib.sdsb200_residual(solver._plan, C.c_void_p(R.data_ptr()), C.c_void_p(X.data_ptr()), n,
                                    C.c_void_p(B.data_ptr()), n, nrhs, nz, solve_mode, stream), lib)
        return R

    def op(v):          # op(A) v on the stacked vector
        return -residual(v.reshape(shape).contiguous(), zeros).reshape(-1)

    opts = solver._opts()
    opts.ir_n_steps = 0
    opts.solve_mode = solve_mode
    steps = C.c_int32(0)

    def precond(v):     # op(A)^{-1} v through the factor
        src = v.reshape(shape).contiguous()
        out = torch.empty_like(src)
        _check(lib.sdsb200_solve(solver._plan, C.c_void_p(out.data_ptr()), n, C.c_void_p(src.data_ptr()), n, nrhs,
                                 nz, C.byref(opts), C.byref(steps), stream), lib)
        return out.reshape(-1)

    R0 = residual(Xcm, Bcm)
    atol = 0.0
    if tol > 0:
        rn = R0.reshape(-1, n).norm(dim=1)
        bn = Bcm.reshape(-1, n).norm(dim=1)
        rel = torch.where(bn > 0, rn / torch.where(bn > 0, bn, torch.ones_like(bn)), rn)
        if float(rel.max()) <= tol:
            return 0
        atol = tol * float(torch.where(bn > 0, bn, torch.ones_like(bn)).min())
    r0 = R0.reshape(-1)
    beta = float(r0.norm())
    if beta == 0.0:
        return 0
    m = int(nsteps)
    V = [r0 / beta]
    Z = []
    H = np.zeros((m + 1, m))
    cs = np.zeros(m)
    sn = np.zeros(m)
    g = np.zeros(m + 1)
    g[0] = beta
    iters = 0
    for j in range(m):
        z = precond(V[j])
        Z.append(z)
        w = op(z)
        Vm = torch.stack(V)
        h = Vm @ w                       # classical Gram-Schmidt, twice
        w = w - Vm.t() @ h
        h2 = Vm @ w
        w = w - Vm.t() @ h2
        hcol = (h + h2).cpu().numpy()
        hn = float(w.norm())
        H[: j + 1, j] = hcol
        H[j + 1, j] = hn
        for i in range(j):               # previous rotations
            a, b = H[i, j], H[i + 1, j]
            H[i, j], H[i + 1, j] = cs[i] * a + sn[i] * b, -sn[i] * a + cs[i] * b
        a, b = H[j, j], H[j + 1, j]
        rho = math.hypot(a, b)
        cs[j], sn[j] = (1.0, 0.0) if rho == 0.0 else (a / rho, b / rho)
        H[j, j], H[j + 1, j] = rho, 0.0
        g[j + 1] = -sn[j] * g[j]
        g[j] = cs[j] * g[j]
        iters = j + 1
        if abs(g[j + 1]) <= atol or hn == 0.0:
            break
        V.append(w / hn)
    k = iters
    y = np.zeros(k)
    for i in range(k - 1, -1, -1):       # back substitution with the rotated Hessenberg matrix
        s = g[i] - H[i, i + 1:k] @ y[i + 1:k]
        y[i] = s / H[i, i] if H[i, i] != 0 else 0.0
    D = torch.zeros_like(r0)
    for i in range(k):
        D += float(y[i]) * Z[i]
    Xcm += D.reshape(shape)
    return iters

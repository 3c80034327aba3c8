"""Differentiation of the solve: x = A^{-1} b with respect to the values of A and to b.

The reference has no automatic differentiation. This module is the differentiation rule a
ChainRulesCore ``rrule`` for ``solve`` would hold, written as a ``torch.autograd.Function``:

* forward: factor A (the solver's plan keeps the factor on the device) and solve;
* backward, for x_bar = dLoss/dx:
  b_bar = A^{-T} x_bar, one solve with the device-resident factor: ``solve_mode = 1`` for "G"
  (U^T then L^T sweeps); A^T = A for "S" and "SPD";
  A_bar = -b_bar x^T sampled on the CSR pattern (``sdsb200_sampled_outer``), over the entries the
  factorization reads. For "S"/"SPD" a kept off-diagonal entry stands for a_ij and a_ji, so it
  collects both terms.

If the solver was refactored with other values between the forward and the backward, or
``refactorize=True`` was given, the backward refactors with the saved values first. A caller whose
batch of factors does not fit in device memory can then drop them after the forward: the backward
pays for one more factorization instead of keeping every factor resident.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from ._native import numeric_lib
from .solver import DirectSolver, FactorizationError, InvalidValueError


def _torch():
    import torch

    return torch


def _device_pattern(solver: DirectSolver):
    """The solver's CSR pattern as device int64 arrays (cached on the solver)."""
    torch = _torch()
    pat = getattr(solver, "_adj_pattern", None)
    if pat is None:
        pat = (torch.from_numpy(solver.rowptr).to(solver.device), torch.from_numpy(solver.colval).to(solver.device))
        solver._adj_pattern = pat
    return pat


def sampled_outer(solver: DirectSolver, U, V, alpha=-1.0):
    """alpha * (U V^T) sampled on the pattern of ``solver`` (symmetrised for "S"/"SPD" as documented).

    ``U`` and ``V`` are device tensors of shape (n,), (n, k), (nbatch, n) or (nbatch, n, k), matching
    the solver's batch. Returns a float64 tensor with one value per stored entry (nnz * nbatch).
    """
    torch = _torch()
    lib = numeric_lib()
    n, nb = solver.n, solver.nbatch
    rowptr, colval = _device_pattern(solver)

    def colmajor(T):
        T = T.to(solver.device, torch.float64)
        if nb == 1:
            T = T.reshape(n, -1)
            return T.t().contiguous(), T.shape[1]
        T = T.reshape(nb, n, -1)
        return T.transpose(1, 2).contiguous(), T.shape[2]

    Uc, k1 = colmajor(U)
    Vc, k2 = colmajor(V)
    if k1 != k2:
        raise InvalidValueError("U and V need the same number of columns")
    out = torch.empty(solver.nnz * nb, dtype=torch.float64, device=solver.device)
    stream = torch.cuda.current_stream(solver.device).cuda_stream
    rc = lib.sdsb200_sampled_outer(n, solver.nnz, C.c_void_p(rowptr.data_ptr()), C.c_void_p(colval.data_ptr()), 8,
                                   solver.index_base, capi.STRUCTURE[solver.structure], ord(solver.view),
                                   C.c_void_p(Uc.data_ptr()), n, C.c_void_p(Vc.data_ptr()), n, k1, nb, float(alpha),
                                   C.c_void_p(out.data_ptr()), C.c_void_p(stream))
    if rc != 0:
        raise InvalidValueError(lib.sdsb200_last_error().decode())
    return out


def _factor(solver, nzval):
    solver.update(nzval)
    if solver._stage < 1:
        solver.execute("analysis")
    info = solver.execute("factorization")
    if np.any(np.asarray(info) != 0):
        raise FactorizationError(f"factorization failed (info = {info})")
    solver._adj_token = object()          # identifies the values the plan's factor belongs to
    return solver._adj_token


def _transposed_solve(solver, xbar):
    mode = solver.params["solve_mode"]
    solver.setparam("solve_mode", 1 if solver.structure == "G" else 0)
    try:
        return solver.execute("solve", None, xbar)
    finally:
        solver.setparam("solve_mode", mode)


class _Solve:
    """Holder of the autograd Function (built lazily so that importing this module needs no torch)."""

    fn = None

    @classmethod
    def get(cls):
        if cls.fn is not None:
            return cls.fn
        torch = _torch()

        class SolveFn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, nzval, b, solver, refactorize):
                nz = nzval.detach().to(solver.device, torch.float64).reshape(-1).contiguous()
                token = _factor(solver, nz)
                x = solver.execute("solve", None, b.detach())
                ctx.solver, ctx.token, ctx.refactorize = solver, token, bool(refactorize)
                ctx.b_shape, ctx.b_dtype = b.shape, b.dtype
                ctx.save_for_backward(nz, x)
                return x

            @staticmethod
            def backward(ctx, xbar):
                solver = ctx.solver
                nz, x = ctx.saved_tensors
                if ctx.refactorize or getattr(solver, "_adj_token", None) is not ctx.token:
                    ctx.token = _factor(solver, nz)
                bbar = _transposed_solve(solver, xbar.detach().contiguous())
                abar = sampled_outer(solver, bbar, x, alpha=-1.0)
                return abar, bbar.reshape(ctx.b_shape).to(ctx.b_dtype), None, None

        cls.fn = SolveFn
        return SolveFn


def solve(solver: DirectSolver, nzval, b, refactorize: bool = False):
    """x = A(nzval)^{-1} b, differentiable in ``nzval`` (one value per stored entry of the solver's
    pattern, times nbatch) and in ``b``. ``solver`` is a DirectSolver on that pattern; it is analysed
    on first use and factored with ``nzval`` in the forward. With ``matching_alg`` the solves run on the
    matched system and map back (the matching is the analysis'), so x, b-bar and A-bar are those of A."""
    return _Solve.get().apply(nzval, b, solver, refactorize)

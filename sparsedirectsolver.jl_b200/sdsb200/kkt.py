"""KKTSolver: the front end for the linear systems of an interior-point method (src/kkt.jl:1-396).

One real symmetric matrix with a fixed pattern, factorized again with new values at every iteration,
one right-hand side at a time, the inertia read after each factorization. It sets the parameters of
the chosen factorization on a :class:`DirectSolver` and drives its phases.

The reference picks between its fused pipeline (src/fused.jl) and the stock one. Only the stock
pipeline is built here, so ``fused=True`` raises :class:`NotSupportedError` and
:meth:`KKTSolver.pipeline` is always ``"stock"``.
"""
from __future__ import annotations

import numpy as np

from .solver import DirectSolver, FactorizationError, InvalidValueError, NotSupportedError

FACTORIZATIONS = ("cholesky", "ldl")
PIVOTINGS = ("none", "diagonal", "bk")
MATCHINGS = ("none", "default", "algo1", "algo2", "algo3", "algo4", "algo5", "algo6")


def _check_options(factorization, pivoting, matching, fused, pivot_threshold, pivot_sign):
    """The constructor's option checks (`_kkt_solver`, src/kkt.jl:162-183), in the reference's order."""
    if factorization not in FACTORIZATIONS:
        raise InvalidValueError(f"factorization must be 'cholesky' or 'ldl', got {factorization!r}")
    if pivoting not in PIVOTINGS:
        raise InvalidValueError(f"pivoting must be 'none', 'diagonal' or 'bk', got {pivoting!r}")
    ldl = factorization == "ldl"
    if pivoting != "none" and not ldl:
        raise InvalidValueError(f"pivoting = {pivoting!r} needs factorization = 'ldl'")
    if pivoting == "bk" and fused is True:
        raise InvalidValueError("fused = True needs pivoting = 'none' or 'diagonal' (the fused pipeline has no "
                                "Bunch-Kaufman pivoting)")
    if pivoting not in ("diagonal", "bk") and pivot_threshold is not None:
        raise InvalidValueError("pivot_threshold needs pivoting = 'diagonal' or 'bk'")
    if not ldl and pivot_sign is not None:
        raise InvalidValueError("pivot_sign needs factorization = 'ldl'")
    if matching not in MATCHINGS:
        raise InvalidValueError(f"unknown matching {matching!r}")
    matched = matching not in ("none", "default")
    if matched and not ldl:
        raise InvalidValueError(f"matching = {matching!r} needs factorization = 'ldl'")
    if fused is True:
        raise NotSupportedError("KKTSolver: the fused pipeline is not built; use fused = None or False")
    return ldl, matched


class KKTSolver:
    """``KKTSolver(A, view='L'; ...)`` (src/kkt.jl:9-160).

    ``A`` is a scipy CSR matrix or ``(rowptr, colval, nzval, n)``, ``view`` the stored triangle.
    A CUDA float64 tensor ``nzval`` is aliased: write new values into it and call :meth:`factorize`.
    Other arrays are copied; pass new values to :meth:`factorize`.

    Keywords as in the reference: ``factorization`` ("cholesky" -> "SPD", "ldl" -> "S"), ``pivoting``
    ("none": static pivoting in the analysis' order, pivot_type 'N'; "diagonal": 1x1 diagonal pivoting,
    'D'; "bk": Bunch-Kaufman), ``matching`` ("none"/"default" off, "algo1"-"algo6"), ``fused``,
    ``pivot_threshold``, ``pivot_epsilon``, ``pivot_sign``, ``ir_n_steps``, ``reordering`` ("algo4":
    nested dissection), ``user_perm``, ``tuning`` and ``deferred_analysis``.
    """

    def __init__(self, A, view="L", *, factorization="cholesky", pivoting="none", matching="none", fused=None,
                 pivot_threshold=None, pivot_epsilon=None, pivot_sign=None, ir_n_steps=None, reordering="algo4",
                 user_perm=None, tuning=None, deferred_analysis=False, device="cuda"):
        ldl, matched = _check_options(factorization, pivoting, matching, fused, pivot_threshold, pivot_sign)
        inner = DirectSolver(A, "S" if ldl else "SPD", view=view, device=device)
        if inner.nbatch != 1:
            raise NotSupportedError(f"KKTSolver: a uniform batch ({inner.nbatch} members) is not supported; "
                                    "use DirectSolver")
        if matched:
            inner.setparam("matching_alg", matching)
        if pivoting == "bk":
            if pivot_threshold is not None:
                inner.setparam("pivot_threshold", pivot_threshold)
        elif ldl:
            inner.setparam("pivot_type", "D" if pivoting == "diagonal" else "N")
            # 1x1 pivots consume no 2x2 pair; the pairs of a job-5 matching would shape the ordering
            if not (matched and matching in ("algo5", "algo6")):
                inner.setparam("pivot_pairs", "none")
            if pivoting == "diagonal" and pivot_threshold is not None:
                inner.setparam("pivot_threshold", pivot_threshold)
        if ldl and pivot_sign is not None:
            inner.setparam("pivot_sign", np.asarray(pivot_sign, dtype=np.int8))
        if pivot_epsilon is not None:
            inner.setparam("pivot_epsilon", pivot_epsilon)
        if ir_n_steps is not None:
            inner.setparam("ir_n_steps", int(ir_n_steps))
        if tuning is not None:
            inner.setparam("tuning", int(tuning))
        if user_perm is not None:
            inner.setparam("user_perm", user_perm)
        else:
            inner.setparam("reordering_alg", reordering)
        self.inner = inner
        self.factorization = factorization
        self.pivoting = pivoting
        self.info = 0
        self.factorized = False
        if not deferred_analysis:
            self._first_factorization()

    # the analysis and the first factorization, on the values the matrix holds now
    def _first_factorization(self):
        self.inner.execute("analysis")
        self.info = int(self.inner.execute("factorization"))
        self.factorized = True
        return self

    def _check_factorized(self, what):
        if not self.factorized:
            raise FactorizationError(f"KKTSolver: {what} needs a factorization; with deferred_analysis = True "
                                     "call factorize() first")

    @property
    def n(self):
        return self.inner.n

    def pipeline(self):
        """``pipeline(K)``: always ``"stock"`` here (the fused pipeline is not built)."""
        return "stock"

    def factorize(self, nzval=None):
        """``factorize!(K)``: factorize the current values (``nzval``, when given, replaces them). The first
        call after ``deferred_analysis = True`` runs the analysis first. A failed factorization does not
        raise: ``getparam("info")`` is then nonzero."""
        if nzval is not None:
            self.inner.update(nzval)
        if not self.factorized:
            return self._first_factorization()
        self.info = int(self.inner.execute("refactorization"))
        return self

    def analyze(self, nzval=None):
        """``analyze!(K)``: redo the analysis (ordering, matching, pairs) on the current values and factorize."""
        if nzval is not None:
            self.inner.update(nzval)
        self.factorized = False
        self.info = 0
        return self._first_factorization()

    def solve(self, x, b=None):
        """``solve!(K, x, b)``, or ``solve!(K, xb)`` with ``b`` omitted (``x`` holds b on entry)."""
        self._check_factorized("solve")
        rhs = x if b is None else b
        out = self.inner.execute("solve", None, rhs)
        try:
            import torch

            if isinstance(x, torch.Tensor):
                x.copy_(out.reshape(x.shape))
                torch.cuda.current_stream(self.inner.device).synchronize()
                return x
        except ImportError:
            pass
        np.copyto(x, out.cpu().numpy().reshape(np.shape(x)))
        return x

    def inertia(self):
        """``inertia(K)`` -> (npos, nzero, nneg) of the matrix factorized last (src/kkt.jl:378-392)."""
        self._check_factorized("inertia")
        npos, nneg = self.inner.getparam("inertia")
        return (int(npos), self.n - int(npos) - int(nneg), int(nneg))

    def getparam(self, name):
        """Forwarded to the inner solver; ``"info"`` is the last factorization's."""
        return self.info if name == "info" else self.inner.getparam(name)

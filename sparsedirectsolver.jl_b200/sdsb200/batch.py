"""Uneven batches: many independent systems of different sizes and patterns as one plan.

The reference batches only systems that share one pattern (``ubatch_size``). Here a batch of
unrelated systems is merged into one block-diagonal matrix. Its elimination tree is a forest with
one tree per system, so:
* the analysis orders and amalgamates every system independently;
* each level-batched factorization launch covers the fronts of that height in every system;
* the whole solve is one cooperative persistent launch, and factorization and solve are replayed
  from captured CUDA graphs.

Each system keeps its own backward error, computed here per block.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .solver import DirectSolver, InvalidValueError


class UnevenBatch:
    """``UnevenBatch(systems, structure, **params)``: a list of square scipy sparse matrices."""

    def __init__(self, systems, structure="SPD", device="cuda:0", **params):
        if not systems:
            raise InvalidValueError("an uneven batch needs at least one system")
        mats = []
        for A in systems:
            A = sp.csr_matrix(A)
            if A.shape[0] != A.shape[1]:
                raise InvalidValueError(f"every system must be square, got {A.shape}")
            mats.append(A)
        self.systems = mats
        self.sizes = np.array([A.shape[0] for A in mats], dtype=np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)])
        A = sp.block_diag(mats, format="csr")
        A.sort_indices()
        self.A = A
        self.solver = DirectSolver(A, structure, device=device, **params)

    @property
    def count(self):
        return len(self.systems)

    def execute(self, phase, X=None, B=None):
        """The DirectSolver phases on the whole batch; B and the result are stacked (sum of n, ...)."""
        return self.solver.execute(phase, X, B)

    def stack(self, vectors):
        """One stacked right-hand side from per-system vectors."""
        return np.concatenate([np.asarray(v, dtype=np.float64).reshape(-1) for v in vectors])

    def split(self, x):
        """Per-system views of a stacked solution."""
        return [x[self.offsets[i]:self.offsets[i + 1]] for i in range(self.count)]

    def backward_errors(self, x, b):
        """Scaled backward error of every system: ||b_i - A_i x_i||_inf / (||A_i||_inf ||x_i||_inf + ||b_i||_inf)."""
        x = np.asarray(x, dtype=np.float64).reshape(-1)
        b = np.asarray(b, dtype=np.float64).reshape(-1)
        r = np.abs(b - self.A @ x)
        rowsum = np.asarray(abs(self.A).sum(axis=1)).reshape(-1)
        starts = self.offsets[:-1]
        rmax = np.maximum.reduceat(r, starts)
        anorm = np.maximum.reduceat(rowsum, starts)
        xmax = np.maximum.reduceat(np.abs(x), starts)
        bmax = np.maximum.reduceat(np.abs(b), starts)
        den = anorm * xmax + bmax
        return np.where(den > 0, rmax / np.where(den > 0, den, 1.0), rmax)

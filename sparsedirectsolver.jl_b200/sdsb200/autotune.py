"""Autotuner of the plan's front tile shapes (``tuning``): no counterpart in the reference.

Two shapes decide how the fronts of a plan map onto the kernels:
* ``fsmall``: the largest front order factored in shared memory by the small-front kernel. Larger
  fronts take the column-owner assembly, diagonal-block and DMMA GEMM path.
* ``wide``: the tallest front (of at most 32 columns) that the dataflow solve gives to one warp;
  taller or wider fronts go to tile tasks spread over the grid.
* ``chains``: 0 solves those tiled fronts through inverse panels [L11^-1; L21 L11^-1], built after the
  factorization (one matrix-vector product per front and sweep); 1 through chains of 64-column
  blocks (no extra factorization work, one dependency link per block).
* ``streams`` (not searched, default 4): independent subtrees of a Cholesky front tree factored on
  separate streams.
* ``subtree``: fused subtrees of shared-memory fronts, one CTA each (4: up to 16 fronts per
  subtree), or none (0: one launch per level and size class).

The autotuner times factorization + solve for each candidate on the solver's own matrix and
right-hand side (CUDA events, after a warm-up), keeps the fastest, and leaves the solver planned
and factored with it. Results are cached in-process per (n, nnz, structure, precision, nbatch).
"""
from __future__ import annotations

from .capi import tuning as make_tuning

CANDIDATES = tuple((fs, wd, ch, 0, 0, sub) for fs in (0, 128, 96) for wd in (0, 64) for ch in (0, 1)
                   for sub in (0, 4))

_cache: dict = {}


def _key(solver):
    return (solver.n, solver.nnz, solver.structure, solver.params["factor_precision"], solver.nbatch)


def autotune(solver, B, candidates=CANDIDATES, reps=3, use_cache=True):
    """Pick the tuning with the smallest factorization + solve time. Returns {tuning: ms}."""
    import torch

    if solver.symbolic is None:
        solver.execute("analysis")
    key = _key(solver)
    if use_cache and key in _cache:
        best, times = _cache[key]
        solver.setparam("tuning", best)
        solver.replan()
        solver.execute("factorization")
        return dict(times)
    times = {}
    for cand in candidates:
        t = make_tuning(*cand)
        solver.setparam("tuning", t)
        try:
            solver.replan()
        except Exception:            # a shape the plan rejects (for example an FP64 class of 224)
            continue
        solver.execute("factorization")
        solver.execute("solve", None, B)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            solver.execute("factorization")
            solver.execute("solve", None, B)
        e1.record()
        torch.cuda.synchronize()
        times[t] = e0.elapsed_time(e1) / reps
    best = min(times, key=times.get)
    _cache[key] = (best, dict(times))
    solver.setparam("tuning", best)
    solver.replan()
    solver.execute("factorization")
    return times


def describe(t):
    return {"fsmall": int(t) & 0x1FF, "wide": (int(t) >> 9) & 0x7FF, "chains": (int(t) >> 20) & 1,
            "streams": (int(t) >> 21) & 15, "steps": (int(t) >> 25) & 1, "subtree": (int(t) >> 26) & 15}


__all__ = ["autotune", "describe", "CANDIDATES"]

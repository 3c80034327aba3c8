"""sdsb200: a B200-native numeric phase (factorization, refactorization, solve)
for SparseDirectSolver.jl's DirectSolver / execute! phase API."""
from .analysis import Symbolic, analyze, analyze_csr  # noqa: F401

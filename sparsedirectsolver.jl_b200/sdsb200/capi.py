"""ctypes declarations of libsdsb200.so (include/sdsb200.h)."""
from __future__ import annotations

import ctypes as C

OK = 0
INVALID_VALUE = 1
NOT_SUPPORTED = 2
PHASE_ORDER = 3
INTERRUPTED = 4
CUDA_ERROR = 5
ALLOC_FAILED = 6
TIMEOUT = 7

STRUCTURE = {"G": 0, "S": 1, "SPD": 3}
PRECISION = {"fp64": 0, "fp32": 1}
PIVOT_TYPE = {"A": 0, "N": 1, "C": 2, "R": 3, "D": 4, "L": 5, "B": 6}

EXPORTS = ("sdsb200_default_opts", "sdsb200_plan_create", "sdsb200_plan_destroy", "sdsb200_factor", "sdsb200_solve",
           "sdsb200_get_stats", "sdsb200_get_pivots", "sdsb200_get_factor", "sdsb200_set_members",
           "sdsb200_set_interrupt", "sdsb200_set_graphs", "sdsb200_set_persistent", "sdsb200_set_profiling", "sdsb200_get_trace", "sdsb200_plan_stat", "sdsb200_last_error",
           "sdsb200_solve_noalloc", "sdsb200_sampled_outer", "sdsb200_residual", "sdsb200_solve_phase",
           "sdsb200_schur_matrix")

# solve sub-phases of sdsb200_solve_phase
PHASE = {"fwd_perm": 1, "fwd": 2, "diag": 3, "bwd": 4, "bwd_perm": 5, "load": 6, "store": 7}


class Symbolic(C.Structure):
    _fields_ = [("n", C.c_int64), ("nnz", C.c_int64), ("ns", C.c_int64), ("index_width", C.c_int32),
                ("structure", C.c_int32)] + [
        (nm, C.c_void_p) for nm in ("perm", "super_ptr", "snparent", "rowptr", "rowval", "front_ptr", "child_ptr",
                                    "child_list", "relind_ptr", "relind", "amap", "amap_ptr", "amap_src",
                                    "full_rowptr", "full_colval", "full_srcptr", "full_src")] + [
        ("full_nnz", C.c_int64), ("full_nsrc", C.c_int64), ("schur", C.c_int64)]


class PlanOptions(C.Structure):
    _fields_ = [("nbatch", C.c_int32), ("precision", C.c_int32), ("max_nrhs", C.c_int32), ("tuning", C.c_int32)]


def tuning(fsmall=0, wide=0, chains=0, streams=0, steps=0, subtree=0):
    """SDSB200_TUNING_STREAMS(fsmall, wide, chains, streams) | SDSB200_TUNING_SUBTREE(subtree) (|
    SDSB200_TUNING_STEPS with steps = 1): the plan's front shapes (0 = defaults); chains = 1 solves the
    tiled fronts by 64-column block chains instead of inverse panels; streams = the factorization streams
    of a single-system Cholesky plan (0 = 4, 1 = level by level); steps = 1 runs its large fronts' steps
    as one dataflow launch per batch instead of one launch per step and kernel; subtree = the fused
    subtrees (1..14: at most 2**subtree fronts each; 0, the default, and 15: none)."""
    return (int(fsmall) | (int(wide) << 9) | (int(chains) << 20) | (int(streams) << 21) | (int(steps) << 25)
            | (int(subtree) << 26))


class Opts(C.Structure):
    _fields_ = [("pivot_type", C.c_int32), ("pivot_epsilon_alg", C.c_int32), ("pivot_threshold", C.c_double),
                ("pivot_epsilon", C.c_double), ("ir_n_steps", C.c_int32), ("ir_mode", C.c_int32),
                ("ir_tol", C.c_double), ("solve_mode", C.c_int32), ("deterministic_mode", C.c_int32)]


def bind(lib):
    P = C.c_void_p
    sig = {
        "sdsb200_default_opts": (None, [C.POINTER(Opts)]),
        "sdsb200_plan_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(Symbolic), C.POINTER(PlanOptions), P]),
        "sdsb200_plan_destroy": (C.c_int, [P]),
        "sdsb200_factor": (C.c_int, [P, P, P, C.POINTER(Opts), P, P]),
        "sdsb200_solve": (C.c_int, [P, P, C.c_int64, P, C.c_int64, C.c_int32, P, C.POINTER(Opts), P, P]),
        "sdsb200_get_stats": (C.c_int, [P, C.c_int32, P, P]),
        "sdsb200_get_pivots": (C.c_int, [P, C.c_int32, P, P, P]),
        "sdsb200_get_factor": (C.c_int, [P, C.c_int32, P, P]),
        "sdsb200_set_members": (C.c_int, [P, P, C.c_int32]),
        "sdsb200_set_interrupt": (C.c_int, [P, P]),
        "sdsb200_set_profiling": (C.c_int, [P, C.c_int32]),
        "sdsb200_set_graphs": (C.c_int, [P, C.c_int32]),
        "sdsb200_set_persistent": (C.c_int, [P, C.c_int32]),
        "sdsb200_plan_stat": (C.c_double, [P, C.c_char_p]),
        "sdsb200_get_trace": (C.c_int64, [P, P, C.c_int64]),
        "sdsb200_last_error": (C.c_char_p, []),
        "sdsb200_solve_noalloc": (C.c_int, [P, P, C.c_int64, P, C.c_int64, C.c_int32, C.c_int32, P, P]),
        "sdsb200_residual": (C.c_int, [P, P, P, C.c_int64, P, C.c_int64, C.c_int32, P, C.c_int32, P]),
        "sdsb200_solve_phase": (C.c_int, [P, C.c_int32, P, C.c_int64, P, C.c_int64, C.c_int32, C.POINTER(Opts), P]),
        "sdsb200_schur_matrix": (C.c_int, [P, C.c_int32, P, C.c_int64, C.c_int32, P]),
        "sdsb200_sampled_outer": (C.c_int, [C.c_int64, C.c_int64, P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                            P, C.c_int64, P, C.c_int64, C.c_int32, C.c_int32, C.c_double, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib

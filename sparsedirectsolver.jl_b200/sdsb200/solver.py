"""DirectSolver: the reference's handle API over the B200 numeric phase.

Mirrors SparseDirectSolver.jl's ``DirectSolver`` / ``execute!`` / ``setparam!``
/ ``getparam`` (src/solver.jl:187-259, 444-460, 1013-1194): the same phase
strings ("analysis", "factorization", "refactorization", "solve",
"solve_refinement"), structures ("SPD", "S", "G"), parameter names and
error classes (src/errors.jl). Analysis runs on the host
(libsdsb200_analysis.so); factorization and solve run on the GPU through the C
ABI of libsdsb200.so, with torch used only to hold device memory. There is no
CPU fallback: without the CUDA library or a device every phase raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from ._native import numeric_lib
from .analysis import analyze, compute_matching, matching_pairs


class SparseDirectSolverError(Exception):
    pass


class InvalidValueError(SparseDirectSolverError):
    pass


class NotSupportedError(SparseDirectSolverError):
    pass


class FactorizationError(SparseDirectSolverError):
    pass


class InterruptedError_(SparseDirectSolverError):
    pass


_ERRORS = {capi.INVALID_VALUE: InvalidValueError, capi.NOT_SUPPORTED: NotSupportedError,
           capi.PHASE_ORDER: FactorizationError, capi.INTERRUPTED: InterruptedError_}

_DEFAULTS = {
    "reordering_alg": "default", "factorization_alg": "default", "solve_alg": "default", "matching_alg": "default",
    "solve_mode": 0, "ir_n_steps": 0, "ir_tol": 0.0, "pivot_type": "A", "pivot_threshold": 0.01,
    "pivot_epsilon": None, "pivot_epsilon_alg": "default", "deterministic_mode": 0, "ubatch_size": 0,
    "ubatch_index": -1, "use_superpanels": 1, "ir_mode": "plain", "factor_precision": None,
    "amalgamation": (32, 0.25, 8), "pivot_pairs": "default", "pivot_pair_tolerance": 1e-6, "user_perm": None,
    "pivot_sign": None, "user_host_interrupt": None, "max_nrhs": 8, "tuning": 0,
    "schur_mode": 0, "user_schur_indices": None, "ubatch_mask": None,
}


def _check(rc, lib):
    if rc != capi.OK:
        msg = lib.sdsb200_last_error().decode()
        raise _ERRORS.get(rc, RuntimeError)(msg)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def memory_slots(structure, n, ns, nbatch, elsize, factor_len, cb_len, device_bytes, host_bytes, extra_device=0):
    """``getparam("memory_estimates")`` (memory_estimates, src/symbolic/maps.jl:307-356): 16 byte counts in
    cuDSS's slot layout, from a plan that allocates every buffer when it is built:
      1 permanent device memory (every buffer but the update stack; plus ``extra_device``, the matching's
        buffers), 2 peak device memory (slot 1 + the update stack), 3 and 4 host memory (the Symbolic
        maps), 5 = slot 2, 6 = 0 (no hybrid memory mode);
      7 factor panels (L and U^T for "G"), 8 D (2n doubles), 9 the update stack (the contribution-block
        arena), 11 per-front statistics, status, pivot order, kinds and sign requests, 10 the rest of the
        plan's buffers (device maps, launch lists, solve and refinement workspaces);
      12-16 = 0."""
    nb = int(nbatch)
    est = [0] * 16
    est[6] = (2 if structure == "G" else 1) * int(factor_len) * int(elsize) * nb
    est[7] = 2 * int(n) * 8 * nb
    est[8] = int(cb_len) * int(elsize) * nb
    est[10] = (6 * int(ns) * 8 + int(ns) * 4 + 6 * 8 + 8 + int(n) * 4 + int(n)) * nb + int(n) + 8
    est[9] = max(int(device_bytes) - est[6] - est[7] - est[8] - est[10], 0)
    est[1] = int(device_bytes) + int(extra_device)
    est[0] = est[1] - est[8]
    est[2] = est[3] = int(host_bytes)
    est[4] = est[1]
    return est


def active_members(nb, index, mask):
    """The members (0-based) the next numeric or solve phase processes (active_members,
    src/numeric/batch.jl:115-129): ``ubatch_index`` (-1 = all) and the 0/1 flags of ``ubatch_mask``
    (None = all) together."""
    if not (index == -1 or 0 <= index < nb):
        raise InvalidValueError(f"ubatch_index = {index} is outside the batch (0:{nb - 1}, or -1 for all members)")
    if mask is not None and len(mask) != nb:
        raise InvalidValueError(f"ubatch_mask has {len(mask)} entries, the batch has {nb} members")
    return [k for k in range(nb) if (index == -1 or k == index) and (mask is None or mask[k] != 0)]


class DirectSolver:
    """``DirectSolver(A, structure, view)`` for a square CSR matrix.

    ``A`` is a scipy CSR matrix (0-based) or a tuple ``(rowptr, colval, nzval, n)``
    with ``index_base`` 0 or 1. ``nzval`` may hold ``nnz * nbatch`` values
    (a uniform batch, member-major), as a numpy array or a CUDA torch tensor.
    """

    def __init__(self, A, structure="SPD", view="F", index_base=0, device="cuda:0", **params):
        import torch  # device memory only

        self._torch = torch
        if structure not in ("SPD", "S", "G"):
            raise InvalidValueError(f'structure must be "G", "S" or "SPD", got {structure!r}')
        if view not in ("L", "U", "F"):
            raise InvalidValueError(f"view must be 'L', 'U' or 'F', got {view!r}")
        if isinstance(A, tuple):
            rowptr, colval, nzval, n = A
        else:
            A = A.tocsr()
            if A.shape[0] != A.shape[1]:
                raise InvalidValueError(f"the matrix must be square, got {A.shape}")
            rowptr, colval, nzval, n = A.indptr, A.indices, A.data, A.shape[0]
            index_base = 0
        self.n = int(n)
        self.rowptr = np.asarray(rowptr, dtype=np.int64)
        self.colval = np.asarray(colval, dtype=np.int64)
        self.nnz = int(self.colval.size)
        self.structure = structure
        self.view = view
        self.index_base = int(index_base)
        self.device = torch.device(device)
        self.params = dict(_DEFAULTS)
        for k, v in params.items():
            self.setparam(k, v)
        self._set_values(nzval)
        self.symbolic = None
        self._plan = None
        self._stage = 0           # 0 created, 1 analyzed, 2 factorized
        self._info = np.zeros(self.nbatch, dtype=np.int64)
        self._ir_steps = -1
        self._keep = []
        self._matching = None     # host Matching of matching_alg (None: no matching)
        self._mdev = None         # its device tensors: entry weights, row / column scalings, permutation

    # -- values ------------------------------------------------------------------------------------------------
    def _set_values(self, nzval):
        torch = self._torch
        if isinstance(nzval, torch.Tensor):
            t = nzval.to(self.device, torch.float64).reshape(-1).contiguous()
        else:
            t = torch.from_numpy(np.ascontiguousarray(nzval, dtype=np.float64).reshape(-1)).to(self.device)
        if self.nnz == 0 or t.numel() % self.nnz != 0:
            if not (self.nnz == 0 and t.numel() == 0):
                raise InvalidValueError(f"nzval has {t.numel()} entries, not a multiple of nnz = {self.nnz}")
        self.nbatch = max(1, t.numel() // max(self.nnz, 1))
        self.nzval = t

    def update(self, nzval):
        """``update!``: new values with the same pattern (src/solver.jl:309-330)."""
        old = self.nbatch
        self._set_values(nzval)
        if self._plan is not None and self.nbatch != old:
            raise InvalidValueError("the number of batch members changed; run the analysis again")

    # -- parameters -------------------------------------------------------------------------------------------
    def setparam(self, name, value):
        if name == "schur_matrix":
            return self._set_schur_dest(value)
        if name not in _DEFAULTS:
            raise InvalidValueError(f"unknown parameter {name!r}")
        if name == "pivot_type" and value not in capi.PIVOT_TYPE:
            raise InvalidValueError(f"pivot_type must be one of {sorted(capi.PIVOT_TYPE)}")
        if name == "pivot_type" and value in ("C", "R"):
            raise NotSupportedError("global pivoting ('C', 'R') is not supported")
        if name == "pivot_threshold" and not (np.isfinite(value) and value >= 0):
            raise InvalidValueError("pivot_threshold must be finite and nonnegative")
        if name == "ir_n_steps" and int(value) < 0:
            raise InvalidValueError("ir_n_steps must be nonnegative")
        if name == "solve_mode" and int(value) not in (0, 1, 2):
            raise InvalidValueError("solve_mode must be 0, 1 or 2")
        if name == "ir_mode" and value not in ("plain", "ir", "fgmres"):
            raise InvalidValueError(f"ir_mode must be \"ir\" or \"fgmres\", got {value!r}")
        if name == "factor_precision" and value not in (None, "fp64", "fp32", "float64", "float32"):
            raise InvalidValueError("factor_precision must be fp64 or fp32")
        if name == "pivot_sign" and value is not None:
            value = np.asarray(value, dtype=np.int8)
            if value.size != self.n if hasattr(self, "n") else False:
                raise InvalidValueError(f"pivot_sign has {value.size} entries, the matrix has {self.n} rows")
        if name == "schur_mode" and int(value) not in (0, 1):
            raise InvalidValueError("schur_mode must be 0 or 1")
        if name == "user_schur_indices" and value is not None:
            value = np.asarray(value).reshape(-1)
            if hasattr(self, "n") and value.size != self.n:
                raise InvalidValueError(f"user_schur_indices has {value.size} entries, the matrix has {self.n} rows")
            if not np.all((value == 0) | (value == 1)):
                raise InvalidValueError("user_schur_indices must hold flags 0 or 1")
        if name == "ubatch_mask" and value is not None:
            value = np.asarray(value).reshape(-1)
            if not np.all((value == 0) | (value == 1)):
                raise InvalidValueError("ubatch_mask must hold flags 0 or 1")
        if name in ("ubatch_index", "ubatch_mask"):
            # checked against the batch by the next factorization or solve, as the reference's _set_members!
            self.params[name] = int(value) if name == "ubatch_index" else value
            self._members_dirty = True
            return
        self.params[name] = value

    def replan(self):
        """Build the device plan again from the current analysis (after a change of a plan-level
        parameter: ``tuning``, ``max_nrhs``, ``factor_precision``). The factorization must be rerun."""
        if self._stage < 1:
            raise FactorizationError("replan before analysis")
        self._create_plan()
        self._stage = 1

    def _prepare_matching(self):
        """Matching and scaling of ``matching_alg`` (the reference's ``_reorder!`` and ``_matching_state``,
        src/solver.jl:545-592), from the first batch member's values: the analysis, factorization and
        solve then work on ``M = (Dr A Dc)[:, q]`` ("G": the matched entry of row i moves to column i;
        its pattern is the stored one with relabeled columns, no value moves) or on ``D A D`` (the
        symmetric structures, whose inertia it keeps). Returns the column indices the analysis reads."""
        torch = self._torch
        alg = self.params["matching_alg"]
        self._matching = self._mdev = None
        if alg in ("default", "none", 0):
            return self.colval
        m = compute_matching(self.rowptr, self.colval, self.nzval[: self.nnz].cpu().numpy(), self.n, self.structure,
                             alg, view=self.view, index_base=self.index_base)
        rp = np.asarray(self.rowptr, np.int64) - self.index_base
        cols = np.asarray(self.colval, np.int64) - self.index_base
        rows = np.repeat(np.arange(self.n), np.diff(rp))
        w = m.rscale[rows] * m.cscale[cols]
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)  # noqa: E731
        perm0 = m.perm - 1
        self._matching = m
        self._mdev = {"w": dev(w), "w_host": w, "r": dev(m.rscale), "c": dev(m.cscale), "perm0": dev(perm0),
                      "c_perm": dev(m.cscale[perm0])}
        if self.structure != "G":
            return self.colval
        inv = np.empty(self.n, np.int64)
        inv[perm0] = np.arange(self.n)
        return inv[cols] + self.index_base

    def _factor_values(self):
        """The values the numeric phase factors: the user's, or scaled by the matching's entry weights."""
        if self._matching is None:
            return self.nzval
        w = self._mdev["w"]
        return (self.nzval.reshape(self.nbatch, -1) * w).reshape(-1).contiguous()

    def _scaled_rhs(self, Bcm, mode):
        """The right-hand sides of the matched system (last axis: the n rows). "G": M y = Dr b, or for
        A^T: M^T z = Q^T Dc b; the symmetric structures: (D A D) y = D b."""
        d = self._mdev
        if self._matching.symmetric or mode == 0:
            return (Bcm * d["r"]).contiguous()
        return (Bcm * d["c"])[..., d["perm0"]].contiguous()

    def _scaled_solution(self, Xcm, mode):
        """The matched system's unknowns from x (the inverse of _unscaled_solution)."""
        d = self._mdev
        if self._matching.symmetric or mode != 0:
            return (Xcm / d["r"]).contiguous()
        return (Xcm[..., d["perm0"]] / d["c_perm"]).contiguous()

    def _unscaled_solution(self, Ycm, mode):
        """x from the matched system's solution: "G" x = Dc Q y (A), x = Dr z (A^T); symmetric x = D y."""
        d = self._mdev
        if self._matching.symmetric or mode != 0:
            return Ycm * d["r"]
        X = self._torch.empty_like(Ycm)
        X[..., d["perm0"]] = Ycm * d["c_perm"]
        return X

    def _plan_exists(self):
        return getattr(self, "_plan", None) is not None

    def getparam(self, name):
        lib = numeric_lib()
        if name == "info":
            return int(self._info[0]) if self.nbatch == 1 else self._info.copy()
        if name == "ir_n_steps" and self._ir_steps >= 0:
            return self._ir_steps
        if name in ("perm_matching", "scale_row", "scale_col"):
            self._need(1, name)
            if self._matching is None:
                raise InvalidValueError(f"{name!r} needs matching_alg other than \"default\"")
            m = self._matching
            return {"perm_matching": m.perm, "scale_row": m.rscale, "scale_col": m.cscale}[name].copy()
        if name in ("perm_reorder_row", "perm_reorder_col") and self._stage < 1 and getattr(self, "_reordered", False):
            # after "reordering" alone: the ordering algorithm's permutation (src/solver.jl:1082-1085)
            return self.symbolic.ordering.copy()
        if name in ("perm_reorder_row", "perm_reorder_col", "perm_col"):
            self._need(1, name)
            if name == "perm_col" and self._matching is not None and self.structure == "G":
                return self._matching.perm[self.symbolic.perm - 1]
            return self.symbolic.perm.copy()
        if name == "perm_row":
            self._need(1, name)
            if self.structure == "G" and self._stage >= 2:
                piv = np.zeros(self.n, np.int32)
                _check(lib.sdsb200_get_pivots(self._plan, 0, piv.ctypes.data, None, None), lib)
                return self.symbolic.perm[piv - 1]
            return self.symbolic.perm.copy()
        if name in ("lu_nnz", "flops", "nsuperpanels"):
            self._need(1, name)
            return {"lu_nnz": self.symbolic.nnz_L, "flops": self.symbolic.flops, "nsuperpanels": self.symbolic.ns}[name]
        if name in ("inertia", "npivots", "pivot_stats"):
            self._need(2, name)
            out = []
            for k in range(self.nbatch):
                tot = np.zeros(6, np.int64)
                _check(lib.sdsb200_get_stats(self._plan, k, None, tot.ctypes.data), lib)
                st = dict(npos=int(tot[0]), nneg=int(tot[1]), nzero=int(tot[2]), nperturbed=int(tot[3]),
                          n2x2=int(tot[4]))
                out.append(st["nperturbed"] if name == "npivots" else
                           (st["npos"], st["nneg"]) if name == "inertia" else st)
            return out[0] if self.nbatch == 1 else out
        if name == "diag":
            self._need(2, name)
            return self.factor_diag()
        if name == "memory_estimates":
            self._need(1, name)
            st = lambda k: int(lib.sdsb200_plan_stat(self._plan, k.encode()))  # noqa: E731
            host = sum(int(a.nbytes) for a in self.symbolic.maps.values())
            extra = 0
            if self._mdev is not None:
                extra = sum(int(t.numel() * t.element_size()) for t in self._mdev.values()
                            if isinstance(t, self._torch.Tensor) and t.is_cuda)
                extra += self.nnz * self.nbatch * 8          # the scaled values
            es = 4 if self._precision() == 1 else 8
            return memory_slots(self.structure, self.n, self.symbolic.ns, self.nbatch, es, st("factor_len"),
                                st("cb_len"), st("device_bytes"), host, extra)
        if name in ("schur_shape", "schur_matrix"):
            self._need(1 if name == "schur_shape" else 2, name)
            if self.symbolic.schur == 0:
                raise InvalidValueError(f"the data parameter {name!r} needs an analysis with schur_mode = 1")
            return self._schur_shape() if name == "schur_shape" else self._schur_matrix()
        if name in self.params:
            return self.params[name]
        raise InvalidValueError(f"unknown parameter {name!r}")

    def _need(self, stage, name):
        if self._stage < stage:
            raise FactorizationError(f"{name!r} is not available before the "
                                     f"{'analysis' if stage == 1 else 'factorization'}")

    # -- phases -----------------------------------------------------------------------------------------------
    def execute(self, phase, X=None, B=None):
        """``execute!(phase, solver, X, B)``."""
        if phase == "analysis":
            return self._analysis()
        if phase == "reordering":
            return self._analysis(plan=False)
        if phase == "symbolic_factorization":
            return self._symbolic_factorization()
        if phase in ("factorization", "refactorization"):
            return self._factorize(refactor=phase == "refactorization")
        if phase in ("solve", "solve_refinement", "solve_fwd_perm", "solve_fwd", "solve_diag", "solve_bwd",
                     "solve_bwd_perm", "solve_fwd_schur", "solve_bwd_schur"):
            if self._stage < 2:
                raise FactorizationError(f"phase {phase!r} before the factorization")
            self._sync_members()
            if self.symbolic.schur > 0:
                return self._schur_phase(phase, X, B)
            if phase in ("solve_fwd_schur", "solve_bwd_schur"):
                raise FactorizationError(f"phase {phase!r} needs an analysis with schur_mode = 1")
            if phase == "solve_refinement":
                return self._refine(X, B)
            if phase != "solve":
                return self._sub_phase(phase, X, B)
            return self._solve(X, B)
        raise InvalidValueError(f"unknown phase {phase!r}")

    def _opts(self):
        o = capi.Opts()
        lib = numeric_lib()
        lib.sdsb200_default_opts(C.byref(o))
        p = self.params
        o.pivot_type = capi.PIVOT_TYPE[p["pivot_type"]]
        o.pivot_threshold = float(p["pivot_threshold"])
        o.pivot_epsilon = -1.0 if p["pivot_epsilon"] is None else float(p["pivot_epsilon"])
        o.pivot_epsilon_alg = 1 if p["pivot_epsilon_alg"] == "algo1" else 0
        o.ir_n_steps = int(p["ir_n_steps"])
        o.ir_tol = float(p["ir_tol"])
        o.solve_mode = int(p["solve_mode"])
        o.deterministic_mode = int(p["deterministic_mode"])
        return o

    def _precision(self):
        fp = self.params["factor_precision"]
        return 1 if fp in ("fp32", "float32") else 0

    def _analysis(self, plan=True):
        """``"analysis"`` = ``"reordering"`` then ``"symbolic_factorization"`` (src/solver.jl:444-452). The
        host analysis (ordering, supernodes, maps) runs here; ``plan=False`` ("reordering") stops before
        the device plan, which ``"symbolic_factorization"`` then builds."""
        p = self.params
        if self._plan_exists():                 # a new analysis drops the previous one's plan
            numeric_lib().sdsb200_plan_destroy(self._plan)
            self._plan = None
        self._stage = 0
        self._reordered = False
        flags = None
        if int(p["schur_mode"]) == 1:
            # Schur complement mode (src/solver.jl:471-475, 554-559): the flagged rows and columns last, as
            # one root front that the factorization assembles and does not factor
            if p["matching_alg"] != "default":
                raise NotSupportedError("matching_alg is not supported with schur_mode = 1")
            if self.nbatch > 1:
                raise NotSupportedError("schur_mode = 1 is not supported for uniform batches")
            if p["user_schur_indices"] is None:
                raise InvalidValueError("schur_mode = 1 needs \"user_schur_indices\" (n flags 0/1)")
            flags = np.asarray(p["user_schur_indices"]).reshape(-1)
            if flags.size != self.n:
                raise InvalidValueError(f"user_schur_indices has {flags.size} entries, the matrix has {self.n} rows")
            if not np.any(flags != 0):
                raise InvalidValueError("user_schur_indices selects no row: the Schur complement would be empty")
        self._schur_dest = None
        nz_host = self.nzval[: self.nnz].cpu().numpy() if self.structure == "S" else None
        colval = self._prepare_matching()
        user_pairs = None
        if self._matching is not None and nz_host is not None:
            if self._matching.job == 5 and p["pivot_pairs"] != "none":
                # "S" with a job-5 matching: the 2x2 pairs come from the matching's cycles (src/solver.jl:560-566)
                user_pairs = matching_pairs(self.rowptr, self.colval, nz_host, self.n, self._matching,
                                            pivot_pairs=p["pivot_pairs"],
                                            pivot_pair_tolerance=p["pivot_pair_tolerance"], view=self.view,
                                            index_base=self.index_base)
            nz_host = nz_host * self._mdev["w_host"]
        self.symbolic = analyze(self.rowptr, colval, self.n, self.structure, nzval=nz_host, view=self.view,
                                index_base=self.index_base, reordering=p["reordering_alg"],
                                user_perm=p["user_perm"], pivot_pairs=p["pivot_pairs"],
                                pivot_pair_tolerance=p["pivot_pair_tolerance"],
                                pivot_threshold=p["pivot_threshold"], use_superpanels=p["use_superpanels"],
                                amalgamation=tuple(p["amalgamation"]), user_pairs=user_pairs,
                                user_schur_indices=flags)
        self._reordered = True
        if plan:
            self._symbolic_factorization()

    def _symbolic_factorization(self):
        """``"symbolic_factorization"`` (_symbolic!, src/solver.jl:609-660): the device plan of the analysis
        "reordering" computed (the maps and every buffer of the numeric and solve phases)."""
        if not getattr(self, "_reordered", False):
            raise FactorizationError("phase \"symbolic_factorization\" needs \"reordering\" (or run \"analysis\")")
        self._create_plan()
        self._stage = 1

    def _create_plan(self):
        lib = numeric_lib()
        if self._plan is not None:
            lib.sdsb200_plan_destroy(self._plan)
            self._plan = None
        S = self.symbolic
        keep = {}
        sym = capi.Symbolic()
        sym.n, sym.nnz, sym.ns = S.n, S.nnz, S.ns
        sym.index_width = 8
        sym.structure = capi.STRUCTURE[self.structure]
        for nm in ("perm", "super_ptr", "snparent", "rowptr", "rowval", "front_ptr", "child_ptr", "child_list",
                   "relind_ptr", "relind", "amap", "amap_ptr", "amap_src", "full_rowptr", "full_colval",
                   "full_srcptr", "full_src"):
            a = np.ascontiguousarray(getattr(S, nm), dtype=np.int64)
            if a.size == 0:
                a = np.zeros(1, np.int64)
            keep[nm] = a
            setattr(sym, nm, a.ctypes.data)
        sym.full_nnz = int(S.full_colval.size)
        sym.full_nsrc = int(S.full_src.size)
        sym.schur = int(getattr(S, "schur", 0))
        po = capi.PlanOptions(nbatch=self.nbatch, precision=self._precision(), max_nrhs=int(self.params["max_nrhs"]),
                              tuning=int(self.params["tuning"]))
        plan = C.c_void_p()
        stream = self._torch.cuda.current_stream(self.device).cuda_stream
        _check(lib.sdsb200_plan_create(C.byref(plan), C.byref(sym), C.byref(po), C.c_void_p(stream)), lib)
        self._plan = plan
        self._members_dirty = self._subset()     # a new plan processes every member
        if self.params["user_host_interrupt"] is not None:
            flag = self.params["user_host_interrupt"]
            lib.sdsb200_set_interrupt(self._plan, C.addressof(flag))

    def _subset(self):
        return int(self.params["ubatch_index"]) != -1 or self.params["ubatch_mask"] is not None

    def _members(self):
        return active_members(self.nbatch, int(self.params["ubatch_index"]), self.params["ubatch_mask"])

    def _sync_members(self):
        """The members of the next numeric or solve phase (_set_members!, src/solver.jl:694-705), sent to the
        plan when ubatch_index or ubatch_mask changed; InvalidValueError for a selection outside the batch
        or an empty one."""
        if self._plan_exists() and getattr(self, "_members_dirty", False):
            self._apply_members()
            self._members_dirty = False

    def _apply_members(self):
        """set_members! (src/numeric/storage.jl:290-306) for ``ubatch_index`` and ``ubatch_mask``."""
        lib = numeric_lib()
        if not self._subset():
            _check(lib.sdsb200_set_members(self._plan, None, -1), lib)
            return
        members = self._members()
        if not members:
            raise InvalidValueError("ubatch_index and ubatch_mask select no batch member")
        m = np.asarray(members, np.int32)
        _check(lib.sdsb200_set_members(self._plan, m.ctypes.data, len(members)), lib)

    def _factorize(self, refactor=False):
        if self._stage < 1:
            raise FactorizationError("factorization before analysis")
        self._sync_members()
        lib = numeric_lib()
        ps = self.params["pivot_sign"]
        ps_arr = None if ps is None else np.ascontiguousarray(ps, dtype=np.int8)
        info = np.zeros(self.nbatch, np.int64)
        stream = self._torch.cuda.current_stream(self.device).cuda_stream
        o = self._opts()
        self._fvals = self._factor_values()
        rc = lib.sdsb200_factor(self._plan, C.c_void_p(self._fvals.data_ptr()),
                                ps_arr.ctypes.data if ps_arr is not None else None, C.byref(o), info.ctypes.data,
                                C.c_void_p(stream))
        if rc == capi.INTERRUPTED:
            self._stage = 1
        _check(rc, lib)
        self._info = info
        self._stage = 2
        return int(info[0]) if self.nbatch == 1 else info

    def _solve(self, X, B):
        torch = self._torch
        if self._stage < 2:
            raise FactorizationError("solve before factorization")
        lib = numeric_lib()
        n = self.n
        Bt = B if isinstance(B, torch.Tensor) else torch.from_numpy(np.asarray(B, dtype=np.float64))
        Bt = Bt.to(self.device, torch.float64)
        # a batch's right-hand sides are member after member, whatever the shape (a vector too)
        Bm = Bt.reshape(n, -1) if self.nbatch == 1 else Bt.reshape(self.nbatch, n, -1)
        # column-major storage: (members, nrhs, n) contiguous
        if Bm.dim() == 2:
            Bcm = Bm.t().contiguous()
            nrhs = Bm.shape[1]
        else:
            Bcm = Bm.transpose(1, 2).contiguous()
            nrhs = Bm.shape[2]
        o = self._opts()
        if self._matching is not None:
            Bcm = self._scaled_rhs(Bcm, int(o.solve_mode))
        subset = self._subset() and self.nbatch > 1
        Xcm = torch.zeros_like(Bcm) if subset else torch.empty_like(Bcm)
        fgmres = self.params["ir_mode"] == "fgmres" and o.ir_n_steps > 0
        if fgmres:
            # FGMRES-IR (fgmres_refine!, src/solve/refinement.jl:577-614): a plain solve, then the
            # Krylov refinement on the host above the C ABI
            if self._subset():
                raise NotSupportedError("ir_mode \"fgmres\" refines all batch members together")
            fg_steps, fg_tol = int(o.ir_n_steps), float(o.ir_tol)
            o.ir_n_steps = 0
        steps = C.c_int32(0)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        vals = self.nzval if self._matching is None else self._factor_values()
        _check(lib.sdsb200_solve(self._plan, C.c_void_p(Xcm.data_ptr()), n, C.c_void_p(Bcm.data_ptr()), n, nrhs,
                                 C.c_void_p(vals.data_ptr()), C.byref(o), C.byref(steps),
                                 C.c_void_p(stream)), lib)
        self._ir_steps = int(steps.value) if o.ir_n_steps > 0 else -1
        if fgmres:
            from .refinement import fgmres_refine

            self._ir_steps = fgmres_refine(self, Xcm, Bcm, nrhs, int(o.solve_mode), fg_steps, fg_tol, nzval=vals)
        if self._matching is not None:   # refinement ran on the matched system; back to A's unknowns
            Xcm = self._unscaled_solution(Xcm, int(o.solve_mode))
        out = Xcm.t() if Xcm.dim() == 2 else Xcm.transpose(1, 2)
        out = out.reshape(Bt.shape)
        if X is not None and subset:
            out = self._keep_inactive(X, out)
        if X is not None:
            if isinstance(X, torch.Tensor):
                X.copy_(out)
                return X
            np.copyto(X, out.cpu().numpy())
            return X
        return out

    # -- solve sub-phases and Schur complement mode -------------------------------------------------------------
    def _colmajor(self, B):
        """B (n, n x nrhs, or nbatch x n x nrhs; host or device) as a device column-major tensor
        (members, nrhs, n), with its nrhs and a function that maps a result back to B's shape."""
        torch = self._torch
        Bt = B if isinstance(B, torch.Tensor) else torch.from_numpy(np.asarray(B, dtype=np.float64))
        Bt = Bt.to(self.device, torch.float64)
        n = self.n
        # a batch's right-hand sides are member after member, whatever the shape (a vector too)
        Bm = Bt.reshape(n, -1) if self.nbatch == 1 else Bt.reshape(self.nbatch, n, -1)
        if Bm.dim() == 2:
            cm, nrhs = Bm.t().contiguous(), Bm.shape[1]
        else:
            cm, nrhs = Bm.transpose(1, 2).contiguous(), Bm.shape[2]
        shape = Bt.shape

        def back(Xcm):
            out = Xcm.t() if Xcm.dim() == 2 else Xcm.transpose(1, 2)
            return out.reshape(shape)

        return cm, int(nrhs), back

    def _keep_inactive(self, X, out):
        """``out`` with the inactive batch members' entries taken from X (ubatch_index / ubatch_mask: the other
        members' solutions are left as they are)."""
        torch = self._torch
        Xt = X if isinstance(X, torch.Tensor) else torch.from_numpy(np.asarray(X, dtype=np.float64))
        cur = Xt.to(self.device, torch.float64).reshape(self.nbatch, self.n, -1).clone()
        sel = torch.as_tensor(self._members(), device=self.device, dtype=torch.int64)
        cur[sel] = out.reshape(self.nbatch, self.n, -1)[sel]
        return cur.reshape(out.shape)

    def _deliver(self, X, out):
        if X is None:
            return out
        if isinstance(X, self._torch.Tensor):
            X.copy_(out)
            return X
        np.copyto(X, out.cpu().numpy())
        return X

    def _run_phase(self, code, Xcm, Bcm, nrhs, o=None):
        lib = numeric_lib()
        stream = self._torch.cuda.current_stream(self.device).cuda_stream
        o = self._opts() if o is None else o
        n = self.n
        _check(lib.sdsb200_solve_phase(self._plan, capi.PHASE[code],
                                       C.c_void_p(Xcm.data_ptr()) if Xcm is not None else None, n,
                                       C.c_void_p(Bcm.data_ptr()) if Bcm is not None else None, n, nrhs,
                                       C.byref(o), C.c_void_p(stream)), lib)

    def _phase_nrhs(self, X, B):
        src = B if B is not None else X
        if src is not None:
            return self._colmajor(src)[1]
        if getattr(self, "_last_phase_nrhs", None) is None:
            raise FactorizationError("no right-hand side: run \"solve_fwd_perm\" first")
        return self._last_phase_nrhs

    def _sub_phase(self, phase, X, B):
        """``execute!(phase)`` for the solve sub-phases (src/solver.jl:856-867): "solve_fwd_perm" reads B into
        the plan's working vectors Y (factor order; with matching, scaled as the complete solve scales it),
        "solve_fwd", "solve_diag" and "solve_bwd" work on Y, and "solve_bwd_perm" writes X from Y (and
        returns it). No refinement."""
        o = self._opts()
        if phase == "solve_fwd_perm":
            if B is None:
                raise InvalidValueError("\"solve_fwd_perm\" needs B")
            Bcm, nrhs, _ = self._colmajor(B)
            if self._matching is not None:
                Bcm = self._scaled_rhs(Bcm, int(o.solve_mode))
            self._run_phase("fwd_perm", None, Bcm, nrhs, o)
            self._last_phase_nrhs = nrhs
            return None
        if phase in ("solve_fwd", "solve_diag", "solve_bwd"):
            self._run_phase(phase[6:], None, None, self._phase_nrhs(X, B), o)
            return None
        # solve_bwd_perm
        src = X if X is not None else B
        if src is None:
            raise InvalidValueError("\"solve_bwd_perm\" needs X (or B for its shape)")
        Xcm, nrhs, back = self._colmajor(src)
        Xcm = self._torch.empty_like(Xcm)
        self._run_phase("bwd_perm", Xcm, None, nrhs, o)
        if self._matching is not None:
            Xcm = self._unscaled_solution(Xcm, int(o.solve_mode))
        out = back(Xcm)
        if X is not None and self._subset() and self.nbatch > 1:
            out = self._keep_inactive(X, out)
        return self._deliver(X, out)

    def _refine(self, X, B):
        """``execute!("solve_refinement", X, B)`` (_refine_phase!, src/solver.jl:902-926): refine the given
        solution X of op(A) X = B in place, ``ir_n_steps`` steps of plain refinement (stopping once
        max_k ||R_k|| / ||B_k|| <= ``ir_tol`` when ir_tol > 0) or of FGMRES-IR (``ir_mode = "fgmres"``).
        With ir_n_steps = 0, X is left as it is. X and B must not alias. With a matching, the
        refinement runs on the matched system, as the complete solve's does."""
        torch = self._torch
        if X is None or B is None:
            raise InvalidValueError("\"solve_refinement\" needs X (the solution to refine) and B")
        if isinstance(X, torch.Tensor) and isinstance(B, torch.Tensor) and X.data_ptr() == B.data_ptr():
            raise InvalidValueError("\"solve_refinement\" needs the original right-hand side: X and B must not alias")
        if isinstance(X, np.ndarray) and isinstance(B, np.ndarray) and np.shares_memory(X, B):
            raise InvalidValueError("\"solve_refinement\" needs the original right-hand side: X and B must not alias")
        o = self._opts()
        nsteps, tol, mode = int(o.ir_n_steps), float(o.ir_tol), int(o.solve_mode)
        if nsteps <= 0:
            self._ir_steps = 0
            return X
        if self._subset():
            raise NotSupportedError("\"solve_refinement\" refines all batch members together")
        Xcm, nrhs, back = self._colmajor(X)
        Bcm, nrhs_b, _ = self._colmajor(B)
        if nrhs_b != nrhs:
            raise InvalidValueError(f"X has {nrhs} right-hand sides, B {nrhs_b}")
        vals = self.nzval if self._matching is None else self._factor_values()
        if self._matching is not None:
            Xcm = self._scaled_solution(Xcm, mode)
            Bcm = self._scaled_rhs(Bcm, mode)
        Xcm = Xcm.clone()
        from .refinement import fgmres_refine, ir_refine

        if self.params["ir_mode"] == "fgmres":
            self._ir_steps = fgmres_refine(self, Xcm, Bcm, nrhs, mode, nsteps, tol, nzval=vals)
            stopped = False
        else:
            flag = self.params["user_host_interrupt"]
            poll = (lambda: flag.value != 0) if flag is not None else None
            self._ir_steps, stopped = ir_refine(self, Xcm, Bcm, nrhs, mode, nsteps, tol, nzval=vals,
                                                interrupted=poll)
        if self._matching is not None:
            Xcm = self._unscaled_solution(Xcm, mode)
        out = self._deliver(X, back(Xcm))
        if stopped:
            raise InterruptedError_("interrupted by user_host_interrupt")
        return out

    def _schur_phase(self, phase, X, B):
        """The solve phases of Schur complement mode (_schur_solve_phase!, src/solver.jl:876-900). Each reads B
        and writes X (returned; X is B allowed); the vectors are in factor order, the last ns entries being the
        Schur block in increasing original order:
        "solve_fwd_schur": permutation and forward sweep; the Schur block of X is b2 - A21 A11^{-1} b1;
        "solve_diag": D^{-1} of LDLT on the factored part (the identity for Cholesky and LU, and on the Schur
        block);
        "solve_bwd_schur": with the Schur solution x2 in the Schur block of B, the diagonal of LU, the
        backward sweep and the inverse permutation: X solves op(A) x = b."""
        if phase not in ("solve_fwd_schur", "solve_diag", "solve_bwd_schur"):
            raise NotSupportedError(f"phase {phase!r} with schur_mode = 1: the factorization is partial; use "
                                    "\"solve_fwd_schur\", \"solve_diag\" and \"solve_bwd_schur\"")
        if B is None:
            raise InvalidValueError(f"phase {phase!r} needs B")
        o = self._opts()
        Bcm, nrhs, back = self._colmajor(B)
        Xcm = self._torch.empty_like(Bcm)
        lu = self.structure == "G"
        if phase == "solve_fwd_schur":
            steps = [("fwd_perm", None, Bcm), ("fwd", None, None), ("store", Xcm, None)]
        elif phase == "solve_diag":
            steps = [("load", None, Bcm)] + ([] if lu else [("diag", None, None)]) + [("store", Xcm, None)]
        else:
            steps = ([("load", None, Bcm)] + ([("diag", None, None)] if lu else []) +
                     [("bwd", None, None), ("bwd_perm", Xcm, None)])
        for code, x, b in steps:
            self._run_phase(code, x, b, nrhs, o)
        return self._deliver(X, back(Xcm))

    def _schur_pattern_nnz(self, lower):
        S = self.symbolic
        rp, cv = S.schur_rowptr, S.schur_colval
        if not lower:
            return int(cv.size)
        rows = np.repeat(np.arange(1, S.schur_n + 1), np.diff(rp))
        return int(np.count_nonzero(cv <= rows))

    def _schur_shape(self):
        """``getparam("schur_shape")`` (src/solver.jl:1267-1271): (ns, ns, nnz of the pattern of S; one triangle
        with the diagonal for the symmetric structures)."""
        ns = self.symbolic.schur_n
        return (ns, ns, self._schur_pattern_nnz(self.structure != "G"))

    def _set_schur_dest(self, value):
        """``setparam!("schur_matrix", dest)`` (src/solver.jl:1303-1316): the destination that
        ``getparam("schur_matrix")`` fills: None (a new dense matrix each time), a dense (ns, ns) float64 CUDA
        tensor, or a sparse ``(rowptr, colval, nzval)`` triple of CUDA tensors (CSR with the pattern of
        ``schur_shape`` over the full matrix or, as a 4th item 'L' or 'U', one triangle; 0- or 1-based)."""
        torch = self._torch
        sym = getattr(self, "symbolic", None)
        if sym is None or sym.schur == 0:
            raise InvalidValueError("the data parameter \"schur_matrix\" needs an analysis with schur_mode = 1")
        ns = self.symbolic.schur_n
        if value is None:
            self._schur_dest = None
            return
        if isinstance(value, torch.Tensor):
            if tuple(value.shape) != (ns, ns) or value.dtype != torch.float64 or value.device.type != "cuda":
                raise InvalidValueError(f"schur_matrix: expected a ({ns}, {ns}) float64 CUDA tensor")
            self._schur_dest = value
            return
        if isinstance(value, tuple) and len(value) in (3, 4):
            view = value[3] if len(value) == 4 else "F"
            if view not in ("F", "L", "U"):
                raise InvalidValueError("schur_matrix: the view must be 'F', 'L' or 'U'")
            rowptr, colval, nzval = value[:3]
            nz = self._schur_pattern_nnz(view != "F")
            if rowptr.numel() != ns + 1 or colval.numel() != nz or nzval.numel() != nz:
                raise InvalidValueError(f"schur_matrix: the sparse Schur complement with view {view!r} has {nz} "
                                        f"entries; see \"schur_shape\"")
            self._schur_dest = (rowptr, colval, nzval, view)
            return
        raise InvalidValueError("schur_matrix: expected None, a dense CUDA tensor or (rowptr, colval, nzval[, view])")

    def _schur_matrix(self):
        """``getparam("schur_matrix")`` (src/solver.jl:1114-1121): S = A22 - A21 A11^{-1} A12 of the last
        factorization, written into the registered destination (or a new dense CUDA matrix) and returned."""
        torch = self._torch
        lib = numeric_lib()
        ns = self.symbolic.schur_n
        stream = torch.cuda.current_stream(self.device).cuda_stream
        dest = getattr(self, "_schur_dest", None)
        D = dest if isinstance(dest, torch.Tensor) else torch.empty((ns, ns), dtype=torch.float64, device=self.device)
        # D is row-major (ns, ns) for torch: the column-major export of S^T lands as S
        _check(lib.sdsb200_schur_matrix(self._plan, 0, C.c_void_p(D.data_ptr()), ns, 1, C.c_void_p(stream)), lib)
        if not isinstance(dest, tuple):
            return D
        rowptr, colval, nzval, _ = dest
        base = int(rowptr[0].item())
        rows = torch.repeat_interleave(torch.arange(ns, device=D.device),
                                       (rowptr[1:] - rowptr[:-1]).to(torch.int64))
        nzval.copy_(D[rows, colval.to(torch.int64) - base])
        return nzval

    # -- outputs for tests -------------------------------------------------------------------------------------
    def factor_host(self, member=0):
        """Panels as host FP64 arrays (factor, ufactor or None), the reference's ``host_numeric``."""
        lib = numeric_lib()
        flen = self.symbolic.factor_len
        fac = np.zeros(max(flen, 1))
        ufac = np.zeros(max(flen, 1)) if self.structure == "G" else None
        _check(lib.sdsb200_get_factor(self._plan, member, fac.ctypes.data,
                                      ufac.ctypes.data if ufac is not None else None), lib)
        return fac, ufac

    def pivots_host(self, member=0):
        lib = numeric_lib()
        piv = np.zeros(max(self.n, 1), np.int32)
        kind = np.zeros(max(self.n, 1), np.int8)
        d = np.zeros(max(2 * self.n, 1))
        _check(lib.sdsb200_get_pivots(self._plan, member, piv.ctypes.data, kind.ctypes.data, d.ctypes.data), lib)
        return piv, kind, d

    def stats_host(self, member=0):
        lib = numeric_lib()
        st = np.zeros(max(6 * self.symbolic.ns, 1), np.int64)
        _check(lib.sdsb200_get_stats(self._plan, member, st.ctypes.data, None), lib)
        return st[: 6 * self.symbolic.ns].reshape(-1, 6)

    def factor_diag(self, member=0):
        """``getparam("diag")``: diagonal of L (Cholesky) or of D (LDLT, LU) in factor order."""
        fac, _ = self.factor_host(member)
        if self.structure == "SPD":
            S = self.symbolic
            out = np.zeros(self.n)
            for s in range(S.ns):
                f, w, base, c0 = (int(S.front_nrows[s]), int(S.front_ncols[s]), int(S.front_ptr[s]) - 1,
                                  int(S.super_ptr[s]) - 1)
                for j in range(w):
                    out[c0 + j] = fac[base + j * f + j]
            return out
        return self.pivots_host(member)[2][: self.n].copy()

    def plan_stat(self, name):
        return numeric_lib().sdsb200_plan_stat(self._plan, name.encode())

    def close(self):
        if self._plan is not None:
            numeric_lib().sdsb200_plan_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

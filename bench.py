"""Benchmark of the numeric phase: factor + solve of the 3-D Laplacian workload.

Workload (one step): factorization of the 7-point Laplacian on a 48 x 48 x 48
grid (n = 110 592, nested dissection) and the solve of 4 right-hand sides
U[-1, 1], to a scaled backward error <= 1e-12, in two forms:

* mixed: FP32 factor (assembly and Schur updates in FP32) + FP64 iterative
  refinement (FP64 residual), the headline form;
* fp64: every operation in FP64.

value = algorithmic GFLOP/s of one step (factorization flops in the
reference's convention sum over panel columns of rows^2, plus 4 nnz_stored
nrhs for the solve), with the values and right-hand sides resident in HBM.
e2e = the same through the public DirectSolver API with host buffers (H2D of
values and right-hand sides, D2H of the solution inside the timed region).

`--impl reference` times the CPU oracle (this repository's restatement of the
reference's CPU factorization and solve; the reference itself is Julia, which
is not installed) on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "sparsedirectsolver.jl_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

METRIC = "factor+solve ms & GFLOP/s at bwd err ≤1e-12: mixed+IR vs FP64, 1 B200"
GRID = 48
NRHS = 4
BERR_TARGET = 1e-12


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=GRID)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--config", default="c2", choices=["c2", "c1", "c3", "c4", "c4u", "c5"],
                    help="c2 (default): lap3d_48 SPD, the headline line. The others print one line each for the "
                         "other workloads: c1 lap2d_64 SPD AMD, c3 KKT LDL^T (n = 55 000), c4 1024 uneven "
                         "systems, c4u uniform batch 96x96 x 256, c5 LU convection-diffusion 40^3 with A and A^T")
    ap.add_argument("--tuning", default=None,
                    help="fsmall,wide,chains[,streams,steps,subtree]: fixed front tile shapes instead of the "
                         "autotuner's search (for profilers)")
    ap.add_argument("--amalgamation", default="512,0.25,8",
                    help="max_width,zero_fraction,min_width of the solver's supernode amalgamation (a solver option "
                         "of the reference's; its default is 32,0.25,8). The metric's flops are always those of the "
                         "default amalgamation, as the reference arm's")
    ap.add_argument("--once", choices=["fp64", "mixed"], default=None,
                    help="one analysis + factorization + solve of the workload in one form, untimed (for profilers); "
                         "with --config c3 or c5 that workload")
    ap.add_argument("--kkt-grid", type=int, default=200,
                    help="c3: the KKT's grid (200: n = 55 000; smaller grids scale the constraint count with the area)")
    return ap.parse_args()


def run_once(args):
    """One factorization and one solve of the workload (the case the profiles in profiles/ capture)."""
    import torch

    from sdsb200 import matrices as M
    from sdsb200.solver import DirectSolver

    kw = dict(factor_precision="fp32", ir_n_steps=20, ir_tol=BERR_TARGET) if args.once == "mixed" else {}
    if args.tuning:
        from sdsb200.capi import tuning as make_tuning

        kw["tuning"] = make_tuning(*[int(v) for v in args.tuning.split(",")])
    if args.config in ("c3", "c5"):
        A, structure, ckw, nrhs = config_matrix(args)
        kw = {**ckw, **kw}
        b = M.rhs(A.shape[0], nrhs, seed=0)
        size = {"kkt_grid": args.kkt_grid} if args.config == "c3" else {"grid": 40}
    else:
        A, b = workload(args.grid)
        structure, nrhs = "SPD", NRHS
        kw["reordering_alg"] = "nd"
        kw["amalgamation"] = amalgamation_of(args)
        size = {"grid": args.grid}
    ds = DirectSolver(A, structure, max_nrhs=nrhs, **kw)
    ds.execute("analysis")
    ds.execute("factorization")
    x = ds.execute("solve", None, torch.from_numpy(np.ascontiguousarray(b)).cuda())
    torch.cuda.synchronize()
    berr = M.scaled_backward_error(A, x.cpu().numpy().reshape(A.shape[0], -1), b.reshape(A.shape[0], -1))
    print(json.dumps({"once": args.once, "config": args.config, **size, "bwd_err": berr}), flush=True)
    assert berr <= BERR_TARGET


def amalgamation_of(args):
    v = [x for x in args.amalgamation.split(",")]
    return (int(v[0]), float(v[1]), int(v[2]))


def config_matrix(args):
    """The matrix, structure, solver options and right-hand-side count of --config c1, c3 or c5."""
    from sdsb200 import matrices as M

    if args.config == "c1":
        return M.lap2d_shifted(64, 64, seed=0), "SPD", dict(reordering_alg="amd"), 1
    if args.config == "c3":
        # statically perturbed pivots make the plain solve inexact: both forms refine to 1e-12
        g = args.kkt_grid
        return M.kkt(g, g, int(round(15000 * (g / 200) ** 2)), seed=0), "S", dict(ir_n_steps=20, ir_tol=BERR_TARGET), 1
    return M.convection_diffusion3d(40, 40, 40, seed=0), "G", dict(pivot_threshold=0.1, reordering_alg="nd"), 8


def _time(torch, fn, steps, warmup):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def max_over_ranks(value, dist, device):
    """The largest value over the ranks of the process group (each replica's step time; the job's
    time is the slowest replica's)."""
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_config(args):
    """One JSON line for a workload other than the headline one (FP64 and mixed forms side by side)."""
    import torch

    from oracle.oracle import Oracle
    from sdsb200 import matrices as M
    from sdsb200.solver import DirectSolver

    rng = np.random.default_rng(0)
    cfg = args.config
    line = {"config": cfg, "steps": args.steps, "warmup": args.warmup, "data": "synthetic", "forms": {}}
    mixed_kw = dict(factor_precision="fp32", ir_n_steps=20, ir_tol=BERR_TARGET)
    if cfg in ("c1", "c3", "c5"):
        A, structure, kw, nrhs = config_matrix(args)
        if cfg == "c1":
            name = "lap2d_64 SPD Cholesky, AMD, 1 RHS"
        elif cfg == "c3":
            name = "KKT [H J^T; J 0] n = %d LDL^T (Bunch-Kaufman, pivot pairs), 1 RHS, FP64 refinement" % A.shape[0]
        else:
            name = "convection-diffusion 40^3 LU (threshold 0.1), 8 RHS, solves with A and A^T"
        n = A.shape[0]
        b = M.rhs(n, nrhs, seed=0)
        bt = torch.from_numpy(np.ascontiguousarray(b)).cuda()
        line["workload"] = name
        line["n"], line["nnz"] = int(n), int(A.nnz)
        if cfg == "c3" and args.kkt_grid == 200:
            line["inertia_expected"] = [40000, 15000]
        base = None
        for form, fkw in (("fp64", {}), ("mixed", mixed_kw)):
            ds = DirectSolver(A, structure, max_nrhs=nrhs, **{**kw, **fkw})
            t0 = time.perf_counter()
            if base is None:
                ds.execute("analysis")
                line["analysis_s"] = round(time.perf_counter() - t0, 2)
                base = ds
            else:                       # the same analysis, planned for this form
                ds.symbolic = base.symbolic
                ds._stage = 1
                ds.replan()
            S = ds.symbolic
            mult = 2.0 if structure == "G" else 1.0
            flops = mult * S.flops + (8.0 if structure == "G" else 4.0) * S.nnz_stored * nrhs
            line["factor_flops"], line["nnz_stored"] = mult * S.flops, int(S.nnz_stored)

            def step():
                ds.execute("factorization")
                ds.execute("solve", None, bt)
                if structure == "G":
                    ds.setparam("solve_mode", 1)
                    ds.execute("solve", None, bt)
                    ds.setparam("solve_mode", 0)

            ms = _time(torch, step, args.steps, args.warmup)
            x = ds.execute("solve", None, bt).cpu().numpy().reshape(n, -1)
            rec = {"ms_per_step": round(ms, 3), "gflops": round(flops / ms / 1e6, 2),
                   "bwd_err": M.scaled_backward_error(A, x, b), "ir_steps": ds.getparam("ir_n_steps") if form == "mixed" else 0}
            if structure == "G":
                ds.setparam("solve_mode", 1)
                xt = ds.execute("solve", None, bt).cpu().numpy().reshape(n, -1)
                ds.setparam("solve_mode", 0)
                rec["bwd_err_transpose"] = M.scaled_backward_error(A.T.tocsr(), xt, b)
            if structure == "S":
                rec["inertia"] = list(ds.getparam("inertia"))
                rec["npivots"] = int(ds.getparam("npivots"))
            line["forms"][form] = rec
            if form == "fp64" and mult * S.flops > 2e11:
                # the serial oracle runs at ~4 GFLOP/s: pivot parity at this size is left to the tests'
                # reduced sizes; the inertia of the KKT is a known answer
                line["cpu_oracle"] = "skipped: %.2e flops" % (mult * S.flops)
            elif form == "fp64":
                # parity with the CPU oracle on the same analysis
                O = Oracle(S)
                t0 = time.perf_counter()
                info = O.factorize(A.data, structure, **({"pivot_threshold": 0.1} if structure == "G" else {}))
                line["cpu_oracle_factor_s"] = round(time.perf_counter() - t0, 3)
                assert info == 0
                if structure == "G":
                    line["perm_row_equal_oracle"] = bool(np.array_equal(ds.getparam("perm_row"),
                                                                        S.perm[O.piv[:n] - 1]))
                    line["perm_col_equal_oracle"] = bool(np.array_equal(ds.getparam("perm_col"), S.perm))
                piv, kind, d = ds.pivots_host()
                line["pivots_equal_oracle"] = bool(np.array_equal(piv[:n], O.piv[:n]) and
                                                   np.array_equal(kind[:n], O.kind[:n]))
                if structure == "S":
                    line["inertia_oracle"] = [int(v) for v in O.stats_matrix().sum(0)[:2]]
                fac, _ = ds.factor_host()
                line["factor_rel_diff_oracle"] = float(np.abs(fac - O.factor[:fac.size]).max() /
                                                       max(1.0, np.abs(O.factor).max()))
        line["speedup_mixed_vs_fp64"] = round(line["forms"]["fp64"]["ms_per_step"] /
                                              line["forms"]["mixed"]["ms_per_step"], 3)
    else:
        from sdsb200.autotune import autotune, describe
        from sdsb200.batch import UnevenBatch

        if cfg == "c4":
            systems = M.uneven_batch(1024, 16, 48, 0.1, 0)
            line["workload"] = "1024 uneven 5-point Laplacians s x s, s ~ U[16, 48], + U[0, 0.1] shift, 1 RHS each"
            base = None
            for form, fkw in (("fp64", {}), ("mixed", dict(factor_precision="fp32", ir_n_steps=2, ir_tol=0.0))):
                ub = UnevenBatch(systems, "SPD", **fkw)
                t0 = time.perf_counter()
                if base is None:
                    ub.execute("analysis")
                    base = ub
                else:
                    ub.solver.symbolic = base.solver.symbolic
                    ub.solver._stage = 1
                    ub.solver.replan()
                analysis_s = time.perf_counter() - t0
                b = rng.uniform(-1, 1, ub.A.shape[0])
                bt = torch.from_numpy(b).cuda()
                times = autotune(ub.solver, bt, reps=2, use_cache=False)
                best = min(times, key=times.get)
                if form == "mixed":
                    # the fewest refinement steps whose every system meets the bound (untimed probe)
                    ub.execute("factorization")
                    for k in range(0, 9):
                        ub.solver.setparam("ir_n_steps", k)
                        if ub.backward_errors(ub.execute("solve", None, bt).cpu().numpy(), b).max() <= BERR_TARGET:
                            break

                def step():
                    ub.execute("factorization")
                    ub.execute("solve", None, bt)

                ms = _time(torch, step, args.steps, args.warmup)
                x = ub.execute("solve", None, bt).cpu().numpy()
                errs = ub.backward_errors(x, b)
                line["forms"][form] = {"ms_per_step": round(ms, 3), "systems_per_s": round(1024 / (ms / 1e3), 1),
                                       "max_bwd_err": float(errs.max()), "analysis_s": round(analysis_s, 2),
                                       "ir_steps": ub.solver.getparam("ir_n_steps") if form == "mixed" else 0,
                                       "tuning": describe(best),
                                       "autotune_ms": {str(describe(k)): round(v, 3) for k, v in times.items()},
                                       "solve_launches": int(ub.solver.plan_stat("launches_done"))}
            line["n_total"] = int(ub.A.shape[0])
        else:
            A = M.lap2d_shifted(96, 96, seed=0)
            vals = M.batch_members(A, 256, spread=0.1, seed=0)
            n = A.shape[0]
            line["workload"] = "uniform batch: 96 x 96 5-point Laplacian pattern, 256 members (values +-10 %), 1 RHS"
            b = rng.uniform(-1, 1, (256, n))
            bt = torch.from_numpy(b).cuda()
            for form, fkw in (("fp64", {}), ("mixed", dict(factor_precision="fp32", ir_n_steps=2, ir_tol=0.0))):
                ds = DirectSolver((A.indptr, A.indices, vals.reshape(-1), n), "SPD", **fkw)
                ds.execute("analysis")

                def member_errs(x):
                    out = []
                    for k in range(256):
                        Ak = A.copy()
                        Ak.data = vals[k]
                        out.append(M.scaled_backward_error(Ak, x[k], b[k]))
                    return out

                if form == "mixed":
                    # the fewest refinement steps whose every member meets the bound (untimed probe)
                    ds.execute("factorization")
                    for k in range(0, 9):
                        ds.setparam("ir_n_steps", k)
                        if max(member_errs(ds.execute("solve", None, bt).cpu().numpy())) <= BERR_TARGET:
                            break

                def step():
                    ds.execute("factorization")
                    ds.execute("solve", None, bt)

                ms = _time(torch, step, args.steps, args.warmup)
                x = ds.execute("solve", None, bt).cpu().numpy()
                errs = member_errs(x)
                line["forms"][form] = {"ms_per_step": round(ms, 3), "systems_per_s": round(256 / (ms / 1e3), 1),
                                       "max_bwd_err": float(max(errs)),
                                       "ir_steps": ds.getparam("ir_n_steps") if form == "mixed" else 0}
        line["speedup_mixed_vs_fp64"] = round(line["forms"]["fp64"]["ms_per_step"] /
                                              line["forms"]["mixed"]["ms_per_step"], 3)
    print(json.dumps(line), flush=True)


def profiled_traffic(form):
    """DRAM bytes per launch of the dataflow solve from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", f"dataflow_solve_{form}_lap3d48.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        return None
    return None


def workload(grid):
    from sdsb200 import matrices as M

    A = M.lap3d(grid, grid, grid)
    b = M.rhs(A.shape[0], NRHS, seed=0)
    return A, b


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        # the raw samples: SDSB200_CLOCKS_DIR when set, else the temporary directory
        base = os.environ.get("SDSB200_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(base, f"sdsb200_clocks_{os.getpid()}.csv")

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return self
        # the timed region is short (~0.1 s): start it only once nvidia-smi writes samples, and drop the
        # samples taken before it
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            self.fh.flush()
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.01)
        self.skip = sum(1 for _ in open(self.path))
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = list(open(self.path))
        # the samples from the timed region on (the last before it when none fell inside)
        for line in lines[max(0, getattr(self, "skip", 0) - 1):]:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_gemm_peak(torch, dtype, tf32=False):
    """Dense GEMM throughput of cuBLAS on this GPU (TFLOP/s), best of a few 8192^3 products. tf32: FP32
    operands on the tensor cores (TF32), the unit the 3xTF32 contribution-block updates run on."""
    n = 8192
    a = torch.randn(n, n, device="cuda", dtype=dtype)
    bm = torch.randn(n, n, device="cuda", dtype=dtype)
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = bool(tf32)
    for _ in range(2):
        torch.matmul(a, bm)
    best = 0.0
    for _ in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, bm)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) / 1e3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, bm
    torch.cuda.empty_cache()
    return best


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def run_reference(args, rank):
    """The reference's CPU path timed on the host cores, same workload, same metric."""
    if rank != 0:
        return
    from oracle.blas_port import CholeskyPort, blas_threads
    from sdsb200 import analyze_csr
    from sdsb200 import matrices as M

    A, b = workload(args.grid)
    S = analyze_csr(A, "SPD", reordering="nd")
    P = CholeskyPort(S)
    flops = S.flops + 4.0 * S.nnz_stored * NRHS
    times = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        P.factorize(A.data)
        x = P.solve(b)
        dt = time.perf_counter() - t0
        if it >= args.warmup:
            times.append(dt)
    cores = blas_threads()
    berr = M.scaled_backward_error(A, x, b)
    ms = 1e3 * statistics.mean(times)
    gflops = flops / (ms / 1e3) / 1e9
    out = {"impl": "reference", "metric": METRIC, "value": round(gflops, 4), "unit": "GFLOP/s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": f"lap3d_{args.grid} SPD Cholesky factor+solve, nested dissection, {NRHS} RHS",
                      "n": int(A.shape[0]), "nrhs": NRHS, "form": "fp64"},
           "bwd_err": berr,
           "cpu_baseline": {"value": round(gflops, 4), "unit": "GFLOP/s", "cores": cores, "kind": "port",
                            "sample": f"full workload, {args.steps} steps: the reference's CPU Cholesky path "
                                      "(ref_factorize! and its solve, src/reference/cholesky.jl) over threaded "
                                      f"LAPACK/BLAS, {cores} threads (the Julia reference cannot run here)"},
           "e2e": {"value": round(gflops, 4), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.once:
        run_once(args)
        return
    if args.config != "c2":
        run_config(args)
        return
    import torch

    from sdsb200 import capi
    from sdsb200 import matrices as M
    from sdsb200._native import numeric_lib
    from sdsb200.solver import DirectSolver

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist

        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    lib = numeric_lib()
    A, b = workload(args.grid)
    n = A.shape[0]
    forms = {
        # the refinement's step count is set below: the fewest steps that meet the metric's bound
        "mixed": dict(factor_precision="fp32", ir_n_steps=20, ir_tol=BERR_TARGET),
        "fp64": dict(factor_precision="fp64", ir_n_steps=0),
    }
    from sdsb200.autotune import autotune, describe

    solvers = {}
    tuned = {}
    Bt = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    for name, kw in forms.items():
        ds = DirectSolver(A, "SPD", reordering_alg="nd", max_nrhs=NRHS, amalgamation=amalgamation_of(args), **kw)
        if solvers:                      # one analysis for both forms
            ds.symbolic = next(iter(solvers.values())).symbolic
            ds._stage = 1
            ds.replan()
        else:
            t_an = time.perf_counter()
            ds.execute("analysis")
            analysis_s = time.perf_counter() - t_an
        # front tile shapes picked by the autotuner (outside the timed region, like the analysis)
        if args.tuning:
            from sdsb200.capi import tuning as make_tuning

            ds.setparam("tuning", make_tuning(*[int(v) for v in args.tuning.split(",")]))
            ds.replan()
            tuned[name] = describe(ds.params["tuning"])
        else:
            times = autotune(ds, Bt, reps=2, use_cache=False)
            tuned[name] = describe(min(times, key=times.get))
        solvers[name] = ds
    S = solvers["fp64"].symbolic
    # the metric's flops: the reference's default amalgamation (as the reference arm's), whatever the
    # solver's amalgamation (a wider one stores explicit zeros, whose flops are not counted)
    from sdsb200 import analyze_csr

    S0 = analyze_csr(A, "SPD", reordering="nd")
    flops = S0.flops + 4.0 * S0.nnz_stored * NRHS
    stream = torch.cuda.current_stream()
    st = C.c_void_p(stream.cuda_stream)
    Bd = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()        # column-major n x nrhs
    Xd = torch.empty_like(Bd)
    info = np.zeros(1, np.int64)

    def step(ds):
        o = ds._opts()
        rc = lib.sdsb200_factor(ds._plan, C.c_void_p(ds.nzval.data_ptr()), None, C.byref(o), info.ctypes.data, st)
        assert rc == 0, lib.sdsb200_last_error()
        launches = lib.sdsb200_plan_stat(ds._plan, b"launches_done")
        steps = C.c_int32(0)
        rc = lib.sdsb200_solve(ds._plan, C.c_void_p(Xd.data_ptr()), n, C.c_void_p(Bd.data_ptr()), n, NRHS,
                               C.c_void_p(ds.nzval.data_ptr()), C.byref(o), C.byref(steps), st)
        assert rc == 0, lib.sdsb200_last_error()
        launches += lib.sdsb200_plan_stat(ds._plan, b"launches_done")
        return int(steps.value), int(launches)

    # The mixed form refines a fixed number of steps: the fewest whose solution meets the metric's bound
    # (scaled backward error <= 1e-12), chosen untimed like the tile shapes. With ir_tol = 0 the steps run
    # without a host check of the residual norms after each; the timed solution's error is checked below.
    # The kernels' results do not depend on timing (atomics touch only counters), so the timed solution's
    # error is the probe's.
    mixed = solvers["mixed"]
    ir_probe = []
    for k in range(1, 21):
        mixed.setparam("ir_n_steps", k)
        mixed.setparam("ir_tol", 0.0)
        step(mixed)
        torch.cuda.synchronize()
        ir_probe.append(float(M.scaled_backward_error(A, Xd.t().cpu().numpy(), b)))
        if ir_probe[-1] <= BERR_TARGET:
            break

    results = {}
    for name, ds in solvers.items():
        for _ in range(args.warmup):
            step(ds)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        launches = 0
        irsteps = []
        with ClockSampler(local) as clk:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(args.steps):
                s_, l_ = step(ds)
                irsteps.append(s_)
                launches += l_
            e1.record()
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        if dist:
            ms = max_over_ranks(ms, dist, "cuda")
        x = Xd.t().cpu().numpy()
        berr = M.scaled_backward_error(A, x, b)
        results[name] = dict(ms=ms, gflops=world * flops / (ms / 1e3) / 1e9, berr=berr, ir_steps=irsteps[-1],
                             launches=launches, clocks=clk.summary(), x=x, info=int(info[0]))
    # the API's default refinement loop, timed beside the headline (not the metric's value): the mixed
    # form with a tolerance on max_k ||r_k|| / ||b_k|| (ir_tol = 1e-12, up to 20 steps), which reads the
    # residual norms back to the host after every step and stops at the first step that meets it
    tol_loop = None
    if not dist:
        mixed.setparam("ir_n_steps", 20)
        mixed.setparam("ir_tol", BERR_TARGET)
        for _ in range(args.warmup):
            step(mixed)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        tsteps = 0
        for _ in range(args.steps):
            tsteps = step(mixed)[0]
        e1.record()
        torch.cuda.synchronize()
        tol_loop = {"ms_per_step": round(e0.elapsed_time(e1) / args.steps, 3), "ir_steps": tsteps,
                    "ir_tol": BERR_TARGET, "bwd_err": float(M.scaled_backward_error(A, Xd.t().cpu().numpy(), b))}
        mixed.setparam("ir_n_steps", results["mixed"]["ir_steps"])
        mixed.setparam("ir_tol", 0.0)
    # error of the mixed solution against the FP64 one, per right-hand side
    xf, xm = results["fp64"]["x"], results["mixed"]["x"]
    err_vs_fp64 = [float(np.abs(xm[:, r] - xf[:, r]).max() / np.abs(xf[:, r]).max()) for r in range(NRHS)]

    # profiling pass (separate from the timed region): per-kind kernel time of one step
    prof = {}
    for name, ds in solvers.items():
        lib.sdsb200_set_profiling(ds._plan, 1)
        step(ds)
        torch.cuda.synchronize()
        kinds = {}
        for k in ("small", "assemble", "panel", "gemm", "pivot", "scale", "stats", "fwd", "bwd", "diag", "permute",
                  "residual", "inv"):
            ms_k = lib.sdsb200_plan_stat(ds._plan, f"prof_ms:{k}".encode())
            if ms_k > 0:
                kinds[k] = dict(ms=ms_k, flops=lib.sdsb200_plan_stat(ds._plan, f"prof_flops:{k}".encode()),
                                bytes=lib.sdsb200_plan_stat(ds._plan, f"prof_bytes:{k}".encode()),
                                launches=int(lib.sdsb200_plan_stat(ds._plan, f"prof_launches:{k}".encode())))
        lib.sdsb200_set_profiling(ds._plan, 0)
        prof[name] = kinds

    peaks, peak_kind = measured_peaks()
    fp64_peak = measured_gemm_peak(torch, torch.float64)
    fp32_peak = measured_gemm_peak(torch, torch.float32)
    tf32_peak = measured_gemm_peak(torch, torch.float32, tf32=True)
    head = "mixed"
    kinds = prof[head]

    def kind_roofline(dom):
        d = kinds[dom]
        per_launch_ms = d["ms"] / max(d["launches"], 1)
        if dom in ("gemm", "panel", "pivot"):
            if head != "mixed":
                peak, bound, src = fp64_peak, "fp64", "cuBLAS FP64 GEMM measured in this run (DMMA tensor path)"
            elif dom == "gemm":
                # the FP32 form's updates: 3xTF32 on tcgen05 (three tensor products per product) and the
                # steps' thin updates on the SIMT pipes; the tensor bound is a third of TF32
                peak, bound, src = tf32_peak / 3.0, "tf32x3", "cuBLAS TF32 GEMM measured in this run, / 3 (3xTF32)"
            else:
                peak, bound, src = fp32_peak, "fp32", "cuBLAS FP32 GEMM measured in this run (SIMT)"
            ach = d["flops"] / (d["ms"] / 1e3) / 1e12
            return {"kernel": dom, "bound": bound, "achieved": round(ach, 3),
                    "peak": round(peak, 3), "unit": "TFLOP/s", "frac": round(ach / peak, 4),
                    "peak_source": src,
                    "traffic": None, "launches": d["launches"], "ms_per_launch": round(per_launch_ms, 4)}
        peak = float(peaks.get("hbm_gbs", 6650.0))
        ach = d["bytes"] / (d["ms"] / 1e3) / 1e9
        traffic = profiled_traffic(head) if dom == "fwd" and args.grid == GRID else None
        return {"kernel": dom, "bound": "hbm", "achieved": round(ach, 2), "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4), "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_kind})",
                "traffic": traffic, "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, "
                f"profiles/dataflow_solve_{head}_lap3d48.md" if traffic else None,
                "algorithmic_bytes_per_launch": round(d["bytes"] / max(d["launches"], 1)),
                "launches": d["launches"], "ms_per_launch": round(per_launch_ms, 4)}

    # The dominant kernel: the factorization's kernels run on several streams at once (and the solve's
    # inverses on a side stream beside them), so their summed times overcount their share of the step;
    # the dataflow solve runs alone, one launch per solve. The kind whose launches run alone with the
    # largest time is the headline roofline; the dense update kernels get their own object.
    alone = [k for k in ("fwd", "residual") if k in kinds]
    dom = max(alone, key=lambda k: kinds[k]["ms"]) if alone else None
    roofline = kind_roofline(dom) if dom is not None else None
    roofline_dense = kind_roofline("gemm") if "gemm" in kinds else None

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        ds = solvers[head]
        nz_host = torch.from_numpy(np.ascontiguousarray(A.data)).pin_memory()
        b_host = torch.from_numpy(np.ascontiguousarray(b)).pin_memory()
        x_host = torch.empty_like(b_host).pin_memory()
        for _ in range(args.warmup):
            ds.nzval.copy_(nz_host, non_blocking=True)
            ds.execute("factorization")
            x_host.copy_(ds.execute("solve", None, b_host.cuda(non_blocking=True)), non_blocking=True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            ds.nzval.copy_(nz_host, non_blocking=True)
            ds.execute("factorization")
            x_host.copy_(ds.execute("solve", None, b_host.cuda(non_blocking=True)), non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        ms_e2e = e0.elapsed_time(e1) / args.steps
        if dist:
            ms_e2e = max_over_ranks(ms_e2e, dist, "cuda")
        berr_e2e = M.scaled_backward_error(A, x_host.numpy(), b)
        e2e = {"value": round(world * flops / (ms_e2e / 1e3) / 1e9, 3), "unit": "GFLOP/s",
               "ms_per_step": round(ms_e2e, 3), "h2d_bytes_per_step": int(8 * (A.nnz + n * NRHS)),
               "d2h_bytes_per_step": int(8 * n * NRHS), "bwd_err": berr_e2e}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle.blas_port import CholeskyPort, blas_threads

        P = CholeskyPort(S0)                     # the reference's CPU path on its default Symbolic
        P.factorize(A.data)                      # once untimed: pages in the fronts and the BLAS threads
        t0 = time.perf_counter()
        P.factorize(A.data)
        P.solve(b)
        dt = time.perf_counter() - t0
        cpu = {"value": round(flops / dt / 1e9, 4), "unit": "GFLOP/s", "cores": blas_threads(), "kind": "port",
               "sample": "one full factor+solve of the same workload on the host: the reference's CPU Cholesky "
                         "path (ref_factorize! and its solve) over threaded LAPACK/BLAS "
                         f"({dt:.2f} s)"}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    r = results[head]
    out = {
        "metric": METRIC, "value": round(r["gflops"], 3), "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(r["ms"], 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 factor + f64 refinement", "data": "synthetic",
        "config": {"workload": f"lap3d_{args.grid} SPD Cholesky factor+solve to bwd err <= 1e-12, nested dissection, "
                               f"{NRHS} RHS (form: mixed FP32 factor + FP64 IR)",
                   "n": int(n), "nnz": int(A.nnz), "nnz_stored": int(S.nnz_stored), "flops_per_step": flops,
                   "factor_flops": S0.flops, "amalgamation": list(amalgamation_of(args)),
                   "factor_flops_stored": S.flops, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (factor %.0f MB)" % (S.nnz_stored * 4 / 1e6)},
        "bwd_err": r["berr"], "ir_steps": r["ir_steps"], "ir_probe_bwd_err": ir_probe,
        "mixed_tolerance_loop": tol_loop,
        "err_vs_fp64_per_rhs": err_vs_fp64,
        "fp64": {"ms_per_step": round(results["fp64"]["ms"], 3), "value": round(results["fp64"]["gflops"], 3),
                 "bwd_err": results["fp64"]["berr"], "unit": "GFLOP/s",
                 "speedup_mixed_vs_fp64": round(results["fp64"]["ms"] / r["ms"], 3)},
        "tuning": tuned,
        "analysis_s": round(analysis_s, 3),
        "gpu_launches": int(r["launches"]),
        "clocks": r["clocks"],
        "roofline": roofline,
        "roofline_dense": roofline_dense,
        "kernel_profile": {k: {kk: {"ms": round(v["ms"], 4), "launches": v["launches"]} for kk, v in prof[k].items()}
                           for k in prof},
        "peaks": {"fp64_gemm_tflops_measured": round(fp64_peak, 2), "fp32_gemm_tflops_measured": round(fp32_peak, 2),
                  "tf32_gemm_tflops_measured": round(tf32_peak, 2),
                  "hbm_gbs": peaks.get("hbm_gbs"), "source": peak_kind},
        "cpu_baseline": cpu,
        "e2e": e2e,
    }
    ok = r["berr"] <= BERR_TARGET and results["fp64"]["berr"] <= BERR_TARGET
    out["valid"] = bool(ok)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()

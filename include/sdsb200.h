/*
 * sdsb200.h -- C ABI of the B200 (sm_100a) numeric phase: factorization,
 * refactorization and solve of a multifrontal sparse direct solver, as a
 * drop-in for SparseDirectSolver.jl's numeric and solve phases.
 *
 * Replaced reference interfaces (SparseDirectSolver.jl):
 *   sdsb200_plan_create   allocate_numeric src/numeric/storage.jl:205-256 and
 *                         allocate_solve src/solve/sweeps.jl:164-173, called from
 *                         _symbolic! src/solver.jl:641-642
 *   sdsb200_factor        _numeric_phase_cholesky!/ldlt!/lu! src/solver.jl:728-741,
 *                         i.e. factorize_cholesky! src/numeric/factorize.jl:327-360,
 *                         factorize_ldlt! src/numeric/ldlt.jl:1447-1475,
 *                         factorize_lu! src/numeric/lu.jl:543-555, with the info
 *                         read of _numeric_info! factorize.jl:383-415
 *   sdsb200_solve_phase   the solve sub-phases and Schur phases of _solve_phase!
 *                         src/solver.jl:847-900
 *   sdsb200_schur_matrix  schur_matrix! src/numeric/schur.jl:134-174 (Schur complement mode)
 *   sdsb200_solve         _solve_phase! src/solver.jl:810-871 (permute_rhs!,
 *                         forward_sweep!, diagonal_sweep!, backward_sweep!,
 *                         unpermute_solution!) and _refine_phase! :902-926 (refine!
 *                         src/solve/refinement.jl:359-397)
 *   sdsb200_get_*         the data-parameter outputs of getparam src/solver.jl:1090-1141
 *                         (info, inertia, npivots, pivot_stats, perm_row, diag) and
 *                         host_numeric src/numeric/extract.jl:13-21
 *   sdsb200_set_members   set_members! src/numeric/storage.jl:290-306 (ubatch_index)
 *   sdsb200_set_interrupt user_host_interrupt polling src/logging.jl:60-63
 *   sdsb200_plan_destroy  release of the Numeric / SolveWorkspace buffers
 *
 * Conventions: all Symbolic maps are HOST arrays, 1-based exactly as the
 * reference's `Symbolic` holds them (src/symbolic/maps.jl:62-95), of int32 or
 * int64 (`index_width`). Value arrays (nzval, B, X) are DEVICE pointers unless
 * the name starts with h_. Streams are cudaStream_t passed as void*.
 * The plan owns every device buffer; nzval/B/X are borrowed for the call.
 * Every call is asynchronous on `stream` except the documented host reads.
 */
#ifndef SDSB200_H
#define SDSB200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* return codes (mapped to the reference's errors, src/errors.jl:18-60) */
#define SDSB200_OK 0
#define SDSB200_INVALID_VALUE 1   /* InvalidValueError */
#define SDSB200_NOT_SUPPORTED 2   /* NotSupportedError */
#define SDSB200_PHASE_ORDER 3     /* FactorizationError (solve before factorization) */
#define SDSB200_INTERRUPTED 4     /* InterruptedError (user_host_interrupt) */
#define SDSB200_CUDA_ERROR 5
#define SDSB200_ALLOC_FAILED 6
#define SDSB200_TIMEOUT 7         /* a bounded device wait gave up */

/* structures (reference Structure enum): "G", "S", "SPD" */
#define SDSB200_STRUCTURE_G 0
#define SDSB200_STRUCTURE_S 1
#define SDSB200_STRUCTURE_SPD 3

/* factor precision of the plan */
#define SDSB200_PRECISION_FP64 0  /* the plain form: every operation in FP64 */
#define SDSB200_PRECISION_FP32 1  /* FP32 factor, assembly and Schur updates; FP64 residual + refinement */

/* The reference's Symbolic maps (DEVICE_MAPS, src/symbolic/maps.jl:16-18) as host arrays.
 * Arrays are int32_t* when index_width == 4, int64_t* when 8. */
typedef struct sdsb200_symbolic {
    int64_t n, nnz, ns;
    int32_t index_width;      /* 4 or 8 */
    int32_t structure;        /* SDSB200_STRUCTURE_* */
    const void* perm;         /* n: column k of the factor is original column perm[k] */
    const void* super_ptr;    /* ns + 1 */
    const void* snparent;     /* ns (0 = root) */
    const void* rowptr;       /* ns + 1: solve gather lists */
    const void* rowval;
    const void* front_ptr;    /* ns + 1: panel_ptr of the Layout */
    const void* child_ptr;    /* ns + 1 */
    const void* child_list;
    const void* relind_ptr;   /* ns + 1 */
    const void* relind;
    const void* amap;         /* nnz (signed: negative = conjugate / U^T structure, 0 = ignored) */
    const void* amap_ptr;     /* ns + 1 */
    const void* amap_src;
    /* residual map of the full matrix M (FullPatternMap, src/symbolic/pattern.jl:215-290); NULL disables
     * iterative refinement. full_rowptr: n + 1; full_colval / full_srcptr: nnz(M) (+1); full_src. */
    const void* full_rowptr;
    const void* full_colval;
    const void* full_srcptr;
    const void* full_src;
    int64_t full_nnz;         /* entries of M */
    int64_t full_nsrc;        /* length of full_src */
    /* Schur complement mode (schedule.schur, src/symbolic/schedule.jl:194-227,351-360): the root
     * supernode (1-based) that the factorization assembles and does not factor; 0 = none. It must be
     * a root with no rows below its columns; its columns are the Schur indices. */
    int64_t schur;
} sdsb200_symbolic;

typedef struct sdsb200_plan_options {
    int32_t nbatch;           /* uniform batch members (ubatch_size); 1 for a single matrix */
    int32_t precision;        /* SDSB200_PRECISION_* */
    int32_t max_nrhs;         /* largest nrhs of a solve (workspace) */
    int32_t tuning;           /* front tile shapes, 0 = defaults; SDSB200_TUNING(fsmall, wide) */
} sdsb200_plan_options;

/* Plan tuning (the shapes an autotuner chooses; no counterpart in the reference):
 * fsmall = the largest front order handled by the shared-memory small-front kernel (one of 32, 64,
 * 96, 128, 160, and 224 for FP32; 0 = the largest class); wide = the tallest front (at most 32
 * columns) that the dataflow solve gives to one warp, larger fronts going to tile tasks (16..128,
 * 0 = 128); chains = how the dataflow solve treats those tiled fronts: 0, through their inverse
 * panels [L11^-1; L21 L11^-1] (f x w each, built after every factorization of a single-system plan),
 * 1: through chains of 64-column blocks; streams = the factorization streams of a single-system
 * Cholesky plan (independent subtrees factored concurrently; 0 = 4, 1 = level by level, up to 15);
 * steps (bit 5 of the third field, SDSB200_TUNING_STEPS): 1 = a single-system Cholesky plan runs each
 * batch of its large fronts' 32-column steps as dataflow tasks in one persistent launch, 0 (default) =
 * one launch per step and kernel; subtree (bits 26-29, SDSB200_TUNING_SUBTREE): the fused subtrees
 * (the reference's regime A: maximal subtrees of shared-memory fronts, each factored by one CTA in
 * one launch per size class) hold up to 2^subtree fronts (1..14), or are off (0, the default, and 15).
 * Bits 30 and 31 must be zero. */
#define SDSB200_TUNING(fsmall, wide, chains) \
    ((int32_t)(fsmall) | ((int32_t)(wide) << 9) | ((int32_t)(chains) << 20))
#define SDSB200_TUNING_STREAMS(fsmall, wide, chains, streams) \
    (SDSB200_TUNING(fsmall, wide, chains) | ((int32_t)(streams) << 21))
#define SDSB200_TUNING_STEPS ((int32_t)1 << 25)
#define SDSB200_TUNING_SUBTREE(subtree) ((int32_t)(subtree) << 26)

/* The Options fields the numeric and solve phases read (src/options.jl:155-223). */
typedef struct sdsb200_opts {
    int32_t pivot_type;        /* PivotType: 0 auto, 1 none, 4 diagonal, 5 local block, 6 Bunch-Kaufman */
    int32_t pivot_epsilon_alg; /* 0 default/algo2 (static), 1 algo1 (scaled by max|a_ij|) */
    double pivot_threshold;    /* 0.01 */
    double pivot_epsilon;      /* < 0: default_pivot_epsilon (1e-13 FP64, 1e-5 FP32) */
    int32_t ir_n_steps;        /* iterative refinement steps (0: none) */
    int32_t ir_mode;           /* 0 plain */
    double ir_tol;             /* > 0: stop when max_k ||r_k|| / ||b_k|| <= ir_tol (one host read per step) */
    int32_t solve_mode;        /* 0 A, 1 A^T, 2 A^H (= A^T for real) */
    int32_t deterministic_mode;/* the solve is always deterministic (owner-pull); accepted for parity */
} sdsb200_opts;

typedef struct sdsb200_plan sdsb200_plan;

void sdsb200_default_opts(sdsb200_opts* o);

/* Build the plan: copy the maps to the device, derive the level schedule and
 * the extend-add maps, allocate every buffer of the numeric and solve phases
 * (the only allocations). Synchronous. */
int sdsb200_plan_create(sdsb200_plan** plan, const sdsb200_symbolic* sym, const sdsb200_plan_options* popts,
                        void* stream);
int sdsb200_plan_destroy(sdsb200_plan* plan);

/* Factorize (or refactorize: same call) the values nzval (device, nnz * nbatch, member-major).
 * h_psign: pivot_sign (n int8 on the host, indexed by original row) or NULL.
 * h_info (nbatch, may be NULL): original column (1-based) of the first failed pivot per member,
 * 0 = success; written at the phase's one host synchronization. */
int sdsb200_factor(sdsb200_plan* plan, const double* nzval, const int8_t* h_psign, const sdsb200_opts* opts,
                   int64_t* h_info, void* stream);

/* Solve op(A) X = B for nrhs right-hand sides per member (device, column-major, leading dimension
 * ldb/ldx >= n, members one after the other at stride ld * nrhs). X == B is allowed without refinement.
 * nzval (device) is needed when opts->ir_n_steps > 0. h_ir_steps (may be NULL): refinement steps run. */
int sdsb200_solve(sdsb200_plan* plan, double* X, int64_t ldx, const double* B, int64_t ldb, int32_t nrhs,
                  const double* nzval, const sdsb200_opts* opts, int32_t* h_ir_steps, void* stream);

/* Solve sub-phases (execute! "solve_fwd_perm", "solve_fwd", "solve_diag", "solve_bwd", "solve_bwd_perm"
 * of _solve_phase! src/solver.jl:847-867, and the steps of the Schur phases :876-900): one step of the
 * solve on the plan's working vectors Y (n x nrhs per active member, factor order, kept in the plan
 * between calls; between the forward and backward sweeps each supernode's slice is in its local pivot
 * order, as the reference's ws.Y). No refinement. op(A) as opts->solve_mode; the diagonal step is the
 * identity for "SPD". X and B (device, column-major, ld >= n, members at stride ld * nrhs) are read
 * or written only by the phases that name them. A Schur plan's forward sweep leaves the condensed
 * right-hand side b2 - A21 A11^{-1} b1 in the Schur rows of Y, and its backward sweep takes the Schur
 * solution from there. */
#define SDSB200_PHASE_FWD_PERM 1  /* Y = B[perm]                permute_rhs!        src/solve/permute.jl:117-131 */
#define SDSB200_PHASE_FWD 2       /* Y <- L^{-1} Y              forward_sweep!      src/solve/sweeps.jl:908-942 */
#define SDSB200_PHASE_DIAG 3      /* Y <- D^{-1} Y              diagonal_sweep!     src/solve/sweeps.jl:955-969 */
#define SDSB200_PHASE_BWD 4       /* Y <- L^{-T} Y (LU: U^{-1}) backward_sweep!     src/solve/sweeps.jl:984-1004 */
#define SDSB200_PHASE_BWD_PERM 5  /* X[perm] = Y                unpermute_solution! src/solve/permute.jl:138-149 */
#define SDSB200_PHASE_LOAD 6      /* Y = B, no permutation (the Schur phases' identity permute_rhs!) */
#define SDSB200_PHASE_STORE 7     /* X = Y, no permutation (the Schur phases' identity unpermute_solution!) */
int sdsb200_solve_phase(sdsb200_plan* plan, int32_t phase, double* X, int64_t ldx, const double* B, int64_t ldb,
                        int32_t nrhs, const sdsb200_opts* opts, void* stream);

/* Schur complement mode: S = A22 - A21 A11^{-1} A12 as assembled by the last factorization
 * (schur_matrix!, src/numeric/schur.jl:134-174), written to the dense column-major DEVICE matrix D
 * (ns x ns, ld ldd >= ns; ns = sdsb200_plan_stat "schur_n") in the increasing original order of the
 * Schur indices; transposed != 0 writes S^T (the reference's transposed = true for a CSC input).
 * "G": the lower triangle from L's panel, the strict upper one from the U^T panel; "S" and "SPD": the
 * lower triangle mirrored. */
int sdsb200_schur_matrix(sdsb200_plan* plan, int32_t member, double* D, int64_t ldd, int32_t transposed,
                         void* stream);

/* residual! (src/solve/refinement.jl:229-248): R = B - op(A) X over the full pattern with the values
 * nzval, for the active members (R: n x nrhs per member, ld n, members at stride n * nrhs; X, B as in
 * sdsb200_solve). solve_mode 1 or 2 with "G": op(A) = A^T. Used by FGMRES-IR for its residual and
 * its matrix-vector products (B = 0 gives R = -op(A) X). */
int sdsb200_residual(sdsb200_plan* plan, double* R, const double* X, int64_t ldx, const double* B, int64_t ldb,
                     int32_t nrhs, const double* nzval, int32_t solve_mode, void* stream);

/* Outputs (synchronous host copies; member = 0-based batch member). */
int sdsb200_get_stats(sdsb200_plan* plan, int32_t member, int64_t* h_stats /* 6 * ns */,
                      int64_t* h_totals /* 6 */);
int sdsb200_get_pivots(sdsb200_plan* plan, int32_t member, int32_t* h_piv /* n, 1-based */,
                       int8_t* h_kind /* n */, double* h_d /* 2n */);
/* factor panels of one member as FP64 (factor_len each; h_ufactor: "G" only, may be NULL) */
int sdsb200_get_factor(sdsb200_plan* plan, int32_t member, double* h_factor, double* h_ufactor);

/* ubatch_index / ubatch_mask: restrict later calls to h_members (0-based), nact of them; nact < 0 = all. */
int sdsb200_set_members(sdsb200_plan* plan, const int32_t* h_members, int32_t nact);

/* user_host_interrupt: a host flag polled between launch groups (factorization) and refinement steps. */
int sdsb200_set_interrupt(sdsb200_plan* plan, const volatile int32_t* h_flag);

/* CUDA graphs (on by default): the launch program of sdsb200_factor and of the solve / refinement
 * steps is captured once per set of buffers and options and replayed. The user_host_interrupt flag is
 * then polled before a factorization and before each refinement step, not between launch groups. */
int sdsb200_set_graphs(sdsb200_plan* plan, int32_t on);

/* Solve engine. Nonzero (default): the dataflow solve, one cooperative persistent launch per group of
 * 8 right-hand sides with no grid barrier (tasks in a topological order of the elimination tree,
 * synchronised by per-front counters and per-block flags; a uniform batch runs every active member's
 * tasks in the same launch); 0: one launch per level and sweep (the engine of the solve sub-phases). */
int sdsb200_set_persistent(sdsb200_plan* plan, int32_t on);

/* Profiling mode (on != 0): CUDA events around every launch of the following factor and solve
 * calls, accumulated per kernel kind (resets the totals). Costs one event record per launch. */
int sdsb200_set_profiling(sdsb200_plan* plan, int32_t on);

/* Profiling: the dataflow solve's task trace of its last launch made while profiling was on, 6 int64
 * per task for up to cap tasks (task start, end of its dependency wait and task end in ns of
 * %globaltimer; CTA; task kind; a | b << 32 of the task record). With cap < 0: the factorization's
 * Cholesky step tasks of its last profiled call, 4 int64 per task (start, end of its first waits, end;
 * CTA | kind << 12 | step << 16 | update block << 28 | front << 40) for up to -cap tasks in the plan's
 * task order. Returns the tasks copied or -1. */
int64_t sdsb200_get_trace(sdsb200_plan* plan, int64_t* h_out, int64_t cap);

/* Plan facts: "ns", "nlevels", "factor_len", "cb_len", "launches_factor", "launches_solve",
 * "launches_done" (kernel launches of the last factor or solve call), "device_bytes", "flops",
 * "schur_n" (order of the Schur complement, 0 without one), "schur_level", "subtrees" and
 * "subtree_fronts" (the fused subtrees and the fronts in them),
 * "solve_status" (synchronizes; nonzero when a bounded wait of the persistent solve gave up);
 * with profiling, "prof_ms:<kind>", "prof_flops:<kind>", "prof_bytes:<kind>", "prof_launches:<kind>"
 * for kinds small assemble panel gemm pivot scale stats fwd bwd diag permute residual inv, and per
 * launch of the last calls "prof_records" (their count), "prof_record:<i>:kind|level|ms|start|flops"
 * (start: ms after the call's first launch began; kind: the index of the kind in that list; flops: the
 * launch's algorithmic flops).
 * Returns -1 for an unknown name. */
double sdsb200_plan_stat(const sdsb200_plan* plan, const char* name);

/* Adjoint of x = op(A)^{-1} B with respect to the values (no counterpart in the reference, which has no
 * automatic differentiation): the sampled outer product over the CSR pattern,
 *   out[k] = alpha * sum_r U[i, r] V[j, r]                     structure "G" (0), every entry k = (i, j);
 *   out[k] = alpha * sum_r (U[i, r] V[j, r] + U[j, r] V[i, r])   "S" (1) / "SPD" (3), i != j, kept entry;
 *   out[k] = alpha * sum_r U[i, r] V[i, r]                     "S" / "SPD", kept diagonal entry;
 *   out[k] = 0                                                 "S" / "SPD", an entry the view drops.
 * Kept entries are those the factorization reads: the lower triangle for view 'F' and 'L', the upper
 * for 'U'. With U = A^{-T} X_bar (a transposed solve, solve_mode 1) and V = X, alpha = -1 gives
 * dLoss/d nzval. rowptr (n + 1) and colval (nnz) are DEVICE arrays of int32 (index_width 4) or int64
 * (8) with index_base 0 or 1; U, V (ld >= n, ncols columns) and out (nnz) are device arrays, nbatch
 * members one after the other (strides ldu * ncols, ldv * ncols, nnz). */
int sdsb200_sampled_outer(int64_t n, int64_t nnz, const void* rowptr, const void* colval, int32_t index_width,
                          int32_t index_base, int32_t structure, int32_t view, const double* U, int64_t ldu,
                          const double* V, int64_t ldv, int32_t ncols, int32_t nbatch, double alpha, double* out,
                          void* stream);

/* Solve without allocating (no counterpart in the reference): op(A) X = B for one active batch member,
 * no refinement, as two small memsets (the status word; the plan's flag and counter buffer, which is
 * plan memory allocated at plan creation and shared by every solve on the plan) and one cooperative
 * kernel launch per group of 8 right-hand sides. On a plan with an FP32 factor it returns the
 * unrefined solution through that factor (FP32 accuracy); refine it with sdsb200_residual and further
 * calls when FP64 accuracy is needed. sdsb200_solve keeps its
 * working vectors in the plan and records its launches into a CUDA graph per set of buffers, and
 * building that graph makes the driver allocate device memory on the first call with new buffers.
 * Callers that may not allocate once set-up is over (a framework whose pool allocator owns all device
 * memory, a real-time loop that forbids allocation after start-up) call this entry point instead:
 * the working vectors Y and xtmp (n * nrhs doubles each) and the update vectors (the plan's ulen
 * doubles) live in one static device array of SDSB200_NOALLOC_SCRATCH_BYTES (32 MiB), which every
 * GPU that loads the library holds until the process exits. Sizes beyond it are rejected with
 * SDSB200_INVALID_VALUE: 512 + 8 * (2 * n * nrhs + ulen) bytes must fit, ulen being the plan's
 * update-vector length (the sum over fronts of the rows below the pivot block, times max_nrhs); the
 * error message gives the bytes needed. The first call on a device looks up the array's device address (which may also load the
 * library's device code) and keeps it for the life of the process, so make one call during set-up,
 * before any stream capture; a device reset (cudaDeviceReset) after that first call is not supported. The array is
 * shared by every call on that device and keeps the last call's contents; calls that overlap on the
 * GPU (other streams, other plans, other threads) race on it and must be serialised by the caller.
 * solve_mode as sdsb200_opts (1, 2: A^T for "G"). status (device int32, may be NULL): set to 0, then
 * nonzero if a bounded wait of the launch gave up (X is then not the solution). With status NULL the
 * call reads a status word of its own back at the end, which waits for the stream, and returns
 * SDSB200_TIMEOUT if a wait gave up. */
#define SDSB200_NOALLOC_SCRATCH_BYTES (32ull << 20)
int sdsb200_solve_noalloc(sdsb200_plan* plan, double* X, int64_t ldx, const double* B, int64_t ldb, int32_t nrhs,
                          int32_t solve_mode, int32_t* status, void* stream);

const char* sdsb200_last_error(void);

#ifdef __cplusplus
}
#endif
#endif

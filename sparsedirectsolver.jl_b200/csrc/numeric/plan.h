// The plan of the numeric phase: device copies of the Symbolic maps, the level
// schedule, the launch program of the factorization and every buffer of the
// numeric and solve phases (the only allocations; the phases allocate nothing).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "solve.cuh"

namespace sds {

enum BufId : int32_t { BUF_FACTOR = 0, BUF_UFACTOR, BUF_CB, BUF_WORK, BUF_INV };

struct ProgLaunch {
    LaunchKind kind;
    int32_t level;
    int32_t count;
    int32_t cls;       // small: max rows of the class; panel: kb; pivot: -; gemm: -
    int64_t list;      // offset into the list array of the kind
    int32_t nb;        // panel block width
    int32_t maxw;      // scale: widest front
    BufId abuf, bbuf, cbuf;
    double flops;      // algorithmic flops of the launch (reference convention for the fronts)
    double bytes;      // algorithmic device-memory bytes of the launch
    int32_t coop = -1;      // pivot: offset of the group prefix in coop_first (-1: one CTA per front)
    int32_t coop_grid = 0;  // pivot: CTAs of the cooperative launch
    int32_t exact = 0;      // gemm: the contribution-block update of an LDLT / LU front, which the FP64
                            // form sums in the oracle's order (1: LDLT, 2: LU)
    int32_t side = 0;       // runs on the plan's side stream (the solve's inverses, off the factorization's
                            // critical path), after the main stream's launches that precede it
    int64_t list2 = 0;      // inverses: first (front, block) pair of the block inverses; count2 pairs
    int32_t count2 = 0;
    int32_t fstream = 0;    // factorization stream (0: the caller's)
    int32_t wait_begin = 0, wait_count = 0;   // events (in fwaits) this launch's stream waits for first
    int32_t record = -1;    // event recorded on the launch's stream after it (-1: none)
};

// per-kind accounting of the profiling mode (CUDA events around every launch)
enum ProfKind { PK_SMALL = 0, PK_ASSEMBLE, PK_PANEL, PK_GEMM, PK_PIVOT, PK_SCALE, PK_STATS, PK_FWD, PK_BWD, PK_DIAG,
                PK_PERMUTE, PK_RESIDUAL, PK_INV, PK_COUNT };

struct ProfAcc {
    double ms = 0, flops = 0, bytes = 0;
    int64_t launches = 0;
};

struct Plan {
    int64_t n = 0, nnz = 0, ns = 0;
    int structure = 0, nbatch = 1, precision = 0, elsize = 8, max_nrhs = 1;
    int64_t factor_len = 0, cb_len = 0, ulen = 0, scr_len = 0, work_len = 0, inv_len = 0;
    int nlevels = 0;
    int fsmall_max = 0;
    // Schur complement mode: the root front that is assembled but not factored (-1: none), alone on
    // the last level
    int schur_front = -1, schur_level = -1;
    std::vector<DFront> fronts;
    std::vector<std::vector<int>> level_fronts;
    std::vector<int> level_maxw;
    std::vector<double> level_panel_entries;   // stored lower-trapezoid entries of the panels of each level
    std::vector<int32_t> h_perm0, h_super0;
    double flops = 0;

    DeviceMaps maps{};
    DFront* d_fronts = nullptr;
    int32_t* d_super0 = nullptr;
    int32_t* d_perm0 = nullptr;

    void* d_factor = nullptr;
    void* d_ufactor = nullptr;
    void* d_cb = nullptr;
    double* d_d = nullptr;
    int32_t* d_piv = nullptr;
    int8_t* d_kind = nullptr;
    int64_t* d_stats = nullptr;
    int32_t* d_finfo = nullptr;
    int64_t* d_totals = nullptr;
    int64_t* d_info = nullptr;
    int8_t* d_psign = nullptr;
    int32_t* d_members = nullptr;
    double* d_scratch = nullptr;
    void* d_work = nullptr;
    void* d_inv = nullptr;          // inverses of the diagonal blocks of large Cholesky fronts
    double* d_amax = nullptr;

    std::vector<ProgLaunch> prog;
    int32_t* d_lists = nullptr;
    ColTask* d_coltasks = nullptr;
    GemmTile* d_tiles = nullptr;
    int64_t* d_scr_off = nullptr;
    CholStepTask* d_steptasks = nullptr; // tasks of the large-Cholesky step launches
    int32_t* d_coop_first = nullptr;   // group prefixes of the cooperative pivot launches
    unsigned int* d_coop_bar = nullptr; // their group barrier counters
    int32_t coop_bar_len = 0;
    int64_t* d_woff = nullptr;
    int64_t* d_uoff = nullptr;
    int32_t* d_level_lists = nullptr;   // fronts of each level for the solve sweeps: small first, then large
    std::vector<int64_t> level_list_off;
    std::vector<int> level_nsmall, level_nlarge, level_maxw_small, level_maxw_large;
    // dataflow solve (solve.cuh): per-front classes, the task list, the inverses of every front's diagonal
    // blocks (warp fronts: w x w; tiled fronts: 64 x 64 blocks), flags and counters zeroed per launch
    DfFront* d_df = nullptr;
    DfTask* d_df_tasks = nullptr;
    int32_t n_df_tasks = 0;
    int32_t* d_df_bundles = nullptr;
    int64_t* d_df_inv_off = nullptr;    // per front: offset of its inverses
    int64_t df_inv_len = 0;
    void* d_dfinv_L = nullptr;          // inverses of the factor's (L) diagonal blocks
    void* d_dfinv_U = nullptr;          // ... of the U^T panels (LU)
    int32_t* d_df_small = nullptr;      // warp fronts (the small-inverse launch)
    int32_t n_df_small = 0;
    int32_t* d_df_blkinv = nullptr;     // (front, block) pairs of the tiled fronts' 64 x 64 inverses
    int32_t n_df_blkinv = 0;
    int32_t* d_df_rptr = nullptr;       // per front row: start of its contributions (f + 1 per front)
    int32_t* d_df_csrc = nullptr;       // contributions: the children's global update rows, in child order
    unsigned int* d_df_flags = nullptr; // fcnt (ns), bdone (ns), xflag (nblk), pcnt (nblk), head
    int64_t df_flags_len = 0;            // per member (the task counter follows every member's flags)
    int64_t df_part_len = 0;             // partial-product doubles per member
    int32_t df_nblk = 0;
    int32_t df_ntcnt = 0, df_nccnt = 0;  // inverse panels: forward row-tile and backward column-block counters
    bool df_pinv = false;               // tiled fronts solved through their inverse panels
    PinvTile* d_pinv_tiles = nullptr;   // the GEMM tiles that build the inverse panels (kind L_PINV)
    int64_t pwork_len = 0;              // their scratch (T = L[C, A] X[A, A] of one doubling level), per member and side
    void* d_pwork = nullptr;
    FlowTask* d_flow_tasks = nullptr;   // the Cholesky steps' dataflow tasks (kind L_CHOL_FLOW)
    int64_t n_flow_tasks = 0;
    unsigned int* d_flow_cnt = nullptr; // their counters: per launch count2 + 1 at list2, zeroed per launch
    int64_t flow_cnt_len = 0;
    int32_t* d_flow_status = nullptr;   // nonzero: a bounded wait of the step tasks gave up
    int64_t* d_flow_trace = nullptr;    // profiling: 4 int64 per step task
    int64_t psplit_slots = 0, psplit_cnts = 0;   // split tiles: most partial slots and counters of a launch
    void* d_psplit = nullptr;           // their 64 x 64 partial products
    unsigned int* d_pcnt = nullptr;     // their arrival counters (reset by the last arrival)
    double* d_df_part = nullptr;        // backward partial sums: slots of 64 x DF_MAX_NRHS doubles
    int64_t* d_df_trace = nullptr;      // profiling: 6 int64 per task (start, wait done, end, CTA, kind, a | b << 32)
    int32_t df_fwarp_max = 1;           // tallest warp front
    double* d_xtmp = nullptr;
    int32_t* d_solve_status = nullptr;
    int32_t* d_rect_tiles = nullptr;    // (front, start) pairs: forward row tiles, backward column tiles
    std::vector<int64_t> level_ftile_off, level_btile_off;
    std::vector<int> level_nftile, level_nbtile;

    double* d_Y = nullptr;
    double* d_U = nullptr;
    double* d_R = nullptr;
    double* d_norms = nullptr;
    double* h_norms = nullptr;
    int64_t* h_info_pinned = nullptr;
    bool has_full = false;
    int64_t full_nnz = 0, full_nsrc = 0;
    int64_t *d_full_rowptr = nullptr, *d_full_colval = nullptr, *d_full_srcptr = nullptr, *d_full_src = nullptr;
    int64_t *d_fullT_rowptr = nullptr, *d_fullT_colval = nullptr, *d_fullT_srcptr = nullptr, *d_fullT_src = nullptr;

    bool factored = false;
    int nact = 1;
    bool all_members = true;
    const volatile int32_t* interrupt = nullptr;
    std::vector<void*> allocations;
    int64_t device_bytes = 0;
    int launches_factor = 0;
    int launches_solve = 0;
    int64_t launches_done = 0;   // kernel launches issued by the last factor / solve calls

    // CUDA graphs: the static launch program captured once per key (buffers, options) and replayed
    struct CachedGraph {
        std::vector<uint64_t> key;
        cudaGraphExec_t exec = nullptr;
        int64_t launches = 0;
    };
    bool use_graphs = true;
    bool persistent = true;        // the one-launch dataflow solve (every active member in one launch)
    cudaStream_t own = nullptr;          // capture / replay stream, joined to the caller's by events
    cudaEvent_t join_in = nullptr, join_out = nullptr;
    cudaStream_t side = nullptr;         // low-priority stream of the side launches of the factorization
    cudaEvent_t side_fork = nullptr, side_join = nullptr;
    int nfstreams = 1;                   // factorization streams (stream 0 is the caller's / capture stream)
    int64_t nsubtrees = 0, nsubtree_fronts = 0;   // fused subtrees and the fronts in them
    std::vector<cudaStream_t> fstreams;  // streams 1 .. nfstreams - 1
    std::vector<cudaEvent_t> fevents;    // the cross-stream events of the factorization
    int nfevents = 0;
    std::vector<int32_t> fwaits;         // per launch wait lists (ProgLaunch::wait_begin / wait_count)
    cudaEvent_t fstream_fork = nullptr;  // the extra streams start after the caller's prior work
    CachedGraph g_factor, g_solve, g_resid, g_corr;

    bool profile = false;
    ProfAcc prof[PK_COUNT];
    std::vector<cudaEvent_t> events;
    size_t prof_next = 0;
    std::vector<std::pair<int, std::pair<double, double>>> pending;  // kind, (flops, bytes) per event pair
    std::vector<int> pending_level;
    struct LaunchRecord { int kind, level; double ms, start, flops; };
    std::vector<LaunchRecord> records;   // every profiled launch of the last calls
    int cur_level = -1;
};

struct PlanError {
    int code;
    std::string msg;
};

Plan* build_plan(const sdsb200_symbolic* sym, const sdsb200_plan_options* popts, cudaStream_t stream);
void free_plan(Plan* p);

}  // namespace sds

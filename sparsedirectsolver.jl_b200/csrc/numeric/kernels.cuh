// Kernel argument blocks and launch functions of the numeric phase.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace sds {

template <typename T>
struct SmallArgs {
    DeviceMaps maps;
    int32_t count;           // fronts of the launch (the warp-per-front kernel)
    const int32_t* list;     // fronts of this launch
    const int32_t* sub_ptr;  // fused subtrees: subtree b is list[sub_ptr[b] .. sub_ptr[b + 1]) (NULL: one
                             // front per CTA)
    const int32_t* members;  // active batch members (NULL: 0..nmembers-1)
    const double* nzval;
    T* factor;
    T* ufactor;
    T* cb;
    double* d;
    int32_t* piv;
    int8_t* kind;
    int64_t* stats;
    int32_t* finfo;
    const int8_t* psign;
    int64_t nnz, factor_len, cb_len, n;
    int32_t ns;
    int32_t pivot;
    int32_t lu_pivot;
    double u, eps;
};

template <typename T>
struct LargeAsmArgs {
    DeviceMaps maps;
    const ColTask* tasks;
    int32_t count;
    const int32_t* members;
    const double* nzval;
    T* factor;
    T* ufactor;
    T* cb;
    int64_t nnz, factor_len, cb_len;
};

struct StatsArgs {
    const int64_t* stats;
    const int32_t* members;
    const int32_t* super_ptr0;  // 0-based first column of each front
    const int32_t* perm0;       // 0-based original column of each factor column
    int64_t* totals;            // 6 per member
    int64_t* info;              // 1 per member (original column, 1-based; 0 = success)
    int32_t ns;
};

// Large Cholesky column-block panel: diagonal block + trsm of the rows below.


// Diagonal block of a large Cholesky front: factor in place and write its inverse (ld 64) to scratch.

// One task of a large-Cholesky step: a 64-row tile of the rows below the diagonal block of front
// `front` (tile >= 0), or the diagonal block alone when no rows are below it (tile = -1). The task
// with tile <= 0 is the step's head: it records the statistics and puts L11 at `scr` of the scratch
// buffer (or, for a diagonal block with nothing below, directly into the panel).
struct CholStepTask {
    int32_t front;
    int32_t tile;
    int64_t scr;
    int64_t panel;     // the front's panel offset, order and width (no dependent load of the front
    int32_t f, w;      // record before the block loads)
};

// The 32-column steps of a batch of large Cholesky fronts as dataflow in one persistent launch
// (single-system plans). Tasks, in list order:
//  * STEP: the step's diagonal block (factored by every task of the step, as chol_step_kernel does) and
//    one 64-row tile of the rows below, forward-substituted; for the front's last step;
//  * STEPN: the same, then the step's update of the next column block on the tile's rows, so that the
//    chain of a front's steps is one task per step. After its substitution it signals sig_mid (its rows
//    are in the panel; tile 0 also sig_head) and then waits for tile 0 (w_mid: the next block's rows
//    are tile 0's first rows) and for the block's earlier updates (w2 >= v2);
//  * COPY: the step's L11 from its scratch slot into the panel, once every task of the step is done;
//  * UPD: the step's rank-32 update of one (64-row tile, 32-column block) of the front's trailing
//    columns beyond the next block: C -= X_k[rows] X_k[block rows]^T, lower part only.
// A task waits on counters (>= a target) and signals counters (increments, or a release store of a
// value). Every wait is on tasks earlier in the list, so CTAs that take tasks in order from one counter
// always progress; the updates of the following blocks come after the next step's tasks (lookahead).
enum FlowKind : int32_t { FLOW_STEP = 1, FLOW_COPY = 2, FLOW_UPD = 3, FLOW_STEPN = 4 };
struct FlowTask {
    int32_t kind, front;
    int32_t kb;              // the step's first column
    int32_t a, b;            // STEP/STEPN: row tile (-1: no rows below the block); UPD: the block's first
                             // column, the tile's first row
    int32_t w1, v1, w2, v2;  // waits: counter w >= v (w < 0: none); STEPN waits for w2 after its substitution
    int32_t sig_add;         // counter incremented when done (-1: none)
    int32_t sig_store, sig_val;   // counter set to sig_val when done (-1: none)
    int32_t sig_mid;         // STEPN: counter incremented once the tile's rows are in the panel (-1: none);
    int32_t sig_head;        // tile 0 also increments this one (-1: none)
    int32_t w_mid;           // STEPN tiles > 0 then wait for it (>= 1; -1: none)
    int32_t f, w;
    int64_t panel;           // the front's panel offset
    int64_t scr;             // the step's L11 scratch slot
};
template <typename T>
struct CholFlowArgs {
    const FlowTask* tasks;
    int32_t ntasks;
    T* factor;
    T* scratch;
    int32_t* finfo;
    int64_t* stats;
    double eps;
    unsigned int* cnt;       // the batch's counters, zero at launch; cnt[ncnt] is the task counter
    int32_t ncnt;
    int32_t* status;         // nonzero: a bounded wait gave up
    int64_t* trace;          // profiling, or NULL: per task (start, wait done, end) %globaltimer ns, and
                             // CTA | kind << 12 | step << 16 | update block << 28 | front << 40
};
template <typename T>
cudaError_t launch_chol_flow(const CholFlowArgs<T>& a, cudaStream_t st);

template <typename T>
struct CholStepArgs {
    const DFront* fronts;
    const CholStepTask* tasks;
    int32_t count;
    const int32_t* members;
    T* factor;
    T* scratch;               // L11 of the step heads, per member stride scr_len
    int64_t scr_len;
    int32_t* finfo;
    int64_t* stats;
    int64_t factor_len;
    int32_t ns;
    int32_t kb;
    double eps;
};
template <typename T>
cudaError_t launch_chol_step(const CholStepArgs<T>& a, int nmembers, cudaStream_t st);

template <typename T>
struct GemmArgs {
    const GemmTile* tiles;
    int32_t count;
    const int32_t* members;
    const T* abuf;     // buffer of A (factor or workspace)
    const T* bbuf;     // buffer of B (factor or U^T panels)
    T* cbuf;           // buffer of C (factor or CB arena)
    int64_t astride, bstride, cstride;  // per-member strides of the three buffers
    const int32_t* finfo;
    int32_t ns;
    int32_t* status;   // tensor-core GEMM: nonzero when a bounded wait for the MMAs gave up
    const T* copy_src; // mode-2 tiles: C = copy_src[a ...] (ld lda), m x n
    int64_t copy_stride;   // per-member stride of copy_src
    int32_t exact;     // FP64 mode-0 tiles summed in the oracle's order, every product and sum rounded:
                       // 1 (LDLT) c = c - a_k b_k for k = 0, 1, ...; 2 (LU) c = c - (a_0 b_0 + a_1 b_1 + ...)
    int32_t simt;      // FP32: the SIMT kernel (the panel steps' rank-32 updates) instead of tcgen05
};

// FP32 grouped GEMM on the tensor cores (tcgen05, 3xTF32); tc_kernels.cu
cudaError_t launch_gemm_tc32(const GemmArgs<float>& a, int nmembers, cudaStream_t st);
cudaError_t prepare_tc_kernels();

// Large LDLT / LU fronts: one CTA per front, the in-front steps on the global panels.
template <typename T>
struct LargePivotArgs {
    const DFront* fronts;
    const int32_t* list;
    int32_t count;
    const int32_t* members;
    T* factor;
    T* ufactor;
    double* scratch;         // per-front scratch (offsets in scr_off), per member stride scr_len
    const int64_t* scr_off;  // per listed front
    int64_t scr_len;
    double* d;
    int32_t* piv;
    int8_t* kind;
    int64_t* stats;
    int32_t* finfo;
    const int8_t* psign;
    const int32_t* perm;
    int64_t factor_len, n;
    int32_t ns;
    int32_t pivot, lu_pivot;
    double u, eps;
};

// W = L21 D of large LDLT / LU fronts into a workspace (m x w per front, ld m).
template <typename T>
struct ScaleArgs {
    const DFront* fronts;
    const int32_t* list;
    int32_t count;
    const int64_t* woff;     // workspace offset per listed front
    const int32_t* members;
    const T* factor;
    const double* d;
    const int8_t* kind;
    T* work;
    int64_t factor_len, n, work_len;
};

template <typename T>
cudaError_t launch_small(int structure, const SmallArgs<T>& a, int count, int nmembers, int fmax, cudaStream_t st);
size_t small_front_smem(int fmax, int elsize);
template <typename T>
cudaError_t launch_assemble_large(int structure, const LargeAsmArgs<T>& a, int nmembers, cudaStream_t st);
cudaError_t launch_stats(const StatsArgs& a, int nmembers, cudaStream_t st);
// the Schur complement of the unfactored root panel at p0 as a dense matrix (schur_kernels.cu)
template <typename T>
cudaError_t launch_schur_dense(const T* factor, const T* ufactor, int64_t p0, int ns, double* D, int64_t ldd,
                               int transposed, cudaStream_t st);
template <typename T>
cudaError_t launch_gemm(const GemmArgs<T>& a, int nmembers, cudaStream_t st);
// Inverses of the 64 x 64 diagonal blocks of the L11 panels of the wide fronts (for the solve)
template <typename T>
struct BlockInvArgs {
    const DFront* fronts;
    const int32_t* tasks;      // (front, block) pairs
    int32_t count;
    const int64_t* dinv_off;   // per front
    const int32_t* members;
    const T* panels;           // factor or U^T panels
    T* dinv;
    int64_t factor_len, dinv_len;
    const int32_t* finfo;
    int32_t ns;
    int32_t panel_layout;      // 1: block b goes to rows and columns 64 b of the front's f x w inverse panel
                               // (ld f, only the block's own entries written); 0: 64 x 64 blocks in turn
};

// The inverse-panel GEMMs (pinv_kernels.cu): C = +-A B over a list of 64 x 64 tiles
template <typename T>
struct PinvGemmArgs {
    const PinvTile* tiles;
    int32_t count;
    const int32_t* members;
    const T* abuf;
    const T* bbuf;
    T* cbuf;
    int64_t astride, bstride, cstride;   // per-member strides
    const int32_t* finfo;
    int32_t ns;
    T* part;                   // split tiles: 64 x 64 partial products (single-member plans)
    unsigned int* cnt;         // split tiles: arrival counters, zero between launches
};
template <typename T>
cudaError_t launch_pinv_gemm(const PinvGemmArgs<T>& a, int nmembers, cudaStream_t st);
template <typename T>
cudaError_t launch_block_inv(const BlockInvArgs<T>& a, int nmembers, cudaStream_t st);

// Inverses of L11 (w <= 32) of the dataflow solve's warp fronts, w x w (ld w, zero above the diagonal)
template <typename T>
struct SmallInvArgs {
    const DFront* fronts;
    const int32_t* list;       // the fronts
    int32_t count;
    const int64_t* inv_off;    // per front
    const int32_t* members;
    const T* panels;           // factor or U^T panels
    T* inv;
    int64_t factor_len, inv_len;
    const int32_t* finfo;
    int32_t ns;
};
template <typename T>
cudaError_t launch_small_inv(const SmallInvArgs<T>& a, int nmembers, int wmax, cudaStream_t st);   // wmax: widest
                                                                                             // front (0: 32)
cudaError_t prepare_dataflow_kernels(int max_smem);

constexpr int CHOL_NB = 32;   // column block of the large-front Cholesky (one warp per diagonal block)
cudaError_t prepare_factor_kernels(int max_smem);
cudaError_t prepare_dense_kernels(int max_smem);
cudaError_t prepare_solve_kernels(int max_smem);   // column block of the large-front Cholesky
template <typename T>
cudaError_t launch_large_pivot(int structure, const LargePivotArgs<T>& a, int nmembers, cudaStream_t st);
template <typename T>
cudaError_t launch_scale_ld_front(int structure, const ScaleArgs<T>& a, int maxw, int nmembers, cudaStream_t st);

// groups of co-resident CTAs for the cooperative large-front pivot kernel (single-member plans)
struct CoopGroups {
    const int32_t* cta_first;  // per listed front: first CTA of its group (count + 1 entries)
    unsigned int* bar;         // per listed front: group barrier counter, zeroed before the launch
    int32_t* status;           // nonzero: a group barrier wait gave up
};
constexpr int COOP_THREADS = 256;
template <typename T>
cudaError_t launch_large_pivot_coop(int structure, const LargePivotArgs<T>& a, const CoopGroups& g, int grid,
                                    cudaStream_t st);
template <typename T>
int large_pivot_coop_capacity(int structure);   // co-resident CTAs of the cooperative kernel on this device

// sampled outer product over a CSR pattern (the adjoint of a solve with respect to the values)
template <typename I>
struct OuterArgs {
    const I* rowptr;           // n + 1, base `base`
    const I* colval;           // nnz
    int64_t base, n, nnz;
    int32_t structure;         // STRUCT_G, STRUCT_S or STRUCT_SPD
    int32_t view;              // 'F', 'L' or 'U' (symmetric structures keep one triangle)
    const double* U;           // n x ncols per member (ld ldu, member stride ldu * ncols)
    const double* V;
    int64_t ldu, ldv;
    int32_t ncols;
    double alpha;
    double* out;               // nnz per member
};
template <typename I>
cudaError_t launch_sampled_outer(const OuterArgs<I>& a, int nmembers, cudaStream_t st);

constexpr int GEMM_BM = 64, GEMM_BN = 64;
constexpr int GEMM_BM_TC = 128;   // rows of a tcgen05 contribution-block tile (FP32 plans)

}  // namespace sds

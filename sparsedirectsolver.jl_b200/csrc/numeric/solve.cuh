// Argument blocks of the solve-phase kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace sds {

template <typename T>
struct SweepArgs {
    const DFront* fronts;
    const int32_t* list;
    int32_t count;
    const int32_t* members;
    const T* fac;              // panels of this sweep (factor, or U^T panels)
    double* Y;                 // n x nrhs per member
    double* U;                 // update vectors / gathered rows (per member stride ulen)
    const int64_t* uoff;       // per front (m x nrhs, ld m)
    const int32_t* child_list;
    const int32_t* relind;
    const int32_t* rowval;
    const int32_t* piv;        // 1-based factor columns, per member (NULL without reordering)
    int64_t n, factor_len, ulen;
    int32_t nrhs;
    int32_t unit;              // unit diagonal (LDLT, LU)
    int32_t reorder;           // apply (forward) / undo (backward) the local pivot order
    int32_t rect;              // 1: this CTA also does the rectangular part (L21 x / L21^T x)
    int32_t pull_only;         // forward: only pull the children's updates into Y (the unfactored Schur root)
    const int32_t* tiles;      // split rectangular part of large fronts: (front, first row / column) pairs
};

// ---------------------------------------------------------------------------------------------------
// Dataflow solve: the whole solve (forward, diagonal, backward, both permutations) in one persistent
// cooperative launch with no grid barrier. Work is a list of tasks in a topological order of the
// elimination tree (forward leaves to roots, then backward roots to leaves). CTAs take tasks in list
// order from one atomic counter; a task waits only on tasks earlier in the list (counters and flags
// with bounded waits), so the launch cannot deadlock while all CTAs are resident.
//
// Front classes:
//  * warp fronts (w <= DF_WARP_W and f <= DF_WARP_F): one warp each; DF_BUNDLE fronts of one level per
//    task, taken by the CTA's warps in turn. L11^-1 (w x w, ld w) is precomputed after the factorization.
//  * tiled fronts (the rest), in one of two forms chosen per plan:
//    - inverse panels (default): the front's f x w inverse panel P = [L11^-1; L21 L11^-1] (ld f) is
//      precomputed after the factorization, so that the forward is [x1; u - u_children] = P z1 and the
//      backward x1 = P^T [y1; -x2]: one matrix-vector product per sweep, split into tasks over
//      (64-row tile, DF_PCOLS-column chunk) in the forward and (DF_PBCOLS-column block, DF_PROWS-row
//      chunk) in the backward; the last task of a tile or block to finish (a counter) sums the
//      partial products in chunk order;
//    - block chains: forward = one task per 64-row tile, which gathers its own rows (the right-hand
//      side and the children's updates) and takes the 64-column blocks k <= t in order (block t's own
//      tile solves it with the precomputed 64 x 64 inverse and publishes x_t); backward = partial-sum
//      tasks over DF_CHUNK-row chunks of the update rows (-L21^T x2 per block) and one owner task per
//      64-column block, from the last block to the first.
// The children's updates reach a front through per-row contribution lists (the child update rows that
// land on each front row, in child order), so every row is gathered by one thread with independent
// loads and a fixed summation order.
constexpr int DF_WARP_W = 32;     // widest warp front
constexpr int DF_WARP_F = 128;    // tallest warp front (the plan's tuning may lower it)
constexpr int DF_BUNDLE = 8;      // warp fronts per task (one per warp)
constexpr int DF_BLK = 64;        // tile rows and block columns of the tiled fronts
constexpr int DF_CHUNK = 128;     // update rows per backward partial task
constexpr int DF_MAX_NRHS = 8;    // right-hand sides per launch (more are solved in groups of 8)
constexpr int DF_THREADS = 256;
constexpr int DF_PCOLS = 128;     // inverse panels, forward: columns per task (a 64 x 128 part of P)
constexpr int DF_PBCOLS = 32;     // inverse panels, backward: columns per task ...
constexpr int DF_PROWS = 128;     // ... and rows (a 128 x 32 part of P)

enum DfTaskKind : int32_t {
    DF_FW_BUNDLE = 1, DF_FW_TILE = 3, DF_BW_BUNDLE = 4, DF_BW_PART = 5, DF_BW_OWNER = 6, DF_FW_PINV = 7, DF_BW_PINV = 8
};

struct DfTask {
    int32_t kind, a, b, c;   // bundle: a = offset in the bundle list, b = count; tile: a = front, b = tile;
                             // part: a = front, b = block, c = chunk; owner: a = front, b = block;
                             // inverse panel: a = front, b = row tile (forward) or column block (backward),
                             // c = chunk | first partial slot of the tile or block << 8
};

// inverse-panel fronts: column chunks of forward row tile t, and row chunks of backward column block b
// (the first one, b DF_PBCOLS / DF_PROWS, is the first that reaches the block's diagonal)
__host__ __device__ inline int df_pf_chunks(int w, int t) {
    const int cols = w < DF_BLK * (t + 1) ? w : DF_BLK * (t + 1);
    return (cols + DF_PCOLS - 1) / DF_PCOLS;
}
__host__ __device__ inline int df_pb_first(int b) { return (DF_PBCOLS * b) / DF_PROWS; }
__host__ __device__ inline int df_pb_chunks(int f, int b) { return (f + DF_PROWS - 1) / DF_PROWS - df_pb_first(b); }

struct DfFront {
    int64_t inv;       // offset of the front's inverses (warp: L11^-1, w x w; tiled: the inverse panel,
                       // f x w, or the nblk 64 x 64 diagonal-block inverses)
    int32_t tiled;     // 0: warp front; 1: tiled
    int32_t pinv;      // tiled: solved through its inverse panel
    int32_t bsig;      // backward signals of this front (its children wait for bdone >= bsig)
    int32_t tcnt;      // inverse panel: first of its forward row-tile counters
    int32_t ccnt;      // inverse panel: first of its backward column-block counters
    int32_t pbblk;     // inverse panel: backward column blocks (DF_PBCOLS wide)
    int32_t ntile;     // tiled: 64-row tiles of the forward
    int32_t nblk;      // tiled: 64-column blocks
    int32_t nchunk;    // tiled: backward partial tasks per block (0: the owners sum the update rows themselves)
    int32_t fneed;     // forward signals this front waits for (one per forward task of each child)
    int32_t fsig;      // forward tasks of this front (each signals its parent, or the front itself at a root)
    int32_t blk;       // tiled: first index of its blocks in the per-block flags
    int32_t part;      // tiled: first partial slot (nblk x nchunk slots of 64 x DF_MAX_NRHS doubles)
    int32_t urow;      // first of its update rows in the global numbering of update rows (U is
                       // U[(urow + i) * nrhs + r] for update row i and right-hand side r)
    int32_t rbase;     // its f + 1 row pointers into the contribution lists start at rptr[rbase]
};

template <typename T>
struct DataflowArgs {
    const DfTask* tasks;
    int32_t ntasks;
    const DFront* fronts;
    const DfFront* df;
    const int32_t* bundles;    // fronts of the warp bundles
    const int32_t* rptr;       // per front row: start of its contributions in csrc
    const int32_t* csrc;       // contributions: global update rows of the children, in child order
    const T* facf;             // panels of the forward sweep (L; U^T panels for LU with A^T)
    const T* facb;             // panels of the backward sweep
    const T* invf;             // diagonal-block inverses of facf's panels
    const T* invb;             // ... of facb's panels
    const int32_t* rowval;
    const int32_t* piv;        // 1-based local pivot order (LDLT, LU)
    const int32_t* perm;       // 0-based original index of each factor position
    const double* d;
    const int8_t* kind;
    const double* in;          // B (mode 0) or R (mode 2), column-major, ld ldin
    double* out;               // X, ld ldout
    int64_t ldin, ldout, n;
    double* Y;                 // n x nrhs: forward result (pre-D) then solution, factor order
    double* U;                 // update vectors, (global update row) x nrhs, row-major
    double* xtmp;              // n x nrhs: a tiled front's published block solutions; an inverse-panel
                               // front's forward result (its backward then writes the solution into Y)
    double* part;              // backward partial sums
    unsigned int* fcnt;        // ns: forward signals received (from children; at a root from itself)
    unsigned int* bdone;       // ns: 1 once the front's backward solution is in Y
    unsigned int* xflag;       // per block: 1 forward x_k published, 2 backward x_k published
    unsigned int* pcnt;        // per block: backward partials written
    unsigned int* tcnt;        // inverse panels: per forward row tile, partial products written
    unsigned int* ccnt;        // inverse panels: per backward column block, partial products written
    unsigned int* head;        // the task counter
    int32_t* status;           // nonzero: a bounded wait gave up
    int32_t nrhs;              // <= DF_MAX_NRHS
    int32_t reorder_fw, reorder_bw;
    int32_t diag_mode;         // 0 none (Cholesky), 1 D (LU), 2 D with 2x2 blocks (LDLT)
    int32_t mode;              // 0: X = solve(B); 2: X += solve(R)
    int32_t warp_smem;         // doubles of shared memory per warp of a bundle task
    int64_t* trace;            // profiling, or NULL: per task (start, wait done, end) %globaltimer ns, CTA, kind, a | b << 32
    // uniform batches: the launch runs every task for each of nmembers members (task-major, so a task
    // still waits only on tasks earlier in the launch's order); the member-dependent arrays above are
    // member 0's and advance by these strides (elements)
    int32_t nmembers;
    const int32_t* members;    // the members' indices (NULL: 0 .. nmembers - 1)
    int64_t s_fac, s_inv, s_piv, s_d, s_in, s_out, s_y, s_u, s_part, s_flags;
};

template <typename T>
cudaError_t launch_dataflow_solve(const DataflowArgs<T>& a, int grid, size_t smem, cudaStream_t st);
template <typename T>
int dataflow_solve_grid(int nrhs, size_t smem);

struct DiagArgs {
    const int32_t* members;
    const double* d;
    const int8_t* kind;
    double* Y;
    int64_t n;
    int32_t nrhs;
    int32_t two;               // 2x2 blocks (LDLT)
};

struct PermArgs {
    const int32_t* members;
    const int32_t* perm;       // 0-based original index of each factor position; NULL: the identity
    double* Y;
    const double* in;          // mode 0
    double* out;               // modes 1, 2
    int64_t n, ldin, ldout;
    int32_t nrhs;
    int32_t mode;
};

struct ResidualArgs {
    const int32_t* members;
    const int64_t* rowptr;     // 0-based, n + 1
    const int64_t* colval;     // 0-based
    const int64_t* srcptr;     // 0-based, entries + 1
    const int64_t* src;        // 0-based nzval positions
    const double* nzval;
    const double* X;
    const double* B;
    double* R;
    int64_t n, nnz, ldx, ldb;
    int32_t nrhs;
    int64_t entries;           // entries of the map (rowptr[n]): short rows take one thread each
};

struct NormArgs {
    const int32_t* members;
    const double* R;
    const double* B;
    double* out;               // 2 per (member, rhs)
    int64_t n, ldb;
    int32_t nrhs;
};

template <typename T>
cudaError_t launch_sweep(bool forward, const SweepArgs<T>& a, int nmembers, int maxw, cudaStream_t st);
// rectangular part of large fronts: forward u += L21 x (row tiles), backward x1 -= L21^T x2 (column tiles)
template <typename T>
cudaError_t launch_sweep_rect(bool forward, const SweepArgs<T>& a, int ntiles, int nmembers, int maxw, cudaStream_t st);
constexpr int RECT_ROWS = 256;   // rows of a forward tile
constexpr int RECT_COLS = 16;    // columns of a backward tile (one warp each, 16 warps)
cudaError_t launch_diag(const DiagArgs& a, int nmembers, cudaStream_t st);
cudaError_t launch_permute(const PermArgs& a, int nmembers, cudaStream_t st);
cudaError_t launch_residual(const ResidualArgs& a, int nmembers, cudaStream_t st);
cudaError_t launch_norms(const NormArgs& a, int ncols, cudaStream_t st);

}  // namespace sds

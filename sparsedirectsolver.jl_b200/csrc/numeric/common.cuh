// Shared definitions of the B200 numeric phase (device descriptors, plan layout).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../../include/sdsb200.h"

namespace sds {

constexpr int NSTAT = 6;  // per-front statistics: npos, nneg, nzero, nperturbed, n2x2, info
enum { ST_NPOS = 0, ST_NNEG, ST_NZERO, ST_NPERT, ST_N2X2, ST_INFO };
enum { KIND_1X1 = 1, KIND_2X2_FIRST = 2, KIND_2X2_SECOND = 3, KIND_PERTURBED = 4 };
enum { PIVOT_AUTO = 0, PIVOT_NONE = 1, PIVOT_DIAGONAL = 4, PIVOT_LOCAL = 5, PIVOT_BK = 6 };
enum { STRUCT_G = 0, STRUCT_S = 1, STRUCT_SPD = 3 };

// Device descriptor of one front (supernode). All offsets 0-based, per batch member.
struct DFront {
    int64_t panel;     // offset of the f x w panel (column-major, ld f) in the factor buffer
    int64_t cb;        // offset of the m x m contribution block (column-major, ld m) in the CB arena; -1 none
    int32_t f, w, c0;  // rows, fully-summed columns, first factor column
    int32_t parent;    // -1 for a root
    int32_t ch_begin, ch_end;  // children in child_list
    int32_t ri_begin;  // this front's relind (its rows w..f-1 among the parent's), length f - w
    int32_t am_begin, am_end;  // assembly entries (am_src/am_loc)
    int32_t row_begin;         // rows in rowval (f entries; its own columns first)
    int32_t amcol_begin;       // per-column start of the assembly entries: amcol[amcol_begin + j], j <= w
    int32_t eacol_begin;       // column-owner extend-add lists of a large front: eacol[eacol_begin + p], p <= f
    int32_t level;
    int32_t rc_begin;  // this front's row-chunk starts among its parent's rows: rchunk[rc_begin + k], k <= K
};

// Rows of a front column that the large-front assembly builds at a time in shared memory (per warp)
constexpr int ASM_ROWS = 256;

// Row chunk and column group of one update item of the cooperative LDLT / LU kernel
constexpr int COOP_ROWS = 256;
constexpr int COOP_COLS = 32;

// Scratch (in doubles) of a wide LDLT / LU front: multipliers (2 f), D (2 w), local order and
// control (w + 16 ints), kinds (w bytes); then the cooperative kernel's per-chunk column maxima
__host__ __device__ inline int64_t pivot_scratch_base(int f, int w) {
    return 2 * (int64_t)f + 2 * (int64_t)w + (w + 16 + 1) / 2 + (w + 7) / 8 + 8;
}
__host__ __device__ inline int64_t pivot_scratch_len(int f, int w) {
    return pivot_scratch_base(f, w) + (int64_t)w * ((f + COOP_ROWS - 1) / COOP_ROWS);
}

// Column task of the large-front assembly: (front, parent index p); one warp each.
struct ColTask {
    int32_t front, p;
};

// One tile of a grouped GEMM  C -= A * B^T  (all column-major). Offsets point at the
// tile's first element: A at its first row, B at its first row (= the tile's first
// column of C), C at (row0, col0). Entry (r, c) of the tile is written only when
// r + diag >= c (diag = row0 - col0 for the lower triangle; a large value disables the mask).
struct GemmTile {
    int64_t a, b, c;
    int32_t lda, ldb, ldc;
    int32_t m, n, k;     // valid rows and columns of this tile (<= tile size), inner dimension
    int32_t diag;
    int32_t front;       // status check: the tile is skipped when this front failed (-1: none)
    int32_t mode;        // 0: C -= A B^T; 1: C = A B^T (in place over A's rows: trsm by an inverse);
                         // 2: C = copy_src block at a (a deferred diagonal-block write)
    int32_t pad;
};

// A launch of the factorization program.
enum LaunchKind : int32_t {
    L_SMALL = 1,       // fused small fronts (one CTA per front, front in shared memory)
    L_ASSEMBLE,        // column-task assembly of large fronts
    L_GEMM,            // grouped GEMM tiles
    L_PIVOT_FRONT,     // large LDLT / LU: cooperative pivoting over the panel
    L_STATS,           // statistics reduction
    L_SCALE,           // W = L21 D of large LDLT / LU fronts
    L_CHOL_STEP,       // large Cholesky: one 32-column step (diagonal block + trsm of the rows below)
    L_DFINV,           // diagonal-block inverses of every front for the dataflow solve
    L_PINV,            // GEMM tiles that build the inverse panels of the dataflow solve's tiled fronts
    L_CHOL_FLOW,       // large Cholesky: every 32-column step of a batch as dataflow tasks in one launch
    L_SUBTREE,         // fused subtrees of small fronts (one CTA per subtree, fronts in postorder)
};

// One 64 x 64 output tile of the inverse-panel GEMMs: C = A B, or C = -A B (column-major operands).
// A long inner dimension is split over nsplit CTAs (split = this CTA's part, its A and B offsets and k
// already advanced): each writes its partial product to slot `slot + split` of the launch's partial
// buffer and the last of them to finish (counter `cnt`, which it resets) sums the parts in order.
struct PinvTile {
    int64_t a, b, c;     // element offsets of A (m x k), B (k x n) and C (m x n)
    int32_t lda, ldb, ldc;
    int32_t m, n, k;
    int32_t front;       // skipped when this front failed
    int32_t neg;
    int32_t nsplit, split, slot, cnt;
};
constexpr int PINV_KSPLIT = 256;   // longest inner dimension of one CTA's part

constexpr int FSTREAM_DEFAULT = 4;   // factorization streams of a single-system Cholesky plan
constexpr int FSTREAM_MIN_CP = 16;   // the critical path (32-column steps) of a subtree given its own stream

struct Launch {
    LaunchKind kind;
    int32_t level;
    int32_t count;       // fronts / tasks / tiles
    int32_t cls;         // small-front class (max rows), or column-block start (panel)
    int64_t list;        // offset of the front/task/tile list in its device array
    int32_t nb;          // panel block width
    int32_t smem;        // dynamic shared memory bytes
};

struct DeviceMaps {
    const DFront* fronts;
    const int32_t* child_list;
    const int32_t* relind;
    const int32_t* am_src;
    const int32_t* am_loc;   // (loc + 1) for L entries, -(loc + 1) for U^T entries; loc within the panel
    const int32_t* amcol;    // per-column starts of the assembly entries
    const int32_t* ea;       // extend-add pairs (child, t) packed as 2 int32
    const int32_t* eacol;    // per parent index starts into ea
    const int32_t* rchunk;   // per child of a large front: the first of its relind rows at or beyond each
                             // multiple of ASM_ROWS of the parent's rows (K + 1 entries, K = ceil(f / ASM_ROWS))
    const int32_t* rowval;   // 0-based
    const int32_t* perm;     // 0-based
};

// Strided copy loops with many loads in flight: for q = t0, t0 + step, ... < N, first load U values into
// registers, then store them. The explicit batch keeps loads independent of the stores even when the
// compiler cannot tell the shared- and global-memory pointers apart.
template <int U, class LD, class ST>
__device__ __forceinline__ void batched_copy(int t0, int step, int N, LD load, ST store) {
    for (int q0 = t0; q0 < N; q0 += U * step) {
        double v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int q = q0 + u * step;
            v[u] = q < N ? load(q) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int q = q0 + u * step;
            if (q < N) store(q, v[u]);
        }
    }
}

// Scattered accumulation *dst(q) += val(q) for q = t0, t0 + step, ... < N, where no two q of one call
// share a target (dst returns nullptr to skip q). U values and U current targets are loaded before
// the U stores, so the read-modify-writes of a batch overlap instead of running one after another.
template <int U, class T, class VAL, class DST>
__device__ __forceinline__ void batched_add(int t0, int step, int N, VAL val, DST dst) {
    for (int q0 = t0; q0 < N; q0 += U * step) {
        T* p[U];
        double v[U], c[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int q = q0 + u * step;
            p[u] = q < N ? dst(q) : nullptr;
            v[u] = p[u] ? val(q) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) c[u] = p[u] ? (double)*p[u] : 0.0;
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (p[u]) *p[u] = T(c[u] + v[u]);
    }
}

}  // namespace sds

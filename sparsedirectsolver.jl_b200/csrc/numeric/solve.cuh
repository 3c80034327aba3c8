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

// One cooperative launch for a whole solve (nact == 1): permutation, forward levels, diagonal,
// backward levels, inverse permutation, separated by bounded grid barriers.
template <typename T>
struct PersistArgs {
    SweepArgs<T> fw;           // forward sweep configuration (fac, unit, reorder, piv, Y, U, ...)
    SweepArgs<T> bw;           // backward sweep configuration
    const T* dinv_fw;          // inverses of the 64 x 64 diagonal blocks of the forward panels
    const T* dinv_bw;          // ... of the backward panels
    const int64_t* dinv_off;   // per front (-1: not a wide front)
    const int32_t* lev_small;  // per level: offset and count of small fronts in `list`
    const int32_t* lev_large;  // per level: offset and count of wide fronts in `list`
    const int32_t* lev_maxblk; // per level: largest number of 64-column blocks among its wide fronts
    const int32_t* list;       // fronts of all levels
    int32_t nlevels;
    const double* d;
    const int8_t* kind;
    int32_t diag_mode;         // 0 none (Cholesky), 1 D (LU), 2 D with 2x2 blocks (LDLT)
    const int32_t* perm;
    const double* in;          // B (mode 0) or R (mode 2)
    double* out;               // X
    int64_t ldin, ldout;
    int32_t mode;              // 0: X = solve(B); 2: X += solve(R)
    double* xtmp;              // n x nrhs scratch
    unsigned int* barrier;     // grid barrier counter (zeroed before the launch)
    unsigned int* blkflag;     // per 64-column diagonal block of the wide fronts (front s: from dinv_off[s] /
                               // 4096): 1 once its forward solution is published, 2 once its backward one is
    unsigned int* pullflag;    // per wide front (at its first block's index): 1 once its forward pull is done
    unsigned int* l21cnt;      // per block: columns whose backward -L21^T x2 is applied
                               // (all three zeroed before the launch)
    int32_t* status;           // nonzero: a barrier or flag wait gave up
    int64_t* trace;            // profiling: (tag, %globaltimer ns) pairs written by CTA 0, or NULL
    int32_t trace_cap;
    int32_t warp_smem;         // doubles of shared memory per warp for the small fronts (xs + Ld)
    int32_t warp_xs;           // doubles of xs within it
};

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
template <typename T>
cudaError_t launch_persistent_solve(const PersistArgs<T>& a, int grid, size_t smem, cudaStream_t st);
template <typename T>
int persistent_solve_grid(size_t smem);
constexpr int SOLVE_BLK = 64;    // column block of the wide-front sweeps (the diagonal-block inverses)
cudaError_t launch_permute(const PermArgs& a, int nmembers, cudaStream_t st);
cudaError_t launch_residual(const ResidualArgs& a, int nmembers, cudaStream_t st);
cudaError_t launch_norms(const NormArgs& a, int ncols, cudaStream_t st);

}  // namespace sds

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
    const int32_t* tiles;      // split rectangular part of large fronts: (front, first row / column) pairs
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
    const int32_t* perm;       // 0-based original index of each factor position
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
cudaError_t launch_permute(const PermArgs& a, int nmembers, cudaStream_t st);
cudaError_t launch_residual(const ResidualArgs& a, int nmembers, cudaStream_t st);
cudaError_t launch_norms(const NormArgs& a, int ncols, cudaStream_t st);

}  // namespace sds

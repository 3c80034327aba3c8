// Adjoint of a solve with respect to the matrix values: the sampled outer product over the CSR
// pattern. The reference has no automatic differentiation; this is the matrix half of the
// differentiation rule of x = A^{-1} b (the other half, b_bar = A^{-T} x_bar, is a transposed solve
// with the device-resident factor):
//
//   A_bar[k] = alpha * sum_r U[i, r] V[j, r]                    "G": every stored entry k = (i, j)
//   A_bar[k] = alpha * sum_r (U[i, r] V[j, r] + U[j, r] V[i, r])  "S"/"SPD", a kept entry, i != j
//   A_bar[k] = alpha * sum_r U[i, r] V[i, r]                    "S"/"SPD", a kept diagonal entry
//   A_bar[k] = 0                                               "S"/"SPD", an entry the view drops
//
// With alpha = -1, U = b_bar and V = x this is dL/dA for every value the factorization reads. For the
// symmetric structures the kept entry stands for both a_ij and a_ji, so both terms of the symmetric
// perturbation count. Which entries are kept is the analysis's view filter: the lower triangle for
// views "F" and "L", the upper one for "U".
//
// One CTA per 256 rows: the CTA stages the rows' pointers in shared memory, its threads stride over
// the rows' entries (coalesced colval and output) and find each entry's row by binary search.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "kernels.cuh"

namespace sds {

constexpr int OUTER_ROWS = 256;

template <typename I>
__global__ void __launch_bounds__(OUTER_ROWS) sampled_outer_kernel(OuterArgs<I> A) {
    __shared__ int64_t rp[OUTER_ROWS + 1];
    const int64_t r0 = (int64_t)blockIdx.x * OUTER_ROWS;
    const int64_t member = blockIdx.y;
    const int nr = (int)(A.n - r0 < OUTER_ROWS ? A.n - r0 : OUTER_ROWS);
    for (int t = threadIdx.x; t <= nr; t += blockDim.x) rp[t] = (int64_t)A.rowptr[r0 + t] - A.base;
    __syncthreads();
    const int64_t e0 = rp[0], e1 = rp[nr];
    const double* U = A.U + member * A.ldu * A.ncols;
    const double* V = A.V + member * A.ldv * A.ncols;
    double* out = A.out + member * A.nnz;
    for (int64_t k = e0 + threadIdx.x; k < e1; k += blockDim.x) {
        // row: the last local row whose first entry is at or before k
        int lo = 0, hi = nr - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (rp[mid] <= k) lo = mid;
            else hi = mid - 1;
        }
        const int64_t i = r0 + lo, j = (int64_t)A.colval[k] - A.base;
        double acc = 0.0;
        if (A.structure == STRUCT_G) {
            for (int r = 0; r < A.ncols; ++r) acc += U[i + r * A.ldu] * V[j + r * A.ldv];
        } else {
            const bool keep = A.view == 'U' ? j >= i : j <= i;
            if (keep) {
                for (int r = 0; r < A.ncols; ++r) acc += U[i + r * A.ldu] * V[j + r * A.ldv];
                if (i != j)
                    for (int r = 0; r < A.ncols; ++r) acc += U[j + r * A.ldu] * V[i + r * A.ldv];
            }
        }
        out[k] = A.alpha * acc;
    }
}

template <typename I>
cudaError_t launch_sampled_outer(const OuterArgs<I>& a, int nmembers, cudaStream_t st) {
    if (a.n == 0 || nmembers == 0) return cudaSuccess;
    dim3 grid((unsigned)((a.n + OUTER_ROWS - 1) / OUTER_ROWS), nmembers);
    sampled_outer_kernel<I><<<grid, OUTER_ROWS, 0, st>>>(a);
    return cudaGetLastError();
}

template cudaError_t launch_sampled_outer<int32_t>(const OuterArgs<int32_t>&, int, cudaStream_t);
template cudaError_t launch_sampled_outer<int64_t>(const OuterArgs<int64_t>&, int, cudaStream_t);

}  // namespace sds

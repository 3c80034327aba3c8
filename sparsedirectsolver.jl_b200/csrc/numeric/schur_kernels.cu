// Export of the Schur complement of Schur complement mode (the reference's schur_matrix!,
// src/numeric/schur.jl:100-174). The factorization assembles the unfactored root front (zero, scatter
// of A, extend-add of the children's contribution blocks) and leaves S = A22 - A21 A11^{-1} A12 in its
// panel: the lower triangle in the factor panel, and for "G" the strict upper triangle transposed in
// the U^T panel. This kernel writes it as a dense column-major matrix.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace sds {

// D (ns x ns, ld ldd) = S, or S^T when transposed; the root panel starts at p0 with ld ns. Entry (a, b)
// of S with a >= b is factor[p0 + b ns + a]; with a < b it is ufactor[p0 + a ns + b] ("G") or the
// mirrored factor[p0 + a ns + b] ("S", "SPD").
template <typename T>
__global__ void schur_dense_kernel(const T* factor, const T* ufactor, int64_t p0, int ns, double* D, int64_t ldd,
                                   int transposed) {
    const int64_t total = (int64_t)ns * ns;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % ns), j = (int)(q / ns);
        const int a = transposed ? j : i, b = transposed ? i : j;
        double v;
        if (a >= b) v = (double)factor[p0 + (int64_t)b * ns + a];
        else v = (double)(ufactor ? ufactor[p0 + (int64_t)a * ns + b] : factor[p0 + (int64_t)a * ns + b]);
        D[i + (int64_t)j * ldd] = v;
    }
}

template <typename T>
cudaError_t launch_schur_dense(const T* factor, const T* ufactor, int64_t p0, int ns, double* D, int64_t ldd,
                               int transposed, cudaStream_t st) {
    if (ns <= 0) return cudaSuccess;
    const int64_t total = (int64_t)ns * ns;
    const int blocks = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
    schur_dense_kernel<T><<<blocks, 256, 0, st>>>(factor, ufactor, p0, ns, D, ldd, transposed);
    return cudaGetLastError();
}

template cudaError_t launch_schur_dense<double>(const double*, const double*, int64_t, int, double*, int64_t, int,
                                                cudaStream_t);
template cudaError_t launch_schur_dense<float>(const float*, const float*, int64_t, int, double*, int64_t, int,
                                               cudaStream_t);

}  // namespace sds

// The GEMMs that build the inverse panels P = [L11^-1; L21 L11^-1] of the dataflow solve's tiled
// fronts. L11^-1 is formed by recursive doubling over the 64 x 64 diagonal-block inverses:
// inv([A 0; B C]) = [A^-1 0; -C^-1 (B A^-1) C^-1], two GEMM launches per doubling level over every front;
// then L21 L11^-1 in one more launch. Each output tile is 64 x 64, C = A B or C = -A B with column-major
// operands and any leading dimensions; every entry is summed by one thread in a fixed order (a tile with
// a long inner dimension by several CTAs, whose parts the last one adds in order).
// * FP64: mma.sync m8n8k4 (DMMA), 4 warps of 32 x 32, K staged 16 at a time by cp.async in two buffers;
// * FP32: SIMT, 256 threads of 4 x 4 entries, the same staging.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "kernels.cuh"

namespace sds {

namespace {

__device__ __forceinline__ void pinv_cp_async(void* smem, const double* gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void pinv_cp_async(void* smem, const float* gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 4 : 0));
}
__device__ __forceinline__ void pinv_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void pinv_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

constexpr int PBK = 16;   // K per stage

// The epilogue of a tile: value v (this CTA's sum) of entry (r, c). Unsplit tiles write C = +-v; split
// tiles write their part, and the last part to arrive sums all parts in split order and writes C.
// `put` visits the CTA's entries: put(r, c, v&) for each one it owns.
template <typename T, class Visit>
__device__ __forceinline__ void pinv_epilogue(const PinvGemmArgs<T>& A, const PinvTile& t, T* Cb, Visit visit) {
    __shared__ int last;
    if (t.nsplit <= 1) {
        visit([&](int r, int c, double v) {
            if (r < t.m && c < t.n) Cb[r + (int64_t)c * t.ldc] = T(t.neg ? -v : v);
        });
        return;
    }
    T* mine = A.part + (int64_t)(t.slot + t.split) * 64 * 64;
    visit([&](int r, int c, double v) { mine[r + 64 * c] = T(v); });
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned old;
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(A.cnt + t.cnt) : "memory");
        last = old + 1 == (unsigned)t.nsplit;
        if (last) A.cnt[t.cnt] = 0u;   // every part has arrived: reset for the next launch
    }
    __syncthreads();
    if (!last) return;
    for (int q = threadIdx.x; q < 64 * 64; q += blockDim.x) {
        const int r = q & 63, c = q >> 6;
        if (r >= t.m || c >= t.n) continue;
        double v = 0.0;
        for (int sp = 0; sp < t.nsplit; ++sp) v += (double)__ldcg(A.part + (int64_t)(t.slot + sp) * 64 * 64 + q);
        Cb[r + (int64_t)c * t.ldc] = T(t.neg ? -v : v);
    }
}

// stage the K-slice [k0, k0 + PBK) of A (64 rows) and B (64 columns) into As[kk][r] and Bs[kk][c]
template <typename T, int NT, int LDS>
__device__ __forceinline__ void pinv_stage(const T* Ab, const T* Bb, const PinvTile& t, int k0, T (*As)[LDS],
                                           T (*Bs)[LDS]) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int q = 0; q < (64 * PBK) / NT; ++q) {
        const int e = tid + NT * q;
        const int r = e % 64, kk = e / 64;            // A: consecutive threads down a column
        const bool va = r < t.m && k0 + kk < t.k;
        pinv_cp_async(&As[kk][r], va ? Ab + r + (int64_t)(k0 + kk) * t.lda : Ab, va);
        const int kb = e % PBK, c = e / PBK;          // B: consecutive threads down a column of B
        const bool vb = c < t.n && k0 + kb < t.k;
        pinv_cp_async(&Bs[kb][c], vb ? Bb + (k0 + kb) + (int64_t)c * t.ldb : Bb, vb);
    }
    pinv_commit();
}

__global__ void __launch_bounds__(128) pinv_gemm_dmma_kernel(PinvGemmArgs<double> A) {
    constexpr int LDS = 72;
    __shared__ __align__(16) double As[2][PBK][LDS];
    __shared__ __align__(16) double Bs[2][PBK][LDS];
    const PinvTile t = A.tiles[blockIdx.x];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    if (A.finfo && A.finfo[(int64_t)member * A.ns + t.front] != 0) return;
    const double* Ab = A.abuf + (int64_t)member * A.astride + t.a;
    const double* Bb = A.bbuf + (int64_t)member * A.bstride + t.b;
    double* Cb = A.cbuf + (int64_t)member * A.cstride + t.c;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    const int nk = (t.k + PBK - 1) / PBK;
    if (nk > 0) pinv_stage<double, 128, LDS>(Ab, Bb, t, 0, As[0], Bs[0]);
    for (int it = 0; it < nk; ++it) {
        const int buf = it & 1;
        if (it + 1 < nk) {
            pinv_stage<double, 128, LDS>(Ab, Bb, t, (it + 1) * PBK, As[buf ^ 1], Bs[buf ^ 1]);
            pinv_wait<1>();
        } else {
            pinv_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < PBK; kk += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[buf][kk + (lane & 3)][wm * 32 + i * 8 + (lane >> 2)];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[buf][kk + (lane & 3)][wn * 32 + j * 8 + (lane >> 2)];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                                 : "+d"(acc[i][j][0]), "+d"(acc[i][j][1])
                                 : "d"(a[i]), "d"(b[j]));
        }
        __syncthreads();
    }
    pinv_epilogue<double>(A, t, Cb, [&](auto put) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e)
                    put(wm * 32 + i * 8 + (lane >> 2), wn * 32 + j * 8 + (lane & 3) * 2 + e, acc[i][j][e]);
    });
}

__global__ void __launch_bounds__(256) pinv_gemm_f32_kernel(PinvGemmArgs<float> A) {
    constexpr int LDS = 68;
    __shared__ __align__(16) float As[2][PBK][LDS];
    __shared__ __align__(16) float Bs[2][PBK][LDS];
    const PinvTile t = A.tiles[blockIdx.x];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    if (A.finfo && A.finfo[(int64_t)member * A.ns + t.front] != 0) return;
    const float* Ab = A.abuf + (int64_t)member * A.astride + t.a;
    const float* Bb = A.bbuf + (int64_t)member * A.bstride + t.b;
    float* Cb = A.cbuf + (int64_t)member * A.cstride + t.c;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    const int nk = (t.k + PBK - 1) / PBK;
    if (nk > 0) pinv_stage<float, 256, LDS>(Ab, Bb, t, 0, As[0], Bs[0]);
    for (int it = 0; it < nk; ++it) {
        const int buf = it & 1;
        if (it + 1 < nk) {
            pinv_stage<float, 256, LDS>(Ab, Bb, t, (it + 1) * PBK, As[buf ^ 1], Bs[buf ^ 1]);
            pinv_wait<1>();
        } else {
            pinv_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < PBK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[buf][kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[buf][kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
        }
        __syncthreads();
    }
    pinv_epilogue<float>(A, t, Cb, [&](auto put) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) put(tx + 16 * i, ty + 16 * j, (double)acc[i][j]);
    });
}

}  // namespace

template <>
cudaError_t launch_pinv_gemm<double>(const PinvGemmArgs<double>& a, int nmembers, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    pinv_gemm_dmma_kernel<<<dim3(a.count, nmembers), 128, 0, st>>>(a);
    return cudaGetLastError();
}

template <>
cudaError_t launch_pinv_gemm<float>(const PinvGemmArgs<float>& a, int nmembers, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    pinv_gemm_f32_kernel<<<dim3(a.count, nmembers), 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace sds

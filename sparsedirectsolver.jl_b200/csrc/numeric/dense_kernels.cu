// Dense kernels of the large fronts (the reference's regime C: cuSOLVER potrf,
// cuBLAS trsm/syrk/gemm through src/dense/interface.jl and the KA fallbacks of
// src/dense/fallback/, replaced here by hand-written kernels).
//
// * gemm_nt_dmma_kernel: grouped FP64 C -= A B^T over a list of 64 x 64 tiles on the DMMA tensor
//   path (Schur updates of the fully-summed columns and of the contribution block; "lower" tiles
//   write only on or below the diagonal; mode 2 tiles copy a deferred diagonal block). The FP32
//   form uses the tcgen05 kernel of tc_kernels.cu.
// * chol_step_kernel: one 32-column step of a large Cholesky front (diagonal block + trsm).
// * block_inv_kernel: inverses of the 64 x 64 diagonal blocks of the solve's wide fronts.
// * scale_ld_kernel: W = L21 D for the contribution-block update of those fronts.
// * gemm_nt_exact_kernel: that update in FP64 in the oracle's summation order (SIMT).
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <stdint.h>

#include "common.cuh"
#include "front_factor.cuh"
#include "kernels.cuh"

namespace sds {

// FP64 on the tensor cores: mma.sync m8n8k4 (DMMA). 64 x 64 CTA tile, 4 warps of 32 x 32,
// K in steps of 16 staged by cp.async into two shared-memory buffers.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int sz = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__global__ void __launch_bounds__(128) gemm_nt_dmma_kernel(GemmArgs<double> A) {
    constexpr int BM = 64, BK = 16, LDS = 72;   // 64 x 64 tile
    __shared__ __align__(16) double As[2][BK][LDS];
    __shared__ __align__(16) double Bs[2][BK][LDS];
    const GemmTile t = A.tiles[blockIdx.x];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    if (A.finfo && t.front >= 0 && A.finfo[(int64_t)member * A.ns + t.front] != 0) return;
    if (t.mode == 2) {   // deferred diagonal-block write
        const double* src = A.copy_src + (int64_t)member * A.copy_stride + t.a;
        double* dst = A.cbuf + (int64_t)member * A.cstride + t.c;
        for (int q = threadIdx.x; q < t.m * t.n; q += blockDim.x) dst[q % t.m + (int64_t)(q / t.m) * t.ldc] = src[q % t.m + (int64_t)(q / t.m) * t.lda];
        return;
    }
    const double* Ab = A.abuf + (int64_t)member * A.astride + t.a;
    const double* Bb = A.bbuf + (int64_t)member * A.bstride + t.b;
    double* Cb = A.cbuf + (int64_t)member * A.cstride + t.c;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    const int M = t.m, N = t.n, K = t.k;
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    auto load = [&](int buf, int k0) {
#pragma unroll
        for (int q = 0; q < (BM * BK) / 128; ++q) {
            int e = tid + 128 * q, r = e % BM, kk = e / BM;
            bool va = r < M && k0 + kk < K;
            cp_async8(&As[buf][kk][r], va ? Ab + r + (int64_t)(k0 + kk) * t.lda : Ab, va);
            bool vb = r < N && k0 + kk < K;
            cp_async8(&Bs[buf][kk][r], vb ? Bb + r + (int64_t)(k0 + kk) * t.ldb : Bb, vb);
        }
        cp_async_commit();
    };
    const int nk = (K + BK - 1) / BK;
    load(0, 0);
    for (int it = 0; it < nk; ++it) {
        const int buf = it & 1;
        if (it + 1 < nk) {
            load(buf ^ 1, (it + 1) * BK);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
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
    // epilogue: every C load is issued before the first store (the stores cannot be proven not to
    // alias the loads, so an interleaved read-modify-write would serialise 32 memory round trips)
    if (!t.mode) {
        double cv[4][4][2];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int r = wm * 32 + i * 8 + (lane >> 2);
                    const int c = wn * 32 + j * 8 + (lane & 3) * 2 + e;
                    cv[i][j][e] = (r < M && c < N && r + t.diag >= c) ? Cb[r + (int64_t)c * t.ldc] : 0.0;
                }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e) acc[i][j][e] = cv[i][j][e] - acc[i][j][e];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int r = wm * 32 + i * 8 + (lane >> 2);
                const int c = wn * 32 + j * 8 + (lane & 3) * 2 + e;
                if (r < M && c < N && r + t.diag >= c) Cb[r + (int64_t)c * t.ldc] = acc[i][j][e];
            }
}

// The FP64 contribution-block update of an LDLT / LU front in the oracle's order (ref_ldlt!
// src/reference/ldlt.jl:184-191: F22 -= W L21^T one rank-1 term after another; ref_lu!
// src/reference/lu.jl:142-150: F22 -= sum_k (L21 d)_k U12_k, the sum accumulated from zero first).
// Every product and sum is rounded on its own (__dmul_rn / __dadd_rn / __dsub_rn are never fused),
// so the contribution blocks, and the pivot decisions of the parents that assemble them, are those
// of the oracle bit for bit. SIMT FP64, 64 x 64 tile, 256 threads of 4 x 4 entries, K staged 16 at a
// time in two shared-memory buffers; mode-0 tiles only.
__global__ void __launch_bounds__(256) gemm_nt_exact_kernel(GemmArgs<double> A) {
    constexpr int BM = 64, BK = 16, LDS = 72;
    __shared__ __align__(16) double As[2][BK][LDS];
    __shared__ __align__(16) double Bs[2][BK][LDS];
    const GemmTile t = A.tiles[blockIdx.x];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    if (A.finfo && t.front >= 0 && A.finfo[(int64_t)member * A.ns + t.front] != 0) return;
    const double* Ab = A.abuf + (int64_t)member * A.astride + t.a;
    const double* Bb = A.bbuf + (int64_t)member * A.bstride + t.b;
    double* Cb = A.cbuf + (int64_t)member * A.cstride + t.c;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int M = t.m, N = t.n, K = t.k;
    const bool running = A.exact == 1;
    double c[4][4], acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = tx + 16 * i, col = ty + 16 * j;
            c[i][j] = (r < M && col < N && r + t.diag >= col) ? Cb[r + (int64_t)col * t.ldc] : 0.0;
            acc[i][j] = 0.0;
        }
    auto load = [&](int buf, int k0) {
#pragma unroll
        for (int q = 0; q < (BM * BK) / 256; ++q) {
            int e = tid + 256 * q, r = e % BM, kk = e / BM;
            bool va = r < M && k0 + kk < K;
            cp_async8(&As[buf][kk][r], va ? Ab + r + (int64_t)(k0 + kk) * t.lda : Ab, va);
            bool vb = r < N && k0 + kk < K;
            cp_async8(&Bs[buf][kk][r], vb ? Bb + r + (int64_t)(k0 + kk) * t.ldb : Bb, vb);
        }
        cp_async_commit();
    };
    const int nk = (K + BK - 1) / BK;
    load(0, 0);
    for (int it = 0; it < nk; ++it) {
        const int buf = it & 1;
        if (it + 1 < nk) {
            load(buf ^ 1, (it + 1) * BK);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const int kc = min(BK, K - it * BK);
        for (int kk = 0; kk < kc; ++kk) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[buf][kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[buf][kk][ty + 16 * j];
            if (running) {
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) c[i][j] = __dsub_rn(c[i][j], __dmul_rn(a[i], b[j]));
            } else {
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = __dadd_rn(acc[i][j], __dmul_rn(a[i], b[j]));
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = tx + 16 * i, col = ty + 16 * j;
            if (r < M && col < N && r + t.diag >= col)
                Cb[r + (int64_t)col * t.ldc] = running ? c[i][j] : __dsub_rn(c[i][j], acc[i][j]);
        }
}

// FP32 grouped GEMM on the SIMT pipes for the thin (K = 32) updates of the panel steps: 64 x 64 tile,
// 256 threads of 4 x 4 entries, K staged 16 at a time in two shared-memory buffers; mode 0 (C -= A B^T,
// masked to the tile's lower part) and mode 2 (copy) tiles
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, bool valid) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int sz = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}

__global__ void __launch_bounds__(256) gemm_nt_f32_kernel(GemmArgs<float> A) {
    constexpr int BM = 64, BK = 16, LDS = 68;
    __shared__ __align__(16) float As[2][BK][LDS];
    __shared__ __align__(16) float Bs[2][BK][LDS];
    const GemmTile t = A.tiles[blockIdx.x];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    if (A.finfo && t.front >= 0 && A.finfo[(int64_t)member * A.ns + t.front] != 0) return;
    if (t.mode == 2) {   // deferred diagonal-block write
        const float* src = A.copy_src + (int64_t)member * A.copy_stride + t.a;
        float* dst = A.cbuf + (int64_t)member * A.cstride + t.c;
        for (int q = threadIdx.x; q < t.m * t.n; q += blockDim.x) dst[q % t.m + (int64_t)(q / t.m) * t.ldc] = src[q % t.m + (int64_t)(q / t.m) * t.lda];
        return;
    }
    const float* Ab = A.abuf + (int64_t)member * A.astride + t.a;
    const float* Bb = A.bbuf + (int64_t)member * A.bstride + t.b;
    float* Cb = A.cbuf + (int64_t)member * A.cstride + t.c;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int M = t.m, N = t.n, K = t.k;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    auto load = [&](int buf, int k0) {
#pragma unroll
        for (int q = 0; q < (BM * BK) / 256; ++q) {
            int e = tid + 256 * q, r = e % BM, kk = e / BM;
            bool va = r < M && k0 + kk < K;
            cp_async4(&As[buf][kk][r], va ? Ab + r + (int64_t)(k0 + kk) * t.lda : Ab, va);
            bool vb = r < N && k0 + kk < K;
            cp_async4(&Bs[buf][kk][r], vb ? Bb + r + (int64_t)(k0 + kk) * t.ldb : Bb, vb);
        }
        cp_async_commit();
    };
    const int nk = (K + BK - 1) / BK;
    load(0, 0);
    for (int it = 0; it < nk; ++it) {
        const int buf = it & 1;
        if (it + 1 < nk) {
            load(buf ^ 1, (it + 1) * BK);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
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
    // every C load before the first store (see the DMMA kernel's epilogue)
    float cv[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = tx + 16 * i, c = ty + 16 * j;
            cv[i][j] = (r < M && c < N && r + t.diag >= c) ? Cb[r + (int64_t)c * t.ldc] : 0.f;
        }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = tx + 16 * i, c = ty + 16 * j;
            if (r < M && c < N && r + t.diag >= c) Cb[r + (int64_t)c * t.ldc] = cv[i][j] - acc[i][j];
        }
}

template <typename T>
cudaError_t launch_gemm(const GemmArgs<T>& a, int nmembers, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    dim3 grid(a.count, nmembers);
    if constexpr (sizeof(T) == 8) {
        if (a.exact) gemm_nt_exact_kernel<<<grid, 256, 0, st>>>(a);
        else gemm_nt_dmma_kernel<<<grid, 128, 0, st>>>(a);
    } else {
        if (a.simt) gemm_nt_f32_kernel<<<grid, 256, 0, st>>>(a);
        else return launch_gemm_tc32(a, nmembers, st);   // 3xTF32 on tcgen05
    }
    return cudaGetLastError();
}

// One 32-column step of a large Cholesky front, diagonal block and trsm fused: every CTA factors the
// 32 x 32 diagonal block (warp 0) while warps 1..3 stage its own 64-row tile of the rows below; the
// CTA then replaces the tile by X = B L11^{-T}.
// The diagonal block itself is read by every CTA of the step, so no CTA overwrites it: the head task
// puts L11 in the scratch buffer and a copy tile of the next GEMM launch of the level writes it
// into the panel (a diagonal block with no rows below is written directly by its only task).
template <typename T>
__global__ void __launch_bounds__(128) chol_step_kernel(CholStepArgs<T> A) {
    // the arithmetic type is the factor's: FP32 steps compute in float (one 32-bit shuffle per value,
    // single-precision reciprocal square root) instead of rounding double results to float
    using CT = T;
    constexpr int NB = CHOL_NB, LD = NB + 1, TR = 64;
    __shared__ CT L[NB * LD];
    __shared__ CT rdiag[NB];          // reciprocal diagonal of L11 (zero past the block)
    __shared__ CT Bt[TR * LD];
    __shared__ int s_status;
    const CholStepTask task = A.tasks[blockIdx.x];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    const int s = task.front;
    int32_t* finfo = A.finfo + (int64_t)member * A.ns;
    const int f = task.f, w = task.w, kb = A.kb;
    const int nbb = min(NB, w - kb), r1 = kb + nbb;
    T* P = A.factor + (int64_t)member * A.factor_len + task.panel;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row0 = r1 + max(task.tile, 0) * TR;
    const int rows = task.tile >= 0 ? min(TR, f - row0) : 0;
    if (warp == 0) {
        // lane i holds row i of the block in registers; L[j][l] comes from lane j by shuffle, so the
        // dependent path of a column is one shuffle, a short reduction and one reciprocal square root
        const int i = lane;
        CT x[NB];
#pragma unroll
        for (int j = 0; j < NB; ++j)
            x[j] = (i < nbb && j < nbb && j <= i) ? P[(kb + i) + (int64_t)(kb + j) * f] : CT(0);
        const CT eps = (CT)A.eps;
        int status = 0;
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            if (j < nbb && status == 0) {
                CT a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
                for (int l = 0; l < j; ++l) {
                    const CT t = x[l] * __shfl_sync(0xffffffffu, x[l], j);
                    if ((l & 3) == 0) a0 += t;
                    else if ((l & 3) == 1) a1 += t;
                    else if ((l & 3) == 2) a2 += t;
                    else a3 += t;
                }
                const CT sv = x[j] - ((a0 + a1) + (a2 + a3));
                const CT ajj = __shfl_sync(0xffffffffu, sv, j);
                if (!(ajj > eps || (eps > 0 && ajj >= 0))) {
                    status = j + 1;
                } else {
                    const CT d = ajj > eps ? ajj : eps;
                    const CT r = rsqrt(d);
                    if (i == j) {
                        x[j] = d * r;
                        rdiag[j] = r;
                    } else if (i > j && i < nbb) {
                        x[j] = sv * r;
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < NB; ++j) L[i * LD + j] = x[j];
        if (i >= nbb) rdiag[i] = CT(0);   // reciprocal diagonal beyond the block: zero
        if (lane == 0) s_status = status;
    } else {
        batched_copy<8>(tid - 32, 96, TR * NB,
                        [&](int q) {
                            const int r = q % TR, c = q / TR;
                            return (r < rows && c < nbb) ? (double)P[(row0 + r) + (int64_t)(kb + c) * f] : 0.0;
                        },
                        [&](int q, double v) { Bt[(q % TR) * LD + q / TR] = (CT)v; });
    }
    __syncthreads();
    if (finfo[s] != 0) return;   // an earlier step of this front failed
    const int status = s_status;
    const bool head = task.tile <= 0;
    if (head && tid == 0) {
        int64_t* S = A.stats + ((int64_t)member * A.ns + s) * NSTAT;
        if (status) {
            finfo[s] = kb + status;
            S[ST_NPOS] = kb + status - 1;
            S[ST_INFO] = kb + status;
        } else if (kb + nbb == w) {
            S[ST_NPOS] = w;
            S[ST_INFO] = 0;
        }
    }
    if (head) {
        // L11 with zeros above the diagonal: the scratch (copied by the next GEMM launch), or the panel
        // when the block has no rows below it
        T* dst = task.tile < 0 ? P + kb + (int64_t)kb * f : A.scratch + (int64_t)member * A.scr_len + task.scr;
        const int64_t ld = task.tile < 0 ? f : NB;
        for (int q = tid; q < nbb * nbb; q += blockDim.x) {
            const int i = q % nbb, j = q / nbb;
            dst[i + j * ld] = j <= i ? T(L[i * LD + j]) : T(0);
        }
    }
    if (status || rows <= 0) return;
    // X = B L11^{-T}: each of the first 64 threads solves its row, x L11^T = b, by forward
    // substitution with x in registers (fully unrolled; four partial sums per entry); columns past
    // the block have a zero reciprocal diagonal and come out zero
    const int r = tid;
    if (r < rows) {
        CT x[NB];
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            CT a0 = Bt[r * LD + j], a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
            for (int l = 0; l < j; ++l) {
                const CT t = x[l] * L[j * LD + l];
                if ((l & 3) == 0) a0 -= t;
                else if ((l & 3) == 1) a1 -= t;
                else if ((l & 3) == 2) a2 -= t;
                else a3 -= t;
            }
            x[j] = ((a0 + a1) + (a2 + a3)) * rdiag[j];
        }
#pragma unroll
        for (int j = 0; j < NB; ++j)
            if (j < nbb) P[(row0 + r) + (int64_t)(kb + j) * f] = T(x[j]);
    }
}

// ---------------------------------------------------------------------------------------------------
// The Cholesky steps of a batch as dataflow tasks in one persistent launch (kernels.cuh, FlowTask)

__device__ __forceinline__ uint64_t flow_clock() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// bounded wait of one thread until *p >= target (about two seconds, then the status word)
__device__ __noinline__ void flow_wait(const unsigned int* p, unsigned int target, int32_t* status) {
    unsigned int v;
    uint64_t t0 = 0;
    for (long spins = 0;; ++spins) {
        asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
        if (v >= target) break;
        if ((spins & 255) == 0) {
            if (*(volatile int32_t*)status != 0) return;
            const uint64_t now = flow_clock();
            if (spins == 0) t0 = now;
            else if (now - t0 > 2000000000ull) {
                atomicExch(status, 1);
                return;
            }
        }
        if (spins > 4096) __nanosleep(64);
    }
}

__device__ __forceinline__ void flow_add(unsigned int* p) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(p) : "memory");
}

// acc = A B^T over 32 inner columns on DMMA (mma.sync m8n8k4 f64): warp wp's rows 16 wp .. 16 wp + 15 of
// a 64-row A, all 32 rows of B; getA(i, l) and getB(c, l) read the staged operands. Entry (i2, j, e) of
// acc is row 16 wp + 8 i2 + lane / 4, column 8 j + 2 (lane % 4) + e.
template <class GA, class GB>
__device__ __forceinline__ void flow_dmma_64x32(int wp, int lane, double (&acc)[2][4][2], GA getA, GB getB) {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll
    for (int kk = 0; kk < CHOL_NB; kk += 4) {
        double av[2], bv[4];
#pragma unroll
        for (int i = 0; i < 2; ++i) av[i] = getA(16 * wp + 8 * i + (lane >> 2), kk + (lane & 3));
#pragma unroll
        for (int j = 0; j < 4; ++j) bv[j] = getB(8 * j + (lane >> 2), kk + (lane & 3));
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
                asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                             : "+d"(acc[i][j][0]), "+d"(acc[i][j][1])
                             : "d"(av[i]), "d"(bv[j]));
    }
}

// C[i, c] -= sum_l A(i, l) B(c, l) over a 64 x 32 tile of the panel at (r0, c0) (rows < nr, columns < nc,
// row r0 + i >= column c0 + c only), A and B staged in shared memory (getA, getB). FP64 on DMMA; FP32 on
// the SIMT pipes, thread (tx, ty) owning rows tx + 16 q and columns ty + 8 p. Every C load is issued
// before the arithmetic.
template <typename T, class GA, class GB>
__device__ __forceinline__ void flow_tile_update(T* P, int f, int r0, int c0, int nr, int nc, GA getA, GB getB) {
    const int tid = threadIdx.x;
    if constexpr (sizeof(T) == 8) {
        const int wp = tid >> 5, lane = tid & 31;
        double cd[2][4][2], acc[2][4][2];
#pragma unroll
        for (int i2 = 0; i2 < 2; ++i2)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int i = 16 * wp + 8 * i2 + (lane >> 2), c = 8 * j + 2 * (lane & 3) + e;
                    cd[i2][j][e] = (i < nr && c < nc && r0 + i >= c0 + c) ? (double)P[(r0 + i) + (int64_t)(c0 + c) * f] : 0.0;
                }
        flow_dmma_64x32(wp, lane, acc, getA, getB);
#pragma unroll
        for (int i2 = 0; i2 < 2; ++i2)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int i = 16 * wp + 8 * i2 + (lane >> 2), c = 8 * j + 2 * (lane & 3) + e;
                    if (i < nr && c < nc && r0 + i >= c0 + c) P[(r0 + i) + (int64_t)(c0 + c) * f] = T(cd[i2][j][e] - acc[i2][j][e]);
                }
    } else {
        const int tx = tid & 15, ty = tid >> 4;
        T cv[4][4], acc[4][4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                const int i = tx + 16 * q, c = ty + 8 * p;
                acc[q][p] = T(0);
                cv[q][p] = (i < nr && c < nc && r0 + i >= c0 + c) ? P[(r0 + i) + (int64_t)(c0 + c) * f] : T(0);
            }
#pragma unroll 8
        for (int l = 0; l < CHOL_NB; ++l) {
            T ra[4], rb[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) ra[q] = getA(tx + 16 * q, l);
#pragma unroll
            for (int p = 0; p < 4; ++p) rb[p] = getB(ty + 8 * p, l);
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int p = 0; p < 4; ++p) acc[q][p] += ra[q] * rb[p];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                const int i = tx + 16 * q, c = ty + 8 * p;
                if (i < nr && c < nc && r0 + i >= c0 + c) P[(r0 + i) + (int64_t)(c0 + c) * f] = cv[q][p] - acc[q][p];
            }
    }
}

// One UPD task: C[rows b .., columns a ..] -= X[rows] X[block rows]^T over the step's 32 columns kb ..
// (dynamic shared memory: X[rows] then X[block rows], ld 33). Every load of the operands is issued
// before the first store to shared memory.
template <typename T>
__device__ __forceinline__ void flow_update(const CholFlowArgs<T>& A, const FlowTask& t) {
    constexpr int NB = CHOL_NB, TR = 64, LD = NB + 1;
    extern __shared__ __align__(16) unsigned char flow_dsm[];
    T* As = reinterpret_cast<T*>(flow_dsm);   // X[rows]: As[i * LD + l]
    T* Bs = As + TR * LD;                      // X[block rows]: Bs[c * LD + l]
    T* P = A.factor + t.panel;
    const int f = t.f, kb = t.kb, a = t.a, b = t.b;
    const int nr = min(TR, f - b), nc = min(NB, t.w - a);
    const int tid = threadIdx.x;
    T av[(TR * NB) / 128], bv[(NB * NB) / 128];
#pragma unroll
    for (int e = 0; e < (TR * NB) / 128; ++e) {
        const int q = tid + 128 * e, i = q % TR, l = q / TR;
        av[e] = i < nr ? P[(b + i) + (int64_t)(kb + l) * f] : T(0);
    }
#pragma unroll
    for (int e = 0; e < (NB * NB) / 128; ++e) {
        const int q = tid + 128 * e, c = q % NB, l = q / NB;
        bv[e] = c < nc ? P[(a + c) + (int64_t)(kb + l) * f] : T(0);
    }
#pragma unroll
    for (int e = 0; e < (TR * NB) / 128; ++e) {
        const int q = tid + 128 * e;
        As[(q % TR) * LD + q / TR] = av[e];
    }
#pragma unroll
    for (int e = 0; e < (NB * NB) / 128; ++e) {
        const int q = tid + 128 * e;
        Bs[(q % NB) * LD + q / NB] = bv[e];
    }
    __syncthreads();
    flow_tile_update<T>(P, f, b, a, nr, nc, [&](int i, int l) { return As[i * LD + l]; },
                        [&](int c, int l) { return Bs[c * LD + l]; });
}

// One STEP or STEPN task: step kb of front t.front (a block of nbb <= 32 columns) for its row tile t.a
// (rows r1 + 64 t.a .., r1 = kb + nbb; t.a < 0: no rows below the block), as chol_step_kernel: warp 0
// factors the diagonal block in registers while warps 1-3 stage the tile, whose rows are then
// forward-substituted. STEPN then applies the step's update of the next column block (columns
// kn = kb + 32 ..) to those rows: C[rows, kn ..] -= X[rows] X[kn .. kn + 31]^T (row >= column); the next
// block's rows are tile 0's first rows.
template <typename T>
__device__ __forceinline__ void flow_step(const CholFlowArgs<T>& A, const FlowTask& t) {
    using CT = T;
    constexpr int NB = CHOL_NB, LD = NB + 1, TR = 64;
    __shared__ CT L[NB * LD];
    __shared__ CT rdiag[NB];          // reciprocal diagonal of L11 (zero past the block)
    __shared__ CT Bt[TR * LD];        // the tile's rows: B, then X
    __shared__ CT Ct[NB * LD];        // the next block's rows X (STEPN, tile > 0)
    __shared__ int s_status, s_ok;
    const bool next = t.kind == FLOW_STEPN;
    const int s = t.front, f = t.f, w = t.w, kb = t.kb, tile = t.a;
    const int nbb = min(NB, w - kb), r1 = kb + nbb, kn = kb + NB, nbn = next ? min(NB, w - kn) : 0;
    const int row0 = r1 + max(tile, 0) * TR, rows = tile >= 0 ? min(TR, f - row0) : 0;
    T* P = A.factor + t.panel;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        const int i = lane;
        CT x[NB];
#pragma unroll
        for (int j = 0; j < NB; ++j) x[j] = (i < nbb && j < nbb && j <= i) ? P[(kb + i) + (int64_t)(kb + j) * f] : CT(0);
        const CT eps = (CT)A.eps;
        int status = 0;
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            if (j < nbb && status == 0) {
                CT a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
                for (int l = 0; l < j; ++l) {
                    const CT v = x[l] * __shfl_sync(0xffffffffu, x[l], j);
                    if ((l & 3) == 0) a0 += v;
                    else if ((l & 3) == 1) a1 += v;
                    else if ((l & 3) == 2) a2 += v;
                    else a3 += v;
                }
                const CT sv = x[j] - ((a0 + a1) + (a2 + a3));
                const CT ajj = __shfl_sync(0xffffffffu, sv, j);
                if (!(ajj > eps || (eps > 0 && ajj >= 0))) {
                    status = j + 1;
                } else {
                    const CT d = ajj > eps ? ajj : eps;
                    const CT r = rsqrt(d);
                    if (i == j) {
                        x[j] = d * r;
                        rdiag[j] = r;
                    } else if (i > j && i < nbb) {
                        x[j] = sv * r;
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < NB; ++j) L[i * LD + j] = x[j];
        if (i >= nbb) rdiag[i] = CT(0);
        if (lane == 0) s_status = status;
    } else {
        batched_copy<8>(tid - 32, 96, TR * NB,
                        [&](int q) {
                            const int r = q % TR, c = q / TR;
                            return (r < rows && c < nbb) ? (double)P[(row0 + r) + (int64_t)(kb + c) * f] : 0.0;
                        },
                        [&](int q, double v) { Bt[(q % TR) * LD + q / TR] = (CT)v; });
    }
    __syncthreads();
    const int status = s_status;
    if (tid == 0) {
        const bool alive = A.finfo[s] == 0;   // no earlier step of the front failed
        s_ok = alive && status == 0;
        if (alive && tile <= 0) {
            int64_t* S = A.stats + (int64_t)s * NSTAT;
            if (status) {
                A.finfo[s] = kb + status;
                S[ST_NPOS] = kb + status - 1;
                S[ST_INFO] = kb + status;
            } else if (kb + nbb == w) {
                S[ST_NPOS] = w;
                S[ST_INFO] = 0;
            }
        }
    }
    __syncthreads();
    const bool ok = s_ok != 0;
    if (ok && tile <= 0) {
        // L11 with zeros above the diagonal: the scratch (the COPY task writes it into the panel), or the
        // panel when no rows are below the block
        T* dst = tile < 0 ? P + kb + (int64_t)kb * f : A.scratch + t.scr;
        const int64_t ld = tile < 0 ? f : NB;
        for (int q = tid; q < nbb * nbb; q += blockDim.x) {
            const int i = q % nbb, j = q / nbb;
            dst[i + j * ld] = j <= i ? T(L[i * LD + j]) : T(0);
        }
    }
    // X = B L11^{-T}, threads < rows, into the panel and kept in Bt; columns past the block have a zero
    // reciprocal diagonal
    if (ok && tid < rows) {
        const int r = tid;
        CT x[NB];
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            CT a0 = Bt[r * LD + j], a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
            for (int l = 0; l < j; ++l) {
                const CT v = x[l] * L[j * LD + l];
                if ((l & 3) == 0) a0 -= v;
                else if ((l & 3) == 1) a1 -= v;
                else if ((l & 3) == 2) a2 -= v;
                else a3 -= v;
            }
            x[j] = ((a0 + a1) + (a2 + a3)) * rdiag[j];
        }
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            Bt[r * LD + j] = x[j];
            if (j < nbb) P[(row0 + r) + (int64_t)(kb + j) * f] = T(x[j]);
        }
    }
    if (!next) return;
    __syncthreads();
    if (tid == 0) {
        if (t.sig_mid >= 0) flow_add(A.cnt + t.sig_mid);
        if (t.sig_head >= 0) flow_add(A.cnt + t.sig_head);
        if (t.w_mid >= 0) flow_wait(A.cnt + t.w_mid, 1u, A.status);
        if (t.w2 >= 0) flow_wait(A.cnt + t.w2, (unsigned)t.v2, A.status);
    }
    __syncthreads();
    if (!ok) return;
    if (tile > 0) {   // the next block's rows, solved by tile 0
        for (int q = tid; q < NB * NB; q += blockDim.x) {
            const int r = q % NB, c = q / NB;
            Ct[r * LD + c] = r < nbn ? P[(kn + r) + (int64_t)(kb + c) * f] : CT(0);
        }
        __syncthreads();
    }
    const CT* Xn = tile > 0 ? Ct : Bt;
    flow_tile_update<T>(P, f, row0, kn, rows, nbn, [&](int i, int l) { return Bt[i * LD + l]; },
                        [&](int c, int l) { return Xn[c * LD + l]; });
}

template <typename T>
__global__ void __launch_bounds__(128) chol_flow_kernel(CholFlowArgs<T> A) {
    __shared__ int task_k;
    const int tid = threadIdx.x;
    while (true) {
        if (tid == 0) {
            task_k = (int)atomicAdd(A.cnt + A.ncnt, 1u);
            if (*(volatile int32_t*)A.status != 0) task_k = A.ntasks;   // a wait gave up: stop
        }
        __syncthreads();
        const int k = task_k;
        if (k >= A.ntasks) break;
        const FlowTask t = A.tasks[k];
        if (tid == 0) {
            if (A.trace) {
                A.trace[4 * k] = (int64_t)flow_clock();
                A.trace[4 * k + 3] = (int64_t)blockIdx.x | ((int64_t)t.kind << 12) | ((int64_t)(t.kb / CHOL_NB) << 16) |
                                     ((int64_t)(t.kind == FLOW_UPD ? t.a / CHOL_NB : 0) << 28) | ((int64_t)t.front << 40);
            }
            if (t.w1 >= 0) flow_wait(A.cnt + t.w1, (unsigned)t.v1, A.status);
            if (t.w2 >= 0 && t.kind != FLOW_STEPN) flow_wait(A.cnt + t.w2, (unsigned)t.v2, A.status);
            if (A.trace) A.trace[4 * k + 1] = (int64_t)flow_clock();
        }
        __syncthreads();
        if (t.kind == FLOW_STEP || t.kind == FLOW_STEPN) {
            flow_step<T>(A, t);
        } else if (t.kind == FLOW_COPY) {
            const int nbb = min(CHOL_NB, t.w - t.kb);
            const T* src = A.scratch + t.scr;
            T* dst = A.factor + t.panel + t.kb + (int64_t)t.kb * t.f;
            for (int q = tid; q < nbb * nbb; q += blockDim.x)
                dst[q % nbb + (int64_t)(q / nbb) * t.f] = src[q % nbb + (q / nbb) * CHOL_NB];
        } else if (t.kind == FLOW_UPD) {
            if (A.finfo[t.front] == 0) flow_update<T>(A, t);
        }
        __syncthreads();
        if (tid == 0) {
            if (A.trace) A.trace[4 * k + 2] = (int64_t)flow_clock();
            if (t.sig_add >= 0) flow_add(A.cnt + t.sig_add);
            if (t.sig_store >= 0)
                asm volatile("st.release.gpu.u32 [%0], %1;" ::"l"(A.cnt + t.sig_store), "r"((unsigned)t.sig_val) : "memory");
        }
    }
}

template <typename T>
constexpr size_t chol_flow_smem() {
    return sizeof(T) * (64 + CHOL_NB) * (CHOL_NB + 1);
}

template <typename T>
cudaError_t launch_chol_flow(const CholFlowArgs<T>& a, cudaStream_t st) {
    if (a.ntasks == 0) return cudaSuccess;
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, chol_flow_kernel<T>, 128, chol_flow_smem<T>());
    const int grid = std::max(1, std::min(a.ntasks, sms * std::max(per, 1)));
    chol_flow_kernel<T><<<grid, 128, chol_flow_smem<T>(), st>>>(a);
    return cudaGetLastError();
}

template cudaError_t launch_chol_flow<double>(const CholFlowArgs<double>&, cudaStream_t);
template cudaError_t launch_chol_flow<float>(const CholFlowArgs<float>&, cudaStream_t);

template <typename T>
cudaError_t launch_chol_step(const CholStepArgs<T>& a, int nmembers, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    dim3 grid(a.count, nmembers);
    chol_step_kernel<T><<<grid, 128, 0, st>>>(a);
    return cudaGetLastError();
}

template cudaError_t launch_chol_step<double>(const CholStepArgs<double>&, int, cudaStream_t);
template cudaError_t launch_chol_step<float>(const CholStepArgs<float>&, int, cudaStream_t);

// Inverse of a lower-triangular N x N matrix (N <= 32) held by the warp: lane c computes column c by
// forward substitution, x_k = (delta_kc - sum_{j<k} L[k, j] x_j) r_k, with the reciprocals
// r_k = 1 / L[k, k] taken up front (off the substitution's dependency chain). L(k, j) reads entry (k, j)
// (k, j < N).
template <int N, class Get>
__device__ __forceinline__ void warp_tri_inv(Get L, int lane, double (&x)[N]) {
    double rd[N];
#pragma unroll
    for (int k = 0; k < N; ++k) rd[k] = 1.0 / L(k, k);
#pragma unroll
    for (int k = 0; k < N; ++k) {
        double acc = (k == lane) ? 1.0 : 0.0;
#pragma unroll
        for (int j = 0; j < k; ++j) acc -= L(k, j) * x[j];
        x[k] = acc * rd[k];
    }
}

// Inverse of one 64 x 64 diagonal block of a panel (lower triangle as stored; unit or not). Warps 0 and
// 1 invert the two 32 x 32 diagonal sub-blocks X11 and X22 (a partial block is padded with the
// identity), then X21 = -X22 (L21 X11) in two 32 x 32 products over the four warps. One shared array:
// L, then X in place (X11 and X22 over L11 and L22, X21 over L21 once T = L21 X11 is formed in the
// unused upper right quarter).
template <typename T>
__global__ void __launch_bounds__(128) block_inv_kernel(BlockInvArgs<T> A) {
    constexpr int NB = 64, LD = NB + 1;
    __shared__ double S[NB * LD];        // (i, j) at i + j LD
    const int s = A.tasks[2 * blockIdx.x], b = A.tasks[2 * blockIdx.x + 1];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    if (A.finfo && A.finfo[(int64_t)member * A.ns + s] != 0) return;
    const DFront fd = A.fronts[s];
    const int f = fd.f, jb = b * NB, nbb = min(NB, fd.w - jb);
    const T* P = A.panels + (int64_t)member * A.factor_len + fd.panel;
    const int ldo = A.panel_layout ? f : NB;
    T* inv = A.dinv + (int64_t)member * A.dinv_len + A.dinv_off[s] +
             (A.panel_layout ? (int64_t)jb * (1 + f) : (int64_t)b * NB * NB);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int q = tid; q < NB * NB; q += blockDim.x) {
        const int i = q % NB, j = q / NB;
        double v = 0.0;
        if (i < nbb && j < nbb) {
            if (i >= j) v = (double)P[(jb + i) + (int64_t)(jb + j) * f];
        } else if (i == j) {
            v = 1.0;
        }
        S[i + j * LD] = v;
    }
    __syncthreads();
    if (warp < 2) {
        const int o = 32 * warp;
        double x[32];
        warp_tri_inv<32>([&](int k, int j) { return S[(o + k) + (o + j) * LD]; }, lane, x);
        __syncwarp();
#pragma unroll
        for (int k = 0; k < 32; ++k) S[(o + k) + (o + lane) * LD] = k >= lane ? x[k] : 0.0;
    }
    __syncthreads();
    const int c = tid & 31, r0 = 8 * (tid >> 5);
    // T = L21 X11 into the upper right quarter: thread (c, rows r0 ..); X11 is lower triangular (j >= c)
#pragma unroll
    for (int rr = 0; rr < 8; ++rr) {
        const int r = r0 + rr;
        double acc = 0.0;
        for (int j = c; j < 32; ++j) acc += S[(32 + r) + j * LD] * S[j + c * LD];
        S[r + (32 + c) * LD] = acc;
    }
    __syncthreads();
    // X21 = -X22 T over L21; X22 is lower triangular (j <= r)
    double x21[8];
#pragma unroll
    for (int rr = 0; rr < 8; ++rr) {
        const int r = r0 + rr;
        double acc = 0.0;
        for (int j = 0; j <= r; ++j) acc += S[(32 + r) + (32 + j) * LD] * S[j + (32 + c) * LD];
        x21[rr] = -acc;
    }
    __syncthreads();
#pragma unroll
    for (int rr = 0; rr < 8; ++rr) {
        S[(32 + r0 + rr) + c * LD] = x21[rr];
        S[(r0 + rr) + (32 + c) * LD] = 0.0;
    }
    __syncthreads();
    for (int q = tid; q < NB * NB; q += blockDim.x) {
        const int i = q % NB, j = q / NB;
        if (A.panel_layout) {
            if (i < nbb && j < nbb) inv[i + (int64_t)j * ldo] = T(i >= j ? S[i + j * LD] : 0.0);
        } else {
            inv[i + (int64_t)j * ldo] = T((i >= j && i < nbb && j < nbb) ? S[i + j * LD] : 0.0);
        }
    }
}

// L11^-1 of a warp front of the dataflow solve (w <= N <= 32; unit or not, as stored), one warp per
// front, padded with the identity past w. Instances for N = 8, 16 and 32: the narrow ones hold a
// fraction of the registers, so many more warps are resident (batches of small systems have hundreds
// of thousands of such fronts).
template <typename T, int N>
__global__ void __launch_bounds__(256) small_inv_kernel(SmallInvArgs<T> A) {
    const int wi = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (wi >= A.count) return;
    const int s = A.list[wi];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    if (A.finfo && A.finfo[(int64_t)member * A.ns + s] != 0) return;
    const DFront fd = A.fronts[s];
    const int f = fd.f, w = fd.w;
    const T* P = A.panels + (int64_t)member * A.factor_len + fd.panel;
    T* inv = A.inv + (int64_t)member * A.inv_len + A.inv_off[s];
    double x[N];
    warp_tri_inv<N>([&](int k, int j) { return k < w ? (double)P[k + (int64_t)j * f] : (k == j ? 1.0 : 0.0); }, lane, x);
    if (lane < w) {
#pragma unroll
        for (int k = 0; k < N; ++k)
            if (k < w) inv[k + (int64_t)w * lane] = T(k >= lane ? x[k] : 0.0);
    }
}

template <typename T>
cudaError_t launch_small_inv(const SmallInvArgs<T>& a, int nmembers, int wmax, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    dim3 grid((a.count + 7) / 8, nmembers);
    if (wmax > 0 && wmax <= 8) small_inv_kernel<T, 8><<<grid, 256, 0, st>>>(a);
    else if (wmax > 0 && wmax <= 16) small_inv_kernel<T, 16><<<grid, 256, 0, st>>>(a);
    else small_inv_kernel<T, 32><<<grid, 256, 0, st>>>(a);
    return cudaGetLastError();
}

template cudaError_t launch_small_inv<double>(const SmallInvArgs<double>&, int, int, cudaStream_t);
template cudaError_t launch_small_inv<float>(const SmallInvArgs<float>&, int, int, cudaStream_t);

template <typename T>
cudaError_t launch_block_inv(const BlockInvArgs<T>& a, int nmembers, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    dim3 grid(a.count, nmembers);
    block_inv_kernel<T><<<grid, 128, 0, st>>>(a);
    return cudaGetLastError();
}

template cudaError_t launch_block_inv<double>(const BlockInvArgs<double>&, int, cudaStream_t);
template cudaError_t launch_block_inv<float>(const BlockInvArgs<float>&, int, cudaStream_t);

cudaError_t prepare_dense_kernels(int max_smem) {
    (void)max_smem;   // static shared memory, but for the flow kernel's update stage
    cudaError_t e = cudaFuncSetAttribute(chol_flow_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)chol_flow_smem<double>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(chol_flow_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)chol_flow_smem<float>());
    return e;
}

template cudaError_t launch_gemm<double>(const GemmArgs<double>&, int, cudaStream_t);
template cudaError_t launch_gemm<float>(const GemmArgs<float>&, int, cudaStream_t);


// W = L21 D (1x1 and 2x2 blocks of D), rows w..f-1 of the panel, into work (m x w, ld m)
template <typename T, int STRUCT>
__global__ void scale_ld_kernel(ScaleArgs<T> A) {
    const int s = A.list[blockIdx.x];
    const int member = A.members ? A.members[blockIdx.z] : blockIdx.z;
    const DFront fd = A.fronts[s];
    const int f = fd.f, w = fd.w, m = f - w;
    const int q = blockIdx.y;  // column
    if (q >= w) return;
    const T* P = A.factor + (int64_t)member * A.factor_len + fd.panel;
    const double* d = A.d + (int64_t)member * 2 * A.n;
    const int8_t* kd = A.kind + (int64_t)member * A.n;
    T* W = A.work + (int64_t)member * A.work_len + A.woff[blockIdx.x];
    const int g = fd.c0 + q;
    const int kq = kd[g];
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        double v;
        double x = (double)P[w + i + (int64_t)q * f];
        // each product and the sum rounded on its own, as the oracle's W (ldlt.jl:184-189)
        if (STRUCT == STRUCT_S && kq == KIND_2X2_FIRST) {
            double x2 = (double)P[w + i + (int64_t)(q + 1) * f];
            v = __dadd_rn(__dmul_rn(x, d[g]), __dmul_rn(x2, d[A.n + g]));
        } else if (STRUCT == STRUCT_S && kq == KIND_2X2_SECOND) {
            double x1 = (double)P[w + i + (int64_t)(q - 1) * f];
            v = __dadd_rn(__dmul_rn(x1, d[A.n + g - 1]), __dmul_rn(x, d[g]));
        } else {
            v = __dmul_rn(x, d[g]);
        }
        W[i + (int64_t)q * m] = T(v);
    }
}

template <typename T>
cudaError_t launch_scale_ld_front(int structure, const ScaleArgs<T>& a, int maxw, int nmembers, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    dim3 grid(a.count, maxw, nmembers);
    if (structure == STRUCT_S) scale_ld_kernel<T, STRUCT_S><<<grid, 128, 0, st>>>(a);
    else scale_ld_kernel<T, STRUCT_G><<<grid, 128, 0, st>>>(a);
    return cudaGetLastError();
}

template cudaError_t launch_scale_ld_front<double>(int, const ScaleArgs<double>&, int, int, cudaStream_t);
template cudaError_t launch_scale_ld_front<float>(int, const ScaleArgs<float>&, int, int, cudaStream_t);

}  // namespace sds

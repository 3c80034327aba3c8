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
// * large_pivot_kernel / large_pivot_coop_kernel: LDLT / LU fronts beyond shared memory, the
//   reference's in-front steps (front_factor.cuh) on the global panels, by one CTA or by a group of
//   co-resident CTAs.
// * scale_ld_kernel: W = L21 D for the contribution-block update of those fronts.
#include <cuda_runtime.h>
#include <math.h>
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

template <typename T>
cudaError_t launch_gemm(const GemmArgs<T>& a, int nmembers, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    dim3 grid(a.count, nmembers);
    if constexpr (sizeof(T) == 8) {
        gemm_nt_dmma_kernel<<<grid, 128, 0, st>>>(a);
    } else {
        return launch_gemm_tc32(a, nmembers, st);   // 3xTF32 on tcgen05
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
    constexpr int NB = CHOL_NB, LD = NB + 1, TR = 64;
    __shared__ double L[NB * LD];
    __shared__ double rdiag[NB];          // reciprocal diagonal of L11 (zero past the block)
    __shared__ double Bt[TR * LD];
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
        double x[NB];
#pragma unroll
        for (int j = 0; j < NB; ++j)
            x[j] = (i < nbb && j < nbb && j <= i) ? (double)P[(kb + i) + (int64_t)(kb + j) * f] : 0.0;
        const double eps = A.eps;
        int status = 0;
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            if (j < nbb && status == 0) {
                double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
                for (int l = 0; l < j; ++l) {
                    const double t = x[l] * __shfl_sync(0xffffffffu, x[l], j);
                    if ((l & 3) == 0) a0 += t;
                    else if ((l & 3) == 1) a1 += t;
                    else if ((l & 3) == 2) a2 += t;
                    else a3 += t;
                }
                const double sv = x[j] - ((a0 + a1) + (a2 + a3));
                const double ajj = __shfl_sync(0xffffffffu, sv, j);
                if (!(ajj > eps || (eps > 0 && ajj >= 0))) {
                    status = j + 1;
                } else {
                    const double r = rsqrt(fmax(ajj, eps));
                    if (i == j) {
                        x[j] = (double)T(fmax(ajj, eps) * r);
                        rdiag[j] = r;
                    } else if (i > j && i < nbb) {
                        x[j] = (double)T(sv * r);
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < NB; ++j) L[i * LD + j] = x[j];
        if (i >= nbb) rdiag[i] = 0.0;   // reciprocal diagonal beyond the block: zero
        if (lane == 0) s_status = status;
    } else {
        batched_copy<8>(tid - 32, 96, TR * NB,
                        [&](int q) {
                            const int r = q % TR, c = q / TR;
                            return (r < rows && c < nbb) ? (double)P[(row0 + r) + (int64_t)(kb + c) * f] : 0.0;
                        },
                        [&](int q, double v) { Bt[(q % TR) * LD + q / TR] = v; });
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
        double x[NB];
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            double a0 = Bt[r * LD + j], a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
            for (int l = 0; l < j; ++l) {
                const double t = x[l] * L[j * LD + l];
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

template <typename T>
cudaError_t launch_chol_step(const CholStepArgs<T>& a, int nmembers, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    dim3 grid(a.count, nmembers);
    chol_step_kernel<T><<<grid, 128, 0, st>>>(a);
    return cudaGetLastError();
}

template cudaError_t launch_chol_step<double>(const CholStepArgs<double>&, int, cudaStream_t);
template cudaError_t launch_chol_step<float>(const CholStepArgs<float>&, int, cudaStream_t);

// inverse of one 64 x 64 diagonal block of a panel (lower triangle as stored; unit or not), with the
// register-owned right-looking substitution
template <typename T>
__global__ void __launch_bounds__(256) block_inv_kernel(BlockInvArgs<T> A) {
    constexpr int NB = 64, NE = NB * (NB + 1) / 2, SLOTS = (NE + 255) / 256;
    __shared__ double colv[2][NB];
    __shared__ double rowv[2][NB];
    const int s = A.tasks[2 * blockIdx.x], b = A.tasks[2 * blockIdx.x + 1];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    if (A.finfo && A.finfo[(int64_t)member * A.ns + s] != 0) return;
    const DFront fd = A.fronts[s];
    const int f = fd.f, jb = b * NB, nbb = min(NB, fd.w - jb);
    const T* P = A.panels + (int64_t)member * A.factor_len + fd.panel;
    T* inv = A.dinv + (int64_t)member * A.dinv_len + A.dinv_off[s] + (int64_t)b * NB * NB;
    const int tid = threadIdx.x;
    int ri[SLOTS], ci[SLOTS];
    double a[SLOTS], x[SLOTS];
#pragma unroll
    for (int k = 0; k < SLOTS; ++k) {
        int e = tid + 256 * k, col = 0;
        if (e < NE) {
            int rem = e;
            while (rem >= NB - col) { rem -= NB - col; ++col; }
            ri[k] = col + rem;
            ci[k] = col;
        } else {
            ri[k] = -1;
            ci[k] = NB;
        }
        const bool in = ri[k] >= 0 && ri[k] < nbb && ci[k] < nbb;
        a[k] = in ? (double)P[(jb + ri[k]) + (int64_t)(jb + ci[k]) * f] : 0.0;
        x[k] = (in && ri[k] == ci[k]) ? 1.0 : 0.0;
    }
    for (int l = 0; l < nbb; ++l) {
        double* cv = colv[l & 1];
        double* rv = rowv[l & 1];
#pragma unroll
        for (int k = 0; k < SLOTS; ++k)
            if (ci[k] == l) cv[ri[k]] = a[k];
        __syncthreads();
        const double rl = 1.0 / cv[l];
#pragma unroll
        for (int k = 0; k < SLOTS; ++k)
            if (ri[k] == l) {
                x[k] *= rl;
                rv[ci[k]] = x[k];
            }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < SLOTS; ++k)
            if (ri[k] > l && ri[k] < nbb && ci[k] <= l) x[k] -= cv[ri[k]] * rv[ci[k]];
    }
    for (int q = tid; q < NB * NB; q += 256) {
        int i = q % NB, j = q / NB;
        if (i < j || i >= nbb) inv[i + (int64_t)j * NB] = T(0);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < SLOTS; ++k)
        if (ri[k] >= 0 && ri[k] < nbb && ci[k] < nbb) inv[ri[k] + (int64_t)ci[k] * NB] = T(x[k]);
}

template <typename T>
cudaError_t launch_block_inv(const BlockInvArgs<T>& a, int nmembers, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    dim3 grid(a.count, nmembers);
    block_inv_kernel<T><<<grid, 256, 0, st>>>(a);
    return cudaGetLastError();
}

template cudaError_t launch_block_inv<double>(const BlockInvArgs<double>&, int, cudaStream_t);
template cudaError_t launch_block_inv<float>(const BlockInvArgs<float>&, int, cudaStream_t);

cudaError_t prepare_dense_kernels(int max_smem) {
    (void)max_smem;   // the dense kernels use static shared memory only
    return cudaSuccess;
}

template cudaError_t launch_gemm<double>(const GemmArgs<double>&, int, cudaStream_t);
template cudaError_t launch_gemm<float>(const GemmArgs<float>&, int, cudaStream_t);

// ---------------------------------------------------------------------------
template <typename T, int STRUCT>
__global__ void __launch_bounds__(1024) large_pivot_kernel(LargePivotArgs<T> A) {
    const int s = A.list[blockIdx.x];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    const DFront fd = A.fronts[s];
    const int f = fd.f, w = fd.w;
    constexpr bool GEN = STRUCT == STRUCT_G;
    T* P = A.factor + (int64_t)member * A.factor_len + fd.panel;
    T* U = GEN ? A.ufactor + (int64_t)member * A.factor_len + fd.panel : nullptr;
    double* scr = A.scratch + (int64_t)member * A.scr_len + A.scr_off[blockIdx.x];
    FrontScratch sc;
    sc.lvec = scr;
    sc.dd = scr + 2 * f;
    sc.ee = sc.dd + w;
    sc.lp = reinterpret_cast<int*>(sc.ee + w);
    sc.ctl = sc.lp + w;
    sc.kd = reinterpret_cast<signed char*>(sc.ctl + 16);
    const int tid = threadIdx.x, nt = blockDim.x;
    if (STRUCT == STRUCT_S) {
        for (int q = tid; q < w * w; q += nt) {
            int i = q % w, j = q / w;
            if (i > j) P[j + (int64_t)i * f] = P[i + (int64_t)j * f];
        }
        __syncthreads();
    }
    int64_t st[NSTAT] = {0, 0, 0, 0, 0, 0};
    GlobalStore<T, GEN> store{P, U, f, w};
    if (STRUCT == STRUCT_S)
        ldlt_front_steps<T>(store, sc, f, w, A.pivot, A.u, A.eps, A.psign, A.perm, fd.c0, st);
    else
        lu_front_steps<T>(store, sc, f, w, A.lu_pivot != 0, A.u, A.eps, st);
    __syncthreads();
    // unit diagonals, zero strict upper part of the diagonal block (LDLT used it as workspace)
    for (int q = tid; q < w * w; q += nt) {
        int i = q % w, j = q / w;
        if (i == j) {
            P[i + (int64_t)j * f] = T(1);
            if (GEN) U[i + (int64_t)j * f] = T(1);
        } else if (i < j && !GEN) {
            P[i + (int64_t)j * f] = T(0);
        }
    }
    const int64_t n = A.n;
    for (int q = tid; q < w; q += nt) {
        const int64_t g = fd.c0 + q;
        A.piv[member * n + g] = fd.c0 + sc.lp[q] + 1;
        A.kind[member * n + g] = sc.kd[q];
        A.d[member * 2 * n + g] = sc.dd[q];
        A.d[member * 2 * n + n + g] = STRUCT == STRUCT_S ? sc.ee[q] : 0.0;
    }
    if (tid == 0) {
        int64_t* S = A.stats + ((int64_t)member * A.ns + s) * NSTAT;
        for (int q = 0; q < NSTAT; ++q) S[q] = st[q];
        A.finfo[(int64_t)member * A.ns + s] = (int32_t)st[ST_INFO];
    }
}

template <typename T>
cudaError_t launch_large_pivot(int structure, const LargePivotArgs<T>& a, int nmembers, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    dim3 grid(a.count, nmembers);
    if (structure == STRUCT_S) large_pivot_kernel<T, STRUCT_S><<<grid, 1024, 0, st>>>(a);
    else large_pivot_kernel<T, STRUCT_G><<<grid, 1024, 0, st>>>(a);
    return cudaGetLastError();
}

template cudaError_t launch_large_pivot<double>(int, const LargePivotArgs<double>&, int, cudaStream_t);
template cudaError_t launch_large_pivot<float>(int, const LargePivotArgs<float>&, int, cudaStream_t);

// ---------------------------------------------------------------------------
// Cooperative variant of large_pivot_kernel for wide fronts of a single-member plan: each listed
// front gets a group of co-resident CTAs (cta_first: prefix of the group sizes), and every pivot step
// of ldlt_front_steps / lu_front_steps runs as phases separated by group barriers:
// decision (one warp) | column / row interchanges | multipliers | rank-1 or rank-2 update.
// Each entry receives the same floating-point operations in the same order as in the one-CTA
// kernel, so pivots, D and the panels are identical; only the update is spread over the group.
// A group barrier waits at most ~2 s, then records a nonzero status and goes on (no hang).
__device__ __forceinline__ void group_barrier(unsigned int* bar, unsigned int& epoch, int gs, int32_t* status) {
    __syncthreads();
    epoch += gs;
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
        unsigned int v;
        long spins = 0;
        while (true) {
            asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(bar));
            if ((int)(v - epoch) >= 0) break;
            if (++spins > (1L << 26)) {
                atomicExch(status, 1);
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
    }
    __syncthreads();
}

constexpr int COOP_ROWS = 256;   // rows of one update item (a column chunk, one warp)

template <typename T, int STRUCT>
__global__ void __launch_bounds__(COOP_THREADS) large_pivot_coop_kernel(LargePivotArgs<T> A, CoopGroups G) {
    int lo = 0, hi = A.count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (G.cta_first[mid] <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const int fi = lo, rank = (int)blockIdx.x - G.cta_first[fi], gs = G.cta_first[fi + 1] - G.cta_first[fi];
    const int s = A.list[fi];
    const DFront fd = A.fronts[s];
    const int f = fd.f, w = fd.w;
    constexpr bool GEN = STRUCT == STRUCT_G;
    T* P = A.factor + fd.panel;
    T* U = GEN ? A.ufactor + fd.panel : nullptr;
    double* scr = A.scratch + A.scr_off[fi];
    FrontScratch sc;
    sc.lvec = scr;
    sc.dd = scr + 2 * f;
    sc.ee = sc.dd + w;
    sc.lp = reinterpret_cast<int*>(sc.ee + w);
    sc.ctl = sc.lp + w;
    sc.kd = reinterpret_cast<signed char*>(sc.ctl + 16);
    unsigned int* bar = G.bar + fi;
    unsigned int epoch = 0;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    const int gt = rank * nt + tid, GT = gs * nt, gw = gt >> 5, GW = GT >> 5;
    const bool lead = rank == 0 && tid == 0;
    GlobalStore<T, GEN> F{P, U, f, w};
    __shared__ double team_red[COOP_THREADS / 32];
    __shared__ int team_redi[COOP_THREADS / 32];
    const CtaTeam team{tid, nt, team_red, team_redi};
    if (STRUCT == STRUCT_S) {
        for (int q = gt; q < w * w; q += GT) {
            const int i = q % w, j = q / w;
            if (i > j) P[j + (int64_t)i * f] = P[i + (int64_t)j * f];
        }
    }
    for (int q = gt; q < w; q += GT) sc.lp[q] = q;
    group_barrier(bar, epoch, gs, G.status);
    int64_t st[NSTAT] = {0, 0, 0, 0, 0, 0};
    if (STRUCT == STRUCT_S) {
        int k = 0;
        while (k < w) {
            if (rank == 0) {   // the whole first CTA takes the decision (row scans split over its threads)
                int c, r;
                choose_pivot(F, k, w, A.pivot, A.u, A.eps, team, c, r);
                if (tid == 0) { sc.ctl[0] = c; sc.ctl[1] = r; }
            }
            group_barrier(bar, epoch, gs, G.status);
            const int c = sc.ctl[0], r = sc.ctl[1];
            const int p = r < 0 ? k : k + 1, qsw = r < 0 ? c : r;
            if (p != qsw) {
                for (int i = gt; i < f; i += GT) {
                    T t = F.at(i, p); F.at(i, p) = F.at(i, qsw); F.at(i, qsw) = t;
                }
                group_barrier(bar, epoch, gs, G.status);
                for (int j = gt; j < w; j += GT) {
                    T t = F.at(p, j); F.at(p, j) = F.at(qsw, j); F.at(qsw, j) = t;
                }
                if (lead) { int t = sc.lp[p]; sc.lp[p] = sc.lp[qsw]; sc.lp[qsw] = t; }
                group_barrier(bar, epoch, gs, G.status);
            }
            const int nch = (f - k - 1 + COOP_ROWS - 1) / COOP_ROWS;
            if (r < 0) {
                double dk = F.get(k, k);
                signed char kk = KIND_1X1;
                if (!(fabs(dk) >= A.eps) || dk == 0.0) {
                    if (dk == 0.0) st[ST_NZERO]++;
                    int req = A.psign ? (int)A.psign[A.perm[fd.c0 + sc.lp[k]]] : 0;
                    dk = perturb_sign_of(dk, req) * A.eps;
                    kk = KIND_PERTURBED;
                    st[ST_NPERT]++;
                    if (dk == 0.0 && st[ST_INFO] == 0) st[ST_INFO] = sc.lp[k] + 1;
                }
                if (dk > 0) st[ST_NPOS]++;
                else if (dk < 0) st[ST_NNEG]++;
                for (int i = k + 1 + gt; i < f; i += GT) sc.lvec[i] = F.get(i, k) / dk;
                group_barrier(bar, epoch, gs, G.status);
                if (lead) { F.at(k, k) = T(dk); sc.dd[k] = dk; sc.ee[k] = 0.0; sc.kd[k] = kk; }
                const int nj = w - k - 1;
                for (int item = gw; item < nj * nch; item += GW) {
                    const int j = k + 1 + item % nj, ch = item / nj;
                    const T fkj = F.at(k, j);
                    const int i1 = min(f, k + 1 + (ch + 1) * COOP_ROWS);
                    for (int i = k + 1 + ch * COOP_ROWS + lane; i < i1; i += 32) F.at(i, j) -= T(sc.lvec[i]) * fkj;
                }
                for (int i = k + 1 + gt; i < f; i += GT) F.at(i, k) = T(sc.lvec[i]);
                group_barrier(bar, epoch, gs, G.status);
                k += 1;
            } else {
                const double a = F.get(k, k), b = F.get(k + 1, k), c2 = F.get(k + 1, k + 1);
                const double det = a * c2 - b * b;
                const double e11 = c2 / det, e12 = -b / det, e21 = -b / det, e22 = a / det;
                st[ST_N2X2]++;
                if (det < 0) { st[ST_NPOS]++; st[ST_NNEG]++; }
                else if (a > 0) st[ST_NPOS] += 2;
                else st[ST_NNEG] += 2;
                for (int i = k + 2 + gt; i < f; i += GT) {
                    const double x1 = F.get(i, k), x2 = F.get(i, k + 1);
                    sc.lvec[i] = x1 * e11 + x2 * e21;
                    sc.lvec[f + i] = x1 * e12 + x2 * e22;
                }
                group_barrier(bar, epoch, gs, G.status);
                if (lead) {
                    F.at(k, k + 1) = T(b);
                    sc.dd[k] = a; sc.dd[k + 1] = c2; sc.ee[k] = b; sc.ee[k + 1] = 0.0;
                    sc.kd[k] = KIND_2X2_FIRST; sc.kd[k + 1] = KIND_2X2_SECOND;
                }
                const int nj = w - k - 2;
                const int nch2 = (f - k - 2 + COOP_ROWS - 1) / COOP_ROWS;
                for (int item = gw; nj > 0 && item < nj * nch2; item += GW) {
                    const int j = k + 2 + item % nj, ch = item / nj;
                    const T fkj = F.at(k, j), fk1j = F.at(k + 1, j);
                    const int i1 = min(f, k + 2 + (ch + 1) * COOP_ROWS);
                    for (int i = k + 2 + ch * COOP_ROWS + lane; i < i1; i += 32)
                        F.at(i, j) -= T(sc.lvec[i]) * fkj + T(sc.lvec[f + i]) * fk1j;
                }
                for (int i = k + 2 + gt; i < f; i += GT) {
                    F.at(i, k) = T(sc.lvec[i]);
                    F.at(i, k + 1) = T(sc.lvec[f + i]);
                }
                if (lead) F.at(k + 1, k) = T(0);
                group_barrier(bar, epoch, gs, G.status);
                k += 2;
            }
        }
    } else {
        const bool pivoting = A.lu_pivot != 0;
        for (int k = 0; k < w; ++k) {
            if (rank == 0) {
                int r = pivoting ? lu_choose_row(F, k, w, A.u, team) : k;
                if (tid == 0) sc.ctl[0] = r;
            }
            group_barrier(bar, epoch, gs, G.status);
            const int r = sc.ctl[0];
            if (r != k) {
                for (int j = gt; j < f; j += GT) {
                    T t = F.at(k, j); F.at(k, j) = F.at(r, j); F.at(r, j) = t;
                }
                if (lead) { int t = sc.lp[k]; sc.lp[k] = sc.lp[r]; sc.lp[r] = t; }
                group_barrier(bar, epoch, gs, G.status);
            }
            double dk = F.get(k, k);
            signed char kk = KIND_1X1;
            if (!(fabs(dk) >= A.eps) || dk == 0.0) {
                if (dk == 0.0) st[ST_NZERO]++;
                dk = perturb_sign_of(dk, 0) * A.eps;
                kk = KIND_PERTURBED;
                st[ST_NPERT]++;
                if (dk == 0.0 && st[ST_INFO] == 0) st[ST_INFO] = k + 1;
            }
            group_barrier(bar, epoch, gs, G.status);   // every CTA has read F[k, k]
            if (lead) { F.at(k, k) = T(dk); sc.dd[k] = dk; sc.kd[k] = kk; }
            const T tdk = T(dk);
            const int nj = f - k - 1;
            const int nch = (f - k - 1 + COOP_ROWS - 1) / COOP_ROWS;
            for (int item = gw; item < nj * nch; item += GW) {
                const int j = k + 1 + item % nj, ch = item / nj;
                const int iend = j < w ? f : w;
                const int i0 = k + 1 + ch * COOP_ROWS;
                if (i0 >= iend) continue;
                const T fkj = F.at(k, j);
                const int i1 = min(iend, i0 + COOP_ROWS);
                for (int i = i0 + lane; i < i1; i += 32) F.at(i, j) -= F.at(i, k) / tdk * fkj;
            }
            group_barrier(bar, epoch, gs, G.status);
            for (int i = k + 1 + gt; i < f; i += GT) F.at(i, k) /= tdk;
            for (int j = k + 1 + gt; j < f; j += GT) F.at(k, j) /= tdk;
            group_barrier(bar, epoch, gs, G.status);
        }
    }
    for (int q = gt; q < w * w; q += GT) {
        const int i = q % w, j = q / w;
        if (i == j) {
            P[i + (int64_t)j * f] = T(1);
            if (GEN) U[i + (int64_t)j * f] = T(1);
        } else if (i < j && !GEN) {
            P[i + (int64_t)j * f] = T(0);
        }
    }
    const int64_t n = A.n;
    for (int q = gt; q < w; q += GT) {
        const int64_t g = fd.c0 + q;
        A.piv[g] = fd.c0 + sc.lp[q] + 1;
        A.kind[g] = sc.kd[q];
        A.d[g] = sc.dd[q];
        A.d[n + g] = STRUCT == STRUCT_S ? sc.ee[q] : 0.0;
    }
    if (lead) {
        int64_t* S = A.stats + (int64_t)s * NSTAT;
        for (int q = 0; q < NSTAT; ++q) S[q] = st[q];
        A.finfo[s] = (int32_t)st[ST_INFO];
    }
}

template <typename T>
cudaError_t launch_large_pivot_coop(int structure, const LargePivotArgs<T>& a, const CoopGroups& g, int grid,
                                    cudaStream_t st) {
    if (a.count == 0 || grid == 0) return cudaSuccess;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(COOP_THREADS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (structure == STRUCT_S) return cudaLaunchKernelEx(&cfg, large_pivot_coop_kernel<T, STRUCT_S>, a, g);
    return cudaLaunchKernelEx(&cfg, large_pivot_coop_kernel<T, STRUCT_G>, a, g);
}

template <typename T>
int large_pivot_coop_capacity(int structure) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = structure == STRUCT_S
                        ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, large_pivot_coop_kernel<T, STRUCT_S>,
                                                                        COOP_THREADS, 0)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, large_pivot_coop_kernel<T, STRUCT_G>,
                                                                        COOP_THREADS, 0);
    if (e != cudaSuccess) return 0;
    return sms * per;
}

template cudaError_t launch_large_pivot_coop<double>(int, const LargePivotArgs<double>&, const CoopGroups&, int,
                                                     cudaStream_t);
template cudaError_t launch_large_pivot_coop<float>(int, const LargePivotArgs<float>&, const CoopGroups&, int,
                                                    cudaStream_t);
template int large_pivot_coop_capacity<double>(int);
template int large_pivot_coop_capacity<float>(int);

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
        if (STRUCT == STRUCT_S && kq == KIND_2X2_FIRST) {
            double x2 = (double)P[w + i + (int64_t)(q + 1) * f];
            v = x * d[g] + x2 * d[A.n + g];
        } else if (STRUCT == STRUCT_S && kq == KIND_2X2_SECOND) {
            double x1 = (double)P[w + i + (int64_t)(q - 1) * f];
            v = x1 * d[A.n + g - 1] + x * d[g];
        } else {
            v = x * d[g];
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

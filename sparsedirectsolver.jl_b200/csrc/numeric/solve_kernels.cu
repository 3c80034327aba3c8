// Solve phase: permutation of the right-hand sides, level-batched forward,
// diagonal and backward sweeps over the supernodal factor, and the FP64
// residual / correction of iterative refinement.
//
// Replaces permute_rhs! / unpermute_solution! (src/solve/permute.jl:117-148),
// forward_sweep! / solve_fwd_kernel! (src/solve/sweeps.jl:438-482, 908-942),
// diagonal_sweep! / _sv_diag_kernel! (:549-569, 955-969), backward_sweep! /
// solve_bwd_kernel! (:495-529, 984-1004) and residual! / add_correction!
// (src/solve/refinement.jl:136-153, 190-209, 229-333).
//
// The forward sweep is the deterministic owner-pull variant of the reference
// (sweeps.jl:250-285): every front writes L21 x into its own update vector and
// the parent pulls its children's vectors through relind in child order, so
// the solve is bitwise reproducible without atomics. Right-hand-side vectors
// are FP64 whatever the factor precision (the FP32 factor is read and widened).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"
#include "solve.cuh"

namespace sds {

constexpr int SOLVE_THREADS = 256;

// acc[r] += sum_{j < W} Lrow[j * ld] * x[j + r * ldx] for r < rc (<= 8): sixteen independent loads
// are issued before their FMAs, so that a thread keeps many factor loads in flight
template <typename T>
__device__ __forceinline__ void row_dot(const T* __restrict__ Lrow, int64_t ld, int W, const double* x, int ldx,
                                        int rc, double* acc) {
    int j = 0;
    for (; j + 16 <= W; j += 16) {
        double lv[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) lv[u] = (double)Lrow[(int64_t)(j + u) * ld];
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int r = 0; r < 8; ++r)
                if (r < rc) acc[r] += lv[u] * x[j + u + r * ldx];
    }
    for (; j + 4 <= W; j += 4) {
        double lv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) lv[u] = (double)Lrow[(int64_t)(j + u) * ld];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int r = 0; r < 8; ++r)
                if (r < rc) acc[r] += lv[u] * x[j + u + r * ldx];
    }
    for (; j < W; ++j) {
        const double l = (double)Lrow[(int64_t)j * ld];
#pragma unroll
        for (int r = 0; r < 8; ++r)
            if (r < rc) acc[r] += l * x[j + r * ldx];
    }
}

// acc[r] += sum_{i = lane, lane + 32, ... < M} Lcol[i] * xval(i, r): a warp-strided dot with sixteen
// loads in flight per lane
template <typename T, class XF>
__device__ __forceinline__ void col_dot(const T* __restrict__ Lcol, int M, int lane, int rc, XF xval, double* acc) {
    int i = lane;
    for (; i + 480 < M; i += 512) {
        double lv[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) lv[u] = (double)Lcol[i + 32 * u];
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int r = 0; r < 8; ++r)
                if (r < rc) acc[r] += lv[u] * xval(i + 32 * u, r);
    }
    for (; i + 96 < M; i += 128) {
        double lv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) lv[u] = (double)Lcol[i + 32 * u];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int r = 0; r < 8; ++r)
                if (r < rc) acc[r] += lv[u] * xval(i + 32 * u, r);
    }
    for (; i < M; i += 32) {
        const double l = (double)Lcol[i];
#pragma unroll
        for (int r = 0; r < 8; ++r)
            if (r < rc) acc[r] += l * xval(i, r);
    }
}

// Pull one child's update vectors (mc x nrhs at uc) into a front: row p = ri[i] of the front takes
// x[p + r * ldx] -= uc (p < w, the front's own solution entries) or u[(p - w) + r * m] += uc (its
// update rows). The child's rows map to distinct rows of the front, so one batch of eight never
// touches a target twice and all of its loads go out before its stores.
__device__ __forceinline__ void pull_child(int t0, int step, int N, int mc, const int32_t* ri, const double* uc,
                                           int w, int m, double* x, int64_t ldx, double* u) {
    for (int q0 = t0; q0 < N; q0 += 8 * step) {
        double* dst[8];
        double val[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int q = q0 + k * step;
            dst[k] = nullptr;
            val[k] = 0.0;
            if (q < N) {
                const int p = ri[q % mc], r = q / mc;
                dst[k] = p < w ? x + p + (int64_t)r * ldx : u + (p - w) + (int64_t)r * m;
                val[k] = p < w ? -uc[q] : uc[q];
            }
        }
        double cur[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) cur[k] = dst[k] ? *dst[k] : 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (dst[k]) *dst[k] = cur[k] + val[k];
    }
}

// forward step of one front by one CTA (xs: w x nrhs shared doubles)
template <typename T>
__device__ void forward_front(const SweepArgs<T>& A, int s, int member, double* xs) {
    const DFront fd = A.fronts[s];
    const int f = fd.f, w = fd.w, m = f - w, nrhs = A.nrhs;
    const int64_t n = A.n;
    const T* L = A.fac + (int64_t)member * A.factor_len + fd.panel;
    double* Y = A.Y + (int64_t)member * n * nrhs;
    double* U = A.U + (int64_t)member * A.ulen;
    double* u = m > 0 ? U + A.uoff[s] : nullptr;
    const int32_t* piv = A.piv ? A.piv + (int64_t)member * n : nullptr;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    // gather this front's slice in the numbering before pivoting: the children's updates use it
    batched_copy<4>(tid, nt, w * nrhs, [&](int q) { return Y[fd.c0 + q % w + (int64_t)(q / w) * n]; },
                    [&](int q, double v) { xs[q] = v; });
    for (int q = tid; q < m * nrhs; q += nt) u[q] = 0.0;
    __syncthreads();
    for (int cq = fd.ch_begin; cq < fd.ch_end; ++cq) {
        const int c = A.child_list[cq];
        const DFront cd = A.fronts[c];
        const int mc = cd.f - cd.w;
        if (mc <= 0) continue;
        const double* uc = U + A.uoff[c];
        const int32_t* ri = A.relind + cd.ri_begin;
        pull_child(tid, nt, mc * nrhs, mc, ri, uc, w, m, xs, w, u);
        __syncthreads();
    }
    if (A.pull_only) {
        // the Schur root: its rows keep Y2 - L21 Y1, the condensed right-hand side
        for (int q = tid; q < w * nrhs; q += nt) Y[fd.c0 + q % w + (int64_t)(q / w) * n] = xs[q];
        __syncthreads();
        return;
    }
    if (A.reorder) {
        // apply the local pivot order (the rows of this front's own columns only)
        for (int q = tid; q < w * nrhs; q += nt) {
            int k = q % w, r = q / w;
            Y[fd.c0 + k + (int64_t)r * n] = xs[q];
        }
        __syncthreads();
        batched_copy<4>(tid, nt, w * nrhs, [&](int q) { return Y[piv[fd.c0 + q % w] - 1 + (int64_t)(q / w) * n]; },
                        [&](int q, double v) { xs[q] = v; });
        __syncthreads();
    }
    // L11 solve in blocks of 32 columns: the CTA stages the diagonal block in shared memory, warp 0
    // solves it, the CTA updates the rows of L11 below it
    __shared__ double Ld[32][33];
    for (int jb = 0; jb < w; jb += 32) {
        const int bw = min(32, w - jb);
        batched_copy<4>(tid, nt, 32 * 32,
                        [&](int q) {
                            const int i = q & 31, j = q >> 5;
                            return (i < bw && j < bw && i >= j) ? (double)L[(jb + i) + (int64_t)(jb + j) * f] : 0.0;
                        },
                        [&](int q, double v) { Ld[q & 31][q >> 5] = v; });
        __syncthreads();
        // one warp per right-hand side; each lane applies its own reciprocal diagonal entry
        const double rdl = (!A.unit && lane < bw) ? 1.0 / Ld[lane][lane] : 1.0;
        for (int r = warp; r < nrhs; r += nwarps) {
            double val = lane < bw ? xs[jb + lane + r * w] : 0.0;
            for (int j = 0; j < bw; ++j) {
                if (lane == j) val *= rdl;
                double xj = __shfl_sync(0xffffffffu, val, j);
                if (lane > j) val -= Ld[lane][j] * xj;
            }
            if (lane < bw) xs[jb + lane + r * w] = val;
        }
        __syncthreads();
        for (int q = jb + bw + tid; q < w; q += nt) {
            double acc[8];
            for (int r0 = 0; r0 < nrhs; r0 += 8) {
                const int rc = min(8, nrhs - r0);
#pragma unroll
                for (int r = 0; r < 8; ++r) acc[r] = 0.0;
                row_dot(L + q + (int64_t)jb * f, f, bw, xs + jb + r0 * w, w, rc, acc);
                for (int r = 0; r < rc; ++r) xs[q + (r0 + r) * w] -= acc[r];
            }
        }
        __syncthreads();
    }
    // u += L21 x (large fronts: the row tiles of forward_rect_kernel)
    if (A.rect) {
        for (int i = tid; i < m; i += nt) {
            double acc[8];
            for (int r0 = 0; r0 < nrhs; r0 += 8) {
                const int rc = min(8, nrhs - r0);
#pragma unroll
                for (int r = 0; r < 8; ++r) acc[r] = 0.0;
                row_dot(L + w + i, f, w, xs + r0 * w, w, rc, acc);
                for (int r = 0; r < rc; ++r) u[i + (r0 + r) * m] += acc[r];
            }
        }
    }
    for (int q = tid; q < w * nrhs; q += nt) {
        int k = q % w, r = q / w;
        Y[fd.c0 + k + (int64_t)r * n] = xs[q];
    }
    (void)lane; (void)nwarps;
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(SOLVE_THREADS) forward_kernel(SweepArgs<T> A) {
    extern __shared__ double xs[];  // w x nrhs
    forward_front(A, A.list[blockIdx.x], A.members ? A.members[blockIdx.y] : blockIdx.y, xs);
}

// backward step of one front by one CTA
template <typename T>
__device__ void backward_front(const SweepArgs<T>& A, int s, int member, double* xs) {
    const DFront fd = A.fronts[s];
    const int f = fd.f, w = fd.w, m = f - w, nrhs = A.nrhs;
    const int64_t n = A.n;
    const T* L = A.fac + (int64_t)member * A.factor_len + fd.panel;
    double* Y = A.Y + (int64_t)member * n * nrhs;
    double* xb = m > 0 ? A.U + (int64_t)member * A.ulen + A.uoff[s] : nullptr;
    const int32_t* piv = A.piv ? A.piv + (int64_t)member * n : nullptr;
    const int32_t* rows = A.rowval + fd.row_begin;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    batched_copy<4>(tid, nt, w * nrhs, [&](int q) { return Y[fd.c0 + q % w + (int64_t)(q / w) * n]; },
                    [&](int q, double v) { xs[q] = v; });
    if (A.rect)
        batched_copy<8>(tid, nt, m * nrhs, [&](int q) { return Y[rows[w + q % m] + (int64_t)(q / m) * n]; },
                        [&](int q, double v) { xb[q] = v; });
    __syncthreads();
    // x1 -= L21^T x2: one warp per column (large fronts: the column tiles of backward_rect_kernel)
    if (A.rect) {
        for (int j = warp; j < w; j += nwarps) {
            double acc[8];
            for (int r0 = 0; r0 < nrhs; r0 += 8) {
                const int rc = min(8, nrhs - r0);
#pragma unroll
                for (int r = 0; r < 8; ++r) acc[r] = 0.0;
                col_dot(L + w + (int64_t)j * f, m, lane, rc,
                        [&](int i, int r) { return xb[i + (r0 + r) * m]; }, acc);
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    double v = acc[r];
                    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                    if (lane == 0 && r < rc) xs[j + (r0 + r) * w] -= v;
                }
            }
        }
        __syncthreads();
    }
    // L11^T solve, blocks of 32 from the last, the diagonal block staged in shared memory
    __shared__ double Ld[32][33];
    const int nblk = (w + 31) / 32;
    for (int bq = nblk - 1; bq >= 0; --bq) {
        const int jb = bq * 32, bw = min(32, w - jb);
        batched_copy<4>(tid, nt, 32 * 32,
                        [&](int q) {
                            const int i = q & 31, j = q >> 5;
                            return (i < bw && j < bw && i >= j) ? (double)L[(jb + i) + (int64_t)(jb + j) * f] : 0.0;
                        },
                        [&](int q, double v) { Ld[q & 31][q >> 5] = v; });
        __syncthreads();
        const double rdl = (!A.unit && lane < bw) ? 1.0 / Ld[lane][lane] : 1.0;
        for (int r = warp; r < nrhs; r += nwarps) {
            double val = lane < bw ? xs[jb + lane + r * w] : 0.0;
            for (int j = bw - 1; j >= 0; --j) {
                if (lane == j) val *= rdl;
                double xj = __shfl_sync(0xffffffffu, val, j);
                if (lane < j) val -= Ld[j][lane] * xj;
            }
            if (lane < bw) xs[jb + lane + r * w] = val;
        }
        __syncthreads();
        for (int i = warp; i < jb; i += nwarps) {
            const double l = lane < bw ? (double)L[(jb + lane) + (int64_t)i * f] : 0.0;
            for (int r = 0; r < nrhs; ++r) {
                double v = lane < bw ? l * xs[jb + lane + r * w] : 0.0;
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0) xs[i + r * w] -= v;
            }
        }
        __syncthreads();
    }
    for (int q = tid; q < w * nrhs; q += nt) {
        int k = q % w, r = q / w;
        int dst = A.reorder ? piv[fd.c0 + k] - 1 : fd.c0 + k;
        Y[dst + (int64_t)r * n] = xs[q];
    }
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(SOLVE_THREADS) backward_kernel(SweepArgs<T> A) {
    extern __shared__ double xs[];  // w x nrhs
    backward_front(A, A.list[blockIdx.x], A.members ? A.members[blockIdx.y] : blockIdx.y, xs);
}

// u[rows of the tile] += L21[rows, :] x1 for one row tile of a large front (x1 from Y, pivoted order)
template <typename T>
__global__ void __launch_bounds__(RECT_ROWS) forward_rect_kernel(SweepArgs<T> A) {
    extern __shared__ double xs[];  // w x nrhs
    const int s = A.tiles[2 * blockIdx.x], row0 = A.tiles[2 * blockIdx.x + 1];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    const DFront fd = A.fronts[s];
    const int f = fd.f, w = fd.w, m = f - w, nrhs = A.nrhs;
    const int64_t n = A.n;
    const T* L = A.fac + (int64_t)member * A.factor_len + fd.panel;
    const double* Y = A.Y + (int64_t)member * n * nrhs;
    double* u = A.U + (int64_t)member * A.ulen + A.uoff[s];
    for (int q = threadIdx.x; q < w * nrhs; q += blockDim.x) {
        int k = q % w, r = q / w;
        xs[q] = Y[fd.c0 + k + (int64_t)r * n];
    }
    __syncthreads();
    const int i = row0 + threadIdx.x;
    if (i >= m) return;
    for (int r0 = 0; r0 < nrhs; r0 += 8) {
        const int rc = min(8, nrhs - r0);
        double acc[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) acc[r] = 0.0;
        row_dot(L + w + i, f, w, xs + r0 * w, w, rc, acc);
        for (int r = 0; r < rc; ++r) u[i + (r0 + r) * m] += acc[r];
    }
}

// Y[c0 + j] -= (L21^T x2)[j] for one tile of RECT_COLS columns of a large front, one warp per column;
// x2 gathered from the finished ancestor rows
template <typename T>
__global__ void __launch_bounds__(RECT_COLS * 32) backward_rect_kernel(SweepArgs<T> A) {
    const int s = A.tiles[2 * blockIdx.x], col0 = A.tiles[2 * blockIdx.x + 1];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    const DFront fd = A.fronts[s];
    const int f = fd.f, w = fd.w, m = f - w, nrhs = A.nrhs;
    const int64_t n = A.n;
    const T* L = A.fac + (int64_t)member * A.factor_len + fd.panel;
    double* Y = A.Y + (int64_t)member * n * nrhs;
    const int32_t* rows = A.rowval + fd.row_begin + w;
    const int lane = threadIdx.x & 31;
    const int j = col0 + (threadIdx.x >> 5);
    if (j >= w) return;
    for (int r0 = 0; r0 < nrhs; r0 += 8) {
        const int rc = min(8, nrhs - r0);
        double acc[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) acc[r] = 0.0;
        col_dot(L + w + (int64_t)j * f, m, lane, rc,
                [&](int i, int r) { return Y[rows[i] + (int64_t)(r0 + r) * n]; }, acc);
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            double v = acc[r];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0 && r < rc) Y[fd.c0 + j + (int64_t)(r0 + r) * n] -= v;
        }
    }
}

template <typename T>
cudaError_t launch_sweep_rect(bool forward, const SweepArgs<T>& a, int ntiles, int nmembers, int maxw, cudaStream_t st) {
    if (ntiles == 0) return cudaSuccess;
    dim3 grid(ntiles, nmembers);
    if (forward) {
        size_t smem = (size_t)maxw * a.nrhs * sizeof(double);
        forward_rect_kernel<T><<<grid, RECT_ROWS, smem, st>>>(a);
    } else {
        backward_rect_kernel<T><<<grid, RECT_COLS * 32, 0, st>>>(a);
    }
    return cudaGetLastError();
}

template cudaError_t launch_sweep_rect<double>(bool, const SweepArgs<double>&, int, int, int, cudaStream_t);
template cudaError_t launch_sweep_rect<float>(bool, const SweepArgs<float>&, int, int, int, cudaStream_t);

template <typename T>
cudaError_t launch_sweep(bool forward, const SweepArgs<T>& a, int nmembers, int maxw, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    size_t smem = (size_t)maxw * a.nrhs * sizeof(double);
    dim3 grid(a.count, nmembers);
    if (forward) forward_kernel<T><<<grid, SOLVE_THREADS, smem, st>>>(a);
    else backward_kernel<T><<<grid, SOLVE_THREADS, smem, st>>>(a);
    return cudaGetLastError();
}


template cudaError_t launch_sweep<double>(bool, const SweepArgs<double>&, int, int, cudaStream_t);
template cudaError_t launch_sweep<float>(bool, const SweepArgs<float>&, int, int, cudaStream_t);


// ---------------------------------------------------------------------------
// Warp-per-front sweeps of the small fronts in the persistent solve (w < 96): eight fronts in flight per
// CTA. xs: w x nrhs, Ld: 32 x 33 (both per warp, shared memory).
template <typename T>
__device__ void warp_forward_front(const SweepArgs<T>& A, int s, double* xs, double* Ld) {
    const DFront fd = A.fronts[s];
    const int f = fd.f, w = fd.w, m = f - w, nrhs = A.nrhs, lane = threadIdx.x & 31;
    const int64_t n = A.n;
    const T* L = A.fac + fd.panel;
    double* Y = A.Y;
    double* U = A.U;
    double* u = m > 0 ? U + A.uoff[s] : nullptr;
    batched_copy<8>(lane, 32, w * nrhs, [&](int q) { return Y[fd.c0 + q % w + (int64_t)(q / w) * n]; },
                    [&](int q, double v) { xs[q] = v; });
    for (int q = lane; q < m * nrhs; q += 32) u[q] = 0.0;
    __syncwarp();
    for (int cq = fd.ch_begin; cq < fd.ch_end; ++cq) {
        const int c = A.child_list[cq];
        const DFront cd = A.fronts[c];
        const int mc = cd.f - cd.w;
        if (mc <= 0) continue;
        const double* uc = U + A.uoff[c];
        const int32_t* ri = A.relind + cd.ri_begin;
        pull_child(lane, 32, mc * nrhs, mc, ri, uc, w, m, xs, w, u);
        __syncwarp();
    }
    if (A.reorder) {
        for (int q = lane; q < w * nrhs; q += 32) Y[fd.c0 + q % w + (int64_t)(q / w) * n] = xs[q];
        __syncwarp();
        batched_copy<8>(lane, 32, w * nrhs, [&](int q) { return Y[A.piv[fd.c0 + q % w] - 1 + (int64_t)(q / w) * n]; },
                        [&](int q, double v) { xs[q] = v; });
        __syncwarp();
    }
    for (int jb = 0; jb < w; jb += 32) {
        const int bw = min(32, w - jb);
        batched_copy<8>(0, 1, bw,
                        [&](int j) { return (lane < bw && lane >= j) ? (double)L[(jb + lane) + (int64_t)(jb + j) * f] : 0.0; },
                        [&](int j, double v) { Ld[lane * 33 + j] = v; });
        __syncwarp();
        // all right-hand sides (chunks of 8) in one shuffle chain; reciprocal diagonal per lane
        const double rdl = (!A.unit && lane < bw) ? 1.0 / Ld[lane * 33 + lane] : 1.0;
        for (int r0 = 0; r0 < nrhs; r0 += 8) {
            const int rc = min(8, nrhs - r0);
            double val[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) val[r] = (lane < bw && r < rc) ? xs[jb + lane + (r0 + r) * w] : 0.0;
            for (int j = 0; j < bw; ++j) {
                const double lj = Ld[lane * 33 + j];
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    if (lane == j) val[r] *= rdl;
                    const double xj = __shfl_sync(0xffffffffu, val[r], j);
                    if (lane > j) val[r] -= lj * xj;
                }
            }
#pragma unroll
            for (int r = 0; r < 8; ++r)
                if (lane < bw && r < rc) xs[jb + lane + (r0 + r) * w] = val[r];
        }
        __syncwarp();
        for (int q = jb + bw + lane; q < w; q += 32) {
            for (int r0 = 0; r0 < nrhs; r0 += 8) {
                const int rc = min(8, nrhs - r0);
                double acc[8];
#pragma unroll
                for (int r = 0; r < 8; ++r) acc[r] = 0.0;
                row_dot(L + q + (int64_t)jb * f, f, bw, xs + jb + r0 * w, w, rc, acc);
                for (int r = 0; r < rc; ++r) xs[q + (r0 + r) * w] -= acc[r];
            }
        }
        __syncwarp();
    }
    for (int i = lane; i < m; i += 32) {
        for (int r0 = 0; r0 < nrhs; r0 += 8) {
            const int rc = min(8, nrhs - r0);
            double acc[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) acc[r] = 0.0;
            row_dot(L + w + i, f, w, xs + r0 * w, w, rc, acc);
            for (int r = 0; r < rc; ++r) u[i + (r0 + r) * m] += acc[r];
        }
    }
    for (int q = lane; q < w * nrhs; q += 32) Y[fd.c0 + q % w + (int64_t)(q / w) * n] = xs[q];
    __syncwarp();
}

template <typename T>
__device__ void warp_backward_front(const SweepArgs<T>& A, int s, double* xs, double* Ld) {
    const DFront fd = A.fronts[s];
    const int f = fd.f, w = fd.w, m = f - w, nrhs = A.nrhs, lane = threadIdx.x & 31;
    const int64_t n = A.n;
    const T* L = A.fac + fd.panel;
    double* Y = A.Y;
    const int32_t* rows = A.rowval + fd.row_begin + w;
    batched_copy<8>(lane, 32, w * nrhs, [&](int q) { return Y[fd.c0 + q % w + (int64_t)(q / w) * n]; },
                    [&](int q, double v) { xs[q] = v; });
    __syncwarp();
    // x1 -= L21^T x2: x2 = Y[rows below] gathered in chunks into Ld, lanes over the columns
    const int CH = max(1, (32 * 33) / nrhs);
    for (int i0 = 0; i0 < m; i0 += CH) {
        const int ch = min(CH, m - i0);
        batched_copy<8>(lane, 32, ch * nrhs, [&](int q) { return Y[rows[i0 + q % ch] + (int64_t)(q / ch) * n]; },
                        [&](int q, double v) { Ld[q] = v; });
        __syncwarp();
        for (int j = lane; j < w; j += 32) {
            const T* Lc = L + w + i0 + (int64_t)j * f;
            for (int r0 = 0; r0 < nrhs; r0 += 8) {
                const int rc = min(8, nrhs - r0);
                double acc[8];
#pragma unroll
                for (int r = 0; r < 8; ++r) acc[r] = 0.0;
                int i = 0;
                for (; i + 8 <= ch; i += 8) {
                    double lv[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) lv[u] = (double)Lc[i + u];
#pragma unroll
                    for (int u = 0; u < 8; ++u)
#pragma unroll
                        for (int r = 0; r < 8; ++r)
                            if (r < rc) acc[r] += lv[u] * Ld[i + u + (r0 + r) * ch];
                }
                for (; i < ch; ++i) {
                    const double l = (double)Lc[i];
#pragma unroll
                    for (int r = 0; r < 8; ++r)
                        if (r < rc) acc[r] += l * Ld[i + (r0 + r) * ch];
                }
                for (int r = 0; r < rc; ++r) xs[j + (r0 + r) * w] -= acc[r];
            }
        }
        __syncwarp();
    }
    const int nblk = (w + 31) / 32;
    for (int bq = nblk - 1; bq >= 0; --bq) {
        const int jb = bq * 32, bw = min(32, w - jb);
        batched_copy<8>(0, 1, bw,
                        [&](int j) { return (lane < bw && lane >= j) ? (double)L[(jb + lane) + (int64_t)(jb + j) * f] : 0.0; },
                        [&](int j, double v) { Ld[lane * 33 + j] = v; });
        __syncwarp();
        const double rdl = (!A.unit && lane < bw) ? 1.0 / Ld[lane * 33 + lane] : 1.0;
        for (int r0 = 0; r0 < nrhs; r0 += 8) {
            const int rc = min(8, nrhs - r0);
            double val[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) val[r] = (lane < bw && r < rc) ? xs[jb + lane + (r0 + r) * w] : 0.0;
            for (int j = bw - 1; j >= 0; --j) {
                const double lj = Ld[j * 33 + lane];
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    if (lane == j) val[r] *= rdl;
                    const double xj = __shfl_sync(0xffffffffu, val[r], j);
                    if (lane < j) val[r] -= lj * xj;
                }
            }
#pragma unroll
            for (int r = 0; r < 8; ++r)
                if (lane < bw && r < rc) xs[jb + lane + (r0 + r) * w] = val[r];
        }
        __syncwarp();
        for (int i = lane; i < jb; i += 32) {
            const T* Lr = L + jb + (int64_t)i * f;   // L[jb + k, i], contiguous in k
            for (int r0 = 0; r0 < nrhs; r0 += 8) {
                const int rc = min(8, nrhs - r0);
                double acc[8];
#pragma unroll
                for (int r = 0; r < 8; ++r) acc[r] = 0.0;
                row_dot(Lr, 1, bw, xs + jb + r0 * w, w, rc, acc);
                for (int r = 0; r < rc; ++r) xs[i + (r0 + r) * w] -= acc[r];
            }
        }
        __syncwarp();
    }
    for (int q = lane; q < w * nrhs; q += 32) {
        const int k = q % w;
        const int dst = A.reorder ? A.piv[fd.c0 + k] - 1 : fd.c0 + k;
        Y[dst + (int64_t)(q / w) * n] = xs[q];
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Persistent solve. Grid barrier: one arrival per CTA on a monotonic counter; the wait is bounded
// (about two seconds of spinning), after which the CTA records the failure and goes on, so a lost
// CTA never hangs the device (the results are then garbage and the status word says so).
__device__ __forceinline__ void grid_barrier(unsigned int* bar, unsigned int& epoch, int32_t* status) {
    __syncthreads();
    epoch += gridDim.x;
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

// Shared memory of a wide-front item: the 64 x 64 inverse block, the item's rows (or columns) of y,
// x of the block being applied, and partial sums.
constexpr int WT_SMEM_DOUBLES_FIXED = SOLVE_BLK * (SOLVE_BLK + 1);

// Flags of the wide fronts' dataflow: a block's solution is published by its owner (stores, fence,
// release of the flag) and read by the items that need it after an acquire of the flag. The wait is
// bounded like the grid barrier, and gives up at once when any wait of the launch has given up.
__device__ __forceinline__ void publish_flag(unsigned int* flag, unsigned int v) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) asm volatile("st.release.gpu.u32 [%0], %1;" ::"l"(flag), "r"(v) : "memory");
}

__device__ __forceinline__ void wait_flag(const unsigned int* flag, unsigned int target, int32_t* status) {
    if (threadIdx.x == 0) {
        unsigned int v;
        long spins = 0;
        while (true) {
            asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
            if (v >= target) break;
            if (++spins > (1L << 26) || ((spins & 255) == 0 && *(volatile int32_t*)status != 0)) {
                atomicExch(status, 1);
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
    }
    __syncthreads();
}

// Forward sweep of a wide front, row tile t (rows 64 t .. 64 t + 63), owned by one CTA once the front's
// pull is flagged: the tile takes
// x_b of every block b <= t in increasing order (rows below block b: y -= L x_b for rows of the block
// column, u += L x_b for the rows below the front's columns); at b = t the tile holds block t's rows and
// solves them, x_t = inv(L_tt) y_t, publishing x_t for the tiles below. The arithmetic and its order
// are those of a block-step sweep with a grid barrier after every step.
template <typename T>
__device__ void wide_forward_owner(const PersistArgs<T>& P, int s, int t, double* sm) {
    const SweepArgs<T>& A = P.fw;
    const DFront fd = A.fronts[s];
    const int f = fd.f, w = fd.w, m = f - w, nrhs = A.nrhs;
    const int64_t n = A.n;
    const int nb = (w + SOLVE_BLK - 1) / SOLVE_BLK;
    const int r0 = t * SOLVE_BLK, rows = min(SOLVE_BLK, f - r0);
    const T* L = A.fac + fd.panel;
    double* Y = A.Y;
    double* u = m > 0 ? A.U + A.uoff[s] : nullptr;
    const int64_t base = P.dinv_off[s] / (SOLVE_BLK * SOLVE_BLK);
    unsigned int* flag = P.blkflag + base;
    double* Iv = sm;                                  // SOLVE_BLK x (SOLVE_BLK + 1)
    double* yb = sm + WT_SMEM_DOUBLES_FIXED;          // the tile's rows, SOLVE_BLK x nrhs
    double* xb = yb + SOLVE_BLK * nrhs;               // x of the block being applied
    double* part = xb + SOLVE_BLK * nrhs;             // 4 x SOLVE_BLK x nrhs partial sums
    const int tid = threadIdx.x, nt = blockDim.x;
    wait_flag(P.pullflag + base, 1u, P.status);       // the front's children are pulled into Y and u
    batched_copy<4>(tid, nt, SOLVE_BLK * nrhs,
                    [&](int q) {
                        const int i = q % SOLVE_BLK, r = q / SOLVE_BLK, row = r0 + i;
                        if (i >= rows) return 0.0;
                        return row < w ? Y[fd.c0 + row + (int64_t)r * n] : u[row - w + (int64_t)r * m];
                    },
                    [&](int q, double v) { yb[q] = v; });
    if (t < nb) {
        const int bwt = min(SOLVE_BLK, w - r0);
        const T* inv = P.dinv_fw + P.dinv_off[s] + (int64_t)t * SOLVE_BLK * SOLVE_BLK;
        batched_copy<8>(tid, nt, SOLVE_BLK * SOLVE_BLK,
                        [&](int q) { return (q % SOLVE_BLK < bwt && q / SOLVE_BLK < bwt) ? (double)inv[q] : 0.0; },
                        [&](int q, double v) { Iv[q % SOLVE_BLK + (q / SOLVE_BLK) * (SOLVE_BLK + 1)] = v; });
    }
    __syncthreads();
    const int row = r0 + (tid & (SOLVE_BLK - 1)), quarter = tid / SOLVE_BLK;
    for (int b = 0; b <= min(t, nb - 1); ++b) {
        const int jb = b * SOLVE_BLK, bw = min(SOLVE_BLK, w - jb);
        if (b == t) {
            for (int q = tid; q < SOLVE_BLK * nrhs; q += nt) {
                const int i = q % SOLVE_BLK, r = q / SOLVE_BLK;
                double acc = 0.0;
#pragma unroll 8
                for (int j = 0; j < SOLVE_BLK; ++j)
                    acc += Iv[i + j * (SOLVE_BLK + 1)] * (j < bw ? yb[j + r * SOLVE_BLK] : 0.0);
                xb[q] = acc;
            }
            __syncthreads();
            for (int q = tid; q < bw * nrhs; q += nt) {
                const int k = q % bw, r = q / bw;
                const double v = xb[k + r * SOLVE_BLK];
                P.xtmp[fd.c0 + jb + k + (int64_t)r * n] = v;
                Y[fd.c0 + jb + k + (int64_t)r * n] = v;
            }
            publish_flag(flag + b, 1u);
        } else {
            wait_flag(flag + b, 1u, P.status);
            for (int q = tid; q < SOLVE_BLK * nrhs; q += nt) {
                const int k = q % SOLVE_BLK, r = q / SOLVE_BLK;
                xb[q] = k < bw ? P.xtmp[fd.c0 + jb + k + (int64_t)r * n] : 0.0;
            }
            __syncthreads();
        }
        // rows of the tile below block b: 4 threads per row, 16 block columns each
        const bool upd = tid < 4 * SOLVE_BLK && row < f && row >= jb + bw;
        for (int r0_ = 0; r0_ < nrhs; r0_ += 8) {
            const int rc = min(8, nrhs - r0_);
            double acc[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) acc[r] = 0.0;
            if (upd) {
                const int c0 = quarter * (SOLVE_BLK / 4), cw = max(0, min(SOLVE_BLK / 4, bw - c0));
                row_dot(L + row + (int64_t)(jb + c0) * f, f, cw, xb + c0 + r0_ * SOLVE_BLK, SOLVE_BLK, rc, acc);
            }
            if (tid < 4 * SOLVE_BLK)
                for (int r = 0; r < rc; ++r) part[(tid & (SOLVE_BLK - 1)) + SOLVE_BLK * (quarter + 4 * r)] = acc[r];
            __syncthreads();
            if (tid < SOLVE_BLK && row < f && row >= jb + bw) {
                for (int r = 0; r < rc; ++r) {
                    const double v = part[tid + SOLVE_BLK * (4 * r)] + part[tid + SOLVE_BLK * (1 + 4 * r)] +
                                     part[tid + SOLVE_BLK * (2 + 4 * r)] + part[tid + SOLVE_BLK * (3 + 4 * r)];
                    if (row < w) yb[tid + (r0_ + r) * SOLVE_BLK] -= v;
                    else yb[tid + (r0_ + r) * SOLVE_BLK] += v;
                }
            }
            __syncthreads();
        }
    }
    // the tile's rows below the front's columns go back to the update vector
    for (int q = tid; q < SOLVE_BLK * nrhs; q += nt) {
        const int i = q % SOLVE_BLK, r = q / SOLVE_BLK;
        if (i < rows && r0 + i >= w) u[r0 + i - w + (int64_t)r * m] = yb[q];
    }
    __syncthreads();
}

// Backward sweep of a wide front, block b (columns 64 b .. 64 b + 63), owned by one CTA, once the
// warps of the y1 -= L21^T x2 phase have counted all of the block's columns: y_b takes -L_tb^T x_t of every later block t in decreasing order as each
// is published, and x_b = inv(L_bb)^T y_b is published into the scratch. The arithmetic and its
// order are those of a block-step sweep with a grid barrier after every step.
template <typename T>
__device__ void wide_backward_owner(const PersistArgs<T>& P, int s, int b, double* sm) {
    const SweepArgs<T>& A = P.bw;
    const DFront fd = A.fronts[s];
    const int f = fd.f, w = fd.w, nrhs = A.nrhs;
    const int64_t n = A.n;
    const int nb = (w + SOLVE_BLK - 1) / SOLVE_BLK;
    const int jb = b * SOLVE_BLK, bw = min(SOLVE_BLK, w - jb);
    const T* L = A.fac + fd.panel;
    const T* inv = P.dinv_bw + P.dinv_off[s] + (int64_t)b * SOLVE_BLK * SOLVE_BLK;
    const int64_t base = P.dinv_off[s] / (SOLVE_BLK * SOLVE_BLK);
    unsigned int* flag = P.blkflag + base;
    double* Y = A.Y;
    double* Iv = sm;
    double* yb = sm + WT_SMEM_DOUBLES_FIXED;
    double* xb = yb + SOLVE_BLK * nrhs;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    wait_flag(P.l21cnt + base + b, f > w ? (unsigned int)bw : 0u, P.status);   // y_b has taken -L21^T x2
    batched_copy<8>(tid, nt, SOLVE_BLK * SOLVE_BLK,
                    [&](int q) { return (q % SOLVE_BLK < bw && q / SOLVE_BLK < bw) ? (double)inv[q] : 0.0; },
                    [&](int q, double v) { Iv[q % SOLVE_BLK + (q / SOLVE_BLK) * (SOLVE_BLK + 1)] = v; });
    batched_copy<4>(tid, nt, SOLVE_BLK * nrhs,
                    [&](int q) { return q % SOLVE_BLK < bw ? Y[fd.c0 + jb + q % SOLVE_BLK + (int64_t)(q / SOLVE_BLK) * n] : 0.0; },
                    [&](int q, double v) { yb[q] = v; });
    __syncthreads();
    const int a0 = jb + warp * (SOLVE_BLK / 8);
    for (int t = nb - 1; t > b; --t) {
        const int jt = t * SOLVE_BLK, bwt = min(SOLVE_BLK, w - jt);
        // this warp's 8 columns of block b against the rows of block t, loaded before the wait
        double l1[SOLVE_BLK / 8], l2[SOLVE_BLK / 8];
#pragma unroll
        for (int c = 0; c < SOLVE_BLK / 8; ++c) {
            const int a = a0 + c;
            l1[c] = lane < bwt ? (double)L[(jt + lane) + (int64_t)a * f] : 0.0;
            l2[c] = lane + 32 < bwt ? (double)L[(jt + lane + 32) + (int64_t)a * f] : 0.0;
        }
        wait_flag(flag + t, 2u, P.status);
        for (int q = tid; q < SOLVE_BLK * nrhs; q += nt) {
            const int k = q % SOLVE_BLK, r = q / SOLVE_BLK;
            xb[q] = k < bwt ? P.xtmp[fd.c0 + jt + k + (int64_t)r * n] : 0.0;
        }
        __syncthreads();
        for (int r = 0; r < nrhs; ++r) {
            const double x1 = xb[lane + r * SOLVE_BLK], x2 = xb[lane + 32 + r * SOLVE_BLK];
#pragma unroll
            for (int c = 0; c < SOLVE_BLK / 8; ++c) {
                double v = l1[c] * x1 + l2[c] * x2;
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0) yb[a0 + c - jb + r * SOLVE_BLK] -= v;
            }
        }
        __syncthreads();
    }
    for (int q = tid; q < SOLVE_BLK * nrhs; q += nt) {
        const int i = q % SOLVE_BLK, r = q / SOLVE_BLK;
        double acc = 0.0;
#pragma unroll 8
        for (int j = 0; j < SOLVE_BLK; ++j) acc += Iv[j + i * (SOLVE_BLK + 1)] * yb[j + r * SOLVE_BLK];
        xb[q] = acc;
    }
    __syncthreads();
    for (int q = tid; q < bw * nrhs; q += nt) {
        const int k = q % bw, r = q / bw;
        P.xtmp[fd.c0 + jb + k + (int64_t)r * n] = xb[k + r * SOLVE_BLK];
    }
    publish_flag(flag + b, 2u);
    if (b == 0) {
        // the last block of the front's chain: every other block's solution was acquired above, and
        // every owner of this front has read its y; the solution goes into Y in the original order
        for (int q = tid; q < w * nrhs; q += nt) {
            const int k = q % w, r = q / w;
            const int64_t dst = A.reorder ? A.piv[fd.c0 + k] - 1 : fd.c0 + k;
            Y[dst + (int64_t)r * n] = P.xtmp[fd.c0 + k + (int64_t)r * n];
        }
        __syncthreads();
    }
}

__device__ __forceinline__ void trace_mark(int64_t* trace, int cap, int& n, int64_t tag) {
    if (trace && blockIdx.x == 0 && threadIdx.x == 0 && n < cap) {
        uint64_t t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        trace[2 * n] = tag;
        trace[2 * n + 1] = (int64_t)t;
        ++n;
    }
}

template <typename T>
__global__ void __launch_bounds__(SOLVE_THREADS) persistent_solve_kernel(PersistArgs<T> P) {
    extern __shared__ double psm[];
    unsigned int epoch = 0;
    int ntr = 0;
    // phase tags: 1 perm, 2 fwd level A, 3 fwd block step, 4 diag, 5 bwd L21^T, 6 bwd block step,
    // 7 bwd level end (small fronts), 8 final; tag = kind << 40 | level << 16 | step
#define TRACE(kind, lev, stp) trace_mark(P.trace, P.trace_cap, ntr, ((int64_t)(kind) << 40) | ((int64_t)(lev) << 16) | (stp))
    TRACE(0, 0, 0);
    const int G = gridDim.x;
    const int64_t n = P.fw.n;
    const int nrhs = P.fw.nrhs;
    const int64_t gtid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, gstride = (int64_t)G * blockDim.x;
    // Y = in[perm]
    for (int64_t q = gtid; q < n * nrhs; q += gstride) {
        int64_t k = q % n, r = q / n;
        P.fw.Y[q] = P.in[P.perm[k] + r * P.ldin];
    }
    grid_barrier(P.barrier, epoch, P.status);
    TRACE(1, 0, 0);
    // forward levels
    for (int L = 0; L < P.nlevels; ++L) {
        const int so = P.lev_small[2 * L], sc = P.lev_small[2 * L + 1];
        const int lo = P.lev_large[2 * L], lc = P.lev_large[2 * L + 1];
        if (sc >= G * (blockDim.x >> 5) / 2) {
            // many small fronts: one warp each
            const int wpc = blockDim.x >> 5, warp = threadIdx.x >> 5;
            double* xs = psm + warp * P.warp_smem;
            for (int i = blockIdx.x * wpc + warp; i < sc; i += G * wpc)
                warp_forward_front(P.fw, P.list[so + i], xs, xs + P.warp_xs);
        } else {
            // few: one CTA each
            for (int i = blockIdx.x; i < sc; i += G) forward_front(P.fw, P.list[so + i], 0, psm);
        }
        // wide fronts: pull the children and apply the local pivot order (one CTA each, from the end)
        for (int i = G - 1 - blockIdx.x; i < lc; i += G) {
            const int s = P.list[lo + i];
            const DFront fd = P.fw.fronts[s];
            const int w = fd.w, m = fd.f - fd.w;
            double* Y = P.fw.Y;
            double* xt = P.xtmp;
            double* u = m > 0 ? P.fw.U + P.fw.uoff[s] : nullptr;
            batched_copy<8>(threadIdx.x, blockDim.x, w * nrhs,
                            [&](int q) { return Y[fd.c0 + q % w + (int64_t)(q / w) * n]; },
                            [&](int q, double v) { xt[fd.c0 + q % w + (int64_t)(q / w) * n] = v; });
            for (int q = threadIdx.x; q < m * nrhs; q += blockDim.x) u[q] = 0.0;
            __syncthreads();
            for (int cq = fd.ch_begin; cq < fd.ch_end; ++cq) {
                const int c = P.fw.child_list[cq];
                const DFront cd = P.fw.fronts[c];
                const int mc = cd.f - cd.w;
                if (mc <= 0) continue;
                const double* uc = P.fw.U + P.fw.uoff[c];
                const int32_t* ri = P.fw.relind + cd.ri_begin;
                pull_child(threadIdx.x, blockDim.x, mc * nrhs, mc, ri, uc, w, m, xt + fd.c0, n, u);
                __syncthreads();
            }
            batched_copy<8>(threadIdx.x, blockDim.x, w * nrhs,
                            [&](int q) {
                                const int k = q % w;
                                const int src = P.fw.reorder ? P.fw.piv[fd.c0 + k] - 1 : fd.c0 + k;
                                return xt[src + (int64_t)(q / w) * n];
                            },
                            [&](int q, double v) { Y[fd.c0 + q % w + (int64_t)(q / w) * n] = v; });
            publish_flag(P.pullflag + P.dinv_off[s] / (SOLVE_BLK * SOLVE_BLK), 1u);
        }
        TRACE(2, L, 0);
        if (lc) {
            // wide fronts: one CTA per (front, row tile); a CTA takes its tiles of a front in increasing
            // order, so every tile waits only on tiles taken earlier
            int total = 0;
            for (int i = 0; i < lc; ++i) total += (P.fw.fronts[P.list[lo + i]].f + SOLVE_BLK - 1) / SOLVE_BLK;
            for (int k = blockIdx.x; k < total; k += G) {
                int kk = k;
                for (int i = 0; i < lc; ++i) {
                    const int s = P.list[lo + i];
                    const int cnt = (P.fw.fronts[s].f + SOLVE_BLK - 1) / SOLVE_BLK;
                    if (kk < cnt) {
                        wide_forward_owner(P, s, kk, psm);
                        break;
                    }
                    kk -= cnt;
                }
            }
        }
        grid_barrier(P.barrier, epoch, P.status);
        TRACE(3, L, 0);
    }
    // the copies of the last level's wide fronts must land before Y is read again
    grid_barrier(P.barrier, epoch, P.status);
    // diagonal: D^{-1} with 1x1 and 2x2 blocks
    if (P.diag_mode) {
        for (int64_t q = gtid; q < n * nrhs; q += gstride) {
            const int64_t k = q % n, r = q / n;
            const int kk = P.kind[k];
            double* Y = P.fw.Y;
            if (P.diag_mode == 2 && kk == KIND_2X2_SECOND) continue;
            if (P.diag_mode == 2 && kk == KIND_2X2_FIRST) {
                double a = P.d[k], b = P.d[n + k], c = P.d[k + 1];
                double det = a * c - b * b;
                double y1 = Y[k + r * n], y2 = Y[k + 1 + r * n];
                Y[k + r * n] = (c * y1 - b * y2) / det;
                Y[k + 1 + r * n] = (a * y2 - b * y1) / det;
            } else {
                Y[k + r * n] /= P.d[k];
            }
        }
        grid_barrier(P.barrier, epoch, P.status);
        TRACE(4, 0, 0);
    }
    // backward levels
    for (int L = P.nlevels - 1; L >= 0; --L) {
        const int so = P.lev_small[2 * L], sc = P.lev_small[2 * L + 1];
        const int lo = P.lev_large[2 * L], lc = P.lev_large[2 * L + 1];
        if (lc) {
            // stage x2 = Y[rows below] of the wide fronts in their update vectors (free in this sweep)
            for (int i = 0; i < lc; ++i) {
                const int s = P.list[lo + i];
                const DFront fd = P.bw.fronts[s];
                const int w = fd.w, m = fd.f - fd.w;
                if (m == 0) continue;
                double* xb = P.bw.U + P.bw.uoff[s];
                const int32_t* rows = P.bw.rowval + fd.row_begin + w;
                for (int64_t q = gtid; q < (int64_t)m * nrhs; q += gstride) {
                    const int i2 = (int)(q % m), r = (int)(q / m);
                    xb[q] = P.bw.Y[rows[i2] + (int64_t)r * n];
                }
            }
            grid_barrier(P.barrier, epoch, P.status);
            // x1 -= L21^T x2 for the wide fronts: one warp per column, columns spread over the grid
            const int warps = blockDim.x >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            int totc = 0;
            for (int i = 0; i < lc; ++i) totc += P.bw.fronts[P.list[lo + i]].w;
            for (int col = blockIdx.x * warps + warp; col < totc; col += G * warps) {
                int j = col, i = 0, s = 0;
                for (; i < lc; ++i) {
                    s = P.list[lo + i];
                    const int wi = P.bw.fronts[s].w;
                    if (j < wi) break;
                    j -= wi;
                }
                const DFront fd = P.bw.fronts[s];
                const int f = fd.f, w = fd.w, m = f - w;
                if (m == 0) continue;
                const T* Lp = P.bw.fac + fd.panel;
                const double* xb = P.bw.U + P.bw.uoff[s];
                for (int r0 = 0; r0 < nrhs; r0 += 8) {
                    const int rc = min(8, nrhs - r0);
                    double acc[8];
#pragma unroll
                    for (int r = 0; r < 8; ++r) acc[r] = 0.0;
                    col_dot(Lp + w + (int64_t)j * f, m, lane, rc,
                            [&](int i2, int r) { return xb[i2 + (r0 + r) * m]; }, acc);
#pragma unroll
                    for (int r = 0; r < 8; ++r) {
                        double v = acc[r];
                        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                        if (lane == 0 && r < rc) P.bw.Y[fd.c0 + j + (int64_t)(r0 + r) * n] -= v;
                    }
                }
                if (lane == 0) {   // release the column to its block's owner
                    __threadfence();
                    atomicAdd(P.l21cnt + P.dinv_off[s] / (SOLVE_BLK * SOLVE_BLK) + j / SOLVE_BLK, 1u);
                }
                __syncwarp();
            }
            TRACE(5, L, 0);
        }
        // the level's small fronts (independent of its wide fronts; nothing here waits)
        if (sc >= G * (blockDim.x >> 5) / 2) {
            const int wpc = blockDim.x >> 5, warp = threadIdx.x >> 5;
            double* xs = psm + warp * P.warp_smem;
            for (int i = blockIdx.x * wpc + warp; i < sc; i += G * wpc)
                warp_backward_front(P.bw, P.list[so + i], xs, xs + P.warp_xs);
        } else {
            for (int i = blockIdx.x; i < sc; i += G) backward_front(P.bw, P.list[so + i], 0, psm);
        }
        if (lc) {
            // one CTA per (front, block); a CTA takes its blocks of a front in decreasing order, and the
            // owner of block 0 puts the front's solution into Y
            int total = 0;
            for (int i = 0; i < lc; ++i) total += (P.bw.fronts[P.list[lo + i]].w + SOLVE_BLK - 1) / SOLVE_BLK;
            for (int k = blockIdx.x; k < total; k += G) {
                int kk = k;
                for (int i = 0; i < lc; ++i) {
                    const int s = P.list[lo + i];
                    const int nbs = (P.bw.fronts[s].w + SOLVE_BLK - 1) / SOLVE_BLK;
                    if (kk < nbs) {
                        wide_backward_owner(P, s, nbs - 1 - kk, psm);
                        break;
                    }
                    kk -= nbs;
                }
            }
        }
        grid_barrier(P.barrier, epoch, P.status);
        TRACE(7, L, 0);
    }
    // out[perm] = Y (or +=)
    for (int64_t q = gtid; q < n * nrhs; q += gstride) {
        int64_t k = q % n, r = q / n;
        double* o = P.out + P.perm[k] + r * P.ldout;
        if (P.mode == 2) *o += P.fw.Y[q];
        else *o = P.fw.Y[q];
    }
    TRACE(8, 0, 0);
#undef TRACE
}

template <typename T>
int persistent_solve_grid(size_t smem) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, persistent_solve_kernel<T>, SOLVE_THREADS, smem) !=
        cudaSuccess)
        return 0;
    return sms * std::min(per, 2);
}

template <typename T>
cudaError_t launch_persistent_solve(const PersistArgs<T>& a, int grid, size_t smem, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(SOLVE_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, persistent_solve_kernel<T>, a);
}

template cudaError_t launch_persistent_solve<double>(const PersistArgs<double>&, int, size_t, cudaStream_t);
template cudaError_t launch_persistent_solve<float>(const PersistArgs<float>&, int, size_t, cudaStream_t);
template int persistent_solve_grid<double>(size_t);
template int persistent_solve_grid<float>(size_t);

// D^{-1} (1x1 and 2x2 blocks, d[k], d[n + k], d[k + 1]) -- _sv_diag_kernel! sweeps.jl:549-569
__global__ void diag_kernel(DiagArgs A) {
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    const int64_t n = A.n;
    const double* d = A.d + (int64_t)member * 2 * n;
    const int8_t* kind = A.kind + (int64_t)member * n;
    double* Y = A.Y + (int64_t)member * n * A.nrhs;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n * A.nrhs; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = q % n, r = q / n;
        const int kk = kind[k];
        if (A.two && kk == KIND_2X2_SECOND) continue;
        if (A.two && kk == KIND_2X2_FIRST) {
            double a = d[k], b = d[n + k], c = d[k + 1];
            double det = a * c - b * b;
            double y1 = Y[k + r * n], y2 = Y[k + 1 + r * n];
            Y[k + r * n] = (c * y1 - b * y2) / det;
            Y[k + 1 + r * n] = (a * y2 - b * y1) / det;
        } else {
            Y[k + r * n] /= d[k];
        }
    }
}

cudaError_t launch_diag(const DiagArgs& a, int nmembers, cudaStream_t st) {
    int64_t work = a.n * a.nrhs;
    int blocks = (int)std::min<int64_t>((work + 255) / 256, 4096);
    dim3 grid(blocks > 0 ? blocks : 1, nmembers);
    diag_kernel<<<grid, 256, 0, st>>>(a);
    return cudaGetLastError();
}

// Y[k, r] = B[perm[k], r] (mode 0); X[perm[k], r] = Y[k, r] (mode 1); X[perm[k], r] += Y[k, r] (mode 2)
__global__ void permute_kernel(PermArgs A) {
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    const int64_t n = A.n;
    double* Y = A.Y + (int64_t)member * n * A.nrhs;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n * A.nrhs; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = q % n, r = q / n;
        const int64_t g = A.perm ? A.perm[k] : k;
        if (A.mode == 0) {
            Y[q] = A.in[member * A.ldin * A.nrhs + g + r * A.ldin];
        } else if (A.mode == 1) {
            A.out[member * A.ldout * A.nrhs + g + r * A.ldout] = Y[q];
        } else {
            A.out[member * A.ldout * A.nrhs + g + r * A.ldout] += Y[q];
        }
    }
}

cudaError_t launch_permute(const PermArgs& a, int nmembers, cudaStream_t st) {
    int64_t work = a.n * a.nrhs;
    int blocks = (int)std::min<int64_t>((work + 255) / 256, 4096);
    dim3 grid(blocks > 0 ? blocks : 1, nmembers);
    permute_kernel<<<grid, 256, 0, st>>>(a);
    return cudaGetLastError();
}

// R = B - op(A) X over the full-pattern map (duplicates summed in source order); one warp per row
__global__ void residual_kernel(ResidualArgs A) {
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    const int64_t n = A.n;
    const double* nz = A.nzval + (int64_t)member * A.nnz;
    const double* X = A.X + (int64_t)member * A.ldx * A.nrhs;
    const double* B = A.B + (int64_t)member * A.ldb * A.nrhs;
    double* R = A.R + (int64_t)member * n * A.nrhs;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < n; i += nw) {
        for (int r0 = 0; r0 < A.nrhs; r0 += 8) {
            const int rc = min(8, A.nrhs - r0);
            double acc[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) acc[r] = 0.0;
            for (int64_t e = A.rowptr[i] + lane; e < A.rowptr[i + 1]; e += 32) {
                double v = 0.0;
                for (int64_t q = A.srcptr[e]; q < A.srcptr[e + 1]; ++q) v += nz[A.src[q]];
                const int64_t c = A.colval[e];
#pragma unroll
                for (int r = 0; r < 8; ++r)
                    if (r < rc) acc[r] += v * X[c + (int64_t)(r0 + r) * A.ldx];
            }
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                double v = acc[r];
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0 && r < rc) R[i + (int64_t)(r0 + r) * n] = B[i + (int64_t)(r0 + r) * A.ldb] - v;
            }
        }
    }
}

cudaError_t launch_residual(const ResidualArgs& a, int nmembers, cudaStream_t st) {
    int64_t warps = a.n;
    int blocks = (int)std::min<int64_t>((warps * 32 + 255) / 256, 8192);
    dim3 grid(blocks > 0 ? blocks : 1, nmembers);
    residual_kernel<<<grid, 256, 0, st>>>(a);
    return cudaGetLastError();
}

// ||R_k||^2 and ||B_k||^2 per (member, rhs): one CTA each
__global__ void norms_kernel(NormArgs A) {
    const int col = blockIdx.x;  // member-major: col = j * nrhs + r over the active members
    const int j = col / A.nrhs, r = col % A.nrhs;
    const int member = A.members ? A.members[j] : j;
    const int64_t n = A.n;
    const double* R = A.R + (int64_t)member * n * A.nrhs + (int64_t)r * n;
    const double* B = A.B + (int64_t)member * A.ldb * A.nrhs + (int64_t)r * A.ldb;
    __shared__ double sr[256], sb[256];
    double ar = 0.0, ab = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        ar += R[i] * R[i];
        ab += B[i] * B[i];
    }
    sr[threadIdx.x] = ar;
    sb[threadIdx.x] = ab;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            sr[threadIdx.x] += sr[threadIdx.x + h];
            sb[threadIdx.x] += sb[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        A.out[2 * col] = sr[0];
        A.out[2 * col + 1] = sb[0];
    }
}

cudaError_t launch_norms(const NormArgs& a, int ncols, cudaStream_t st) {
    norms_kernel<<<ncols, 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t prepare_solve_kernels(int max_smem) {
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* k) {
        if (e != cudaSuccess) return;
        cudaFuncAttributes fa;
        e = cudaFuncGetAttributes(&fa, k);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem - (int)fa.sharedSizeBytes);
    };
    set((const void*)forward_kernel<double>);
    set((const void*)forward_kernel<float>);
    set((const void*)backward_kernel<double>);
    set((const void*)backward_kernel<float>);
    set((const void*)forward_rect_kernel<double>);
    set((const void*)forward_rect_kernel<float>);
    set((const void*)persistent_solve_kernel<double>);
    set((const void*)persistent_solve_kernel<float>);
    return e;
}

}  // namespace sds

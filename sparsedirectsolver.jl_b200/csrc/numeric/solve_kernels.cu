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

// R = B - op(A) X over the full-pattern map (duplicates summed in source order); one warp per row (long
// rows; residual_rows_kernel below takes maps of short rows)
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

// The same residual with one thread per row, for maps of short rows (a warp per row leaves most lanes
// idle and holds one row's dependent loads in flight per warp): each row's entries summed in order.
__global__ void residual_rows_kernel(ResidualArgs A) {
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    const int64_t n = A.n;
    const double* nz = A.nzval + (int64_t)member * A.nnz;
    const double* X = A.X + (int64_t)member * A.ldx * A.nrhs;
    const double* B = A.B + (int64_t)member * A.ldb * A.nrhs;
    double* R = A.R + (int64_t)member * n * A.nrhs;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e0 = A.rowptr[i], e1 = A.rowptr[i + 1];
        for (int r0 = 0; r0 < A.nrhs; r0 += 8) {
            const int rc = min(8, A.nrhs - r0);
            double acc[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) acc[r] = 0.0;
            for (int64_t e = e0; e < e1; ++e) {
                double v = 0.0;
                for (int64_t q = A.srcptr[e]; q < A.srcptr[e + 1]; ++q) v += nz[A.src[q]];
                const int64_t c = A.colval[e];
#pragma unroll
                for (int r = 0; r < 8; ++r)
                    if (r < rc) acc[r] += v * X[c + (int64_t)(r0 + r) * A.ldx];
            }
#pragma unroll
            for (int r = 0; r < 8; ++r)
                if (r < rc) R[i + (int64_t)(r0 + r) * n] = B[i + (int64_t)(r0 + r) * A.ldb] - acc[r];
        }
    }
}

cudaError_t launch_residual(const ResidualArgs& a, int nmembers, cudaStream_t st) {
    if (a.n > 0 && a.entries <= 16 * a.n) {   // rows of at most 16 entries on average
        int blocks = (int)std::min<int64_t>((a.n + 255) / 256, 8192);
        dim3 grid(blocks > 0 ? blocks : 1, nmembers);
        residual_rows_kernel<<<grid, 256, 0, st>>>(a);
        return cudaGetLastError();
    }
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
    return e;
}

}  // namespace sds

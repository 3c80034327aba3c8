// Dataflow solve: one persistent cooperative launch for a whole solve of one system, without grid
// barriers (forward_sweep! / diagonal_sweep! / backward_sweep! and the permutations of
// src/solve/sweeps.jl:908-1004 and src/solve/permute.jl:117-148, for one right-hand-side group).
//
// The work is a list of tasks in a topological order of the elimination tree (solve.cuh). Every CTA
// takes the next task from one atomic counter. A task waits only for tasks earlier in the list:
//  * a front's forward waits for its children's forward tasks (a counter per front);
//  * a front's backward waits for its parent's backward (a flag per front), or at a root for its own
//    forward tasks;
//  * inside a tiled front, on per-block flags and partial counters of tasks of the same front that
//    come earlier in the list.
// All CTAs are resident (cooperative launch) and each runs one task at a time, so the earliest
// unfinished task can always run and the launch cannot deadlock. Every wait is bounded (about two
// seconds); a wait that gives up records the status word and every later wait returns at once.
//
// The triangular solves of a front use precomputed inverses of its diagonal blocks (L11^-1 of a warp
// front, the 64 x 64 diagonal-block inverses of a tiled front), so a front's solve is a few
// independent dot products instead of a column-by-column chain. Everything static that a task needs
// after its wait (panel entries, inverses, contribution lists, right-hand-side entries, row indices)
// is read, or prefetched into L2, before the wait: on the critical path only the data produced by the
// awaited tasks is read.
//
// Vectors are FP64 whatever the factor precision (an FP32 factor is read and widened).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"
#include "solve.cuh"

namespace sds {

static_assert(DF_THREADS >= DF_CHUNK && 4 * 32 == DF_CHUNK, "a backward partial task: one update row per thread, 32 per quarter");
static_assert(DF_THREADS == 4 * DF_BLK, "a tiled task has four threads per row of a 64-row tile");

namespace {

__device__ __forceinline__ uint64_t df_clock() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Spin (one thread) until *p >= target. Bounded: gives up after ~2 s, or at once once any wait of the
// launch has given up, and then records the failure in the status word. The first few thousand polls
// spin without sleeping (the waits on the critical path are short); the acquire load orders this
// thread's later reads, and the CTA or warp barrier after the call orders the other threads'.
__device__ __noinline__ void df_wait(const unsigned int* p, unsigned int target, int32_t* status) {
    unsigned int v;
    uint64_t t0 = 0;
    for (long spins = 0;; ++spins) {
        asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
        if (v >= target) break;
        if ((spins & 255) == 0) {
            if (*(volatile int32_t*)status != 0) return;
            const uint64_t now = df_clock();
            if (spins == 0) t0 = now;
            else if (now - t0 > 2000000000ull) {
                atomicExch(status, 1);
                return;
            }
        }
        if (spins > 4096) __nanosleep(64);
    }
}

__device__ __forceinline__ void df_release(unsigned int* p, unsigned int v) {
    asm volatile("st.release.gpu.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// counter increment with release semantics (no fence of its own)
__device__ __forceinline__ void df_release_add(unsigned int* p) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(p) : "memory");
}

// publish: the CTA's writes, then one thread's release of the flag (or release increment of the
// counter); the barrier orders the other threads' writes before that thread's release
__device__ __forceinline__ void df_publish_cta(unsigned int* p, unsigned int v, bool add) {
    __syncthreads();
    if (threadIdx.x == 0) {
        if (add) df_release_add(p);
        else df_release(p, v);
    }
}

// x[r] for the 4 lanes of a quarter group (lanes 4i .. 4i + 3): the sum over the group
__device__ __forceinline__ double quad_sum(double v) {
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    return v;
}

// y = D^{-1} z at factor position g (1x1 pivots, and the 2x2 blocks of LDLT: a = d[k], b = d[n + k],
// c = d[k + 1] of the block's first position k) for right-hand side r, z read from Z (n x nrhs: Y, or
// xtmp for an inverse-panel front)
template <typename T>
__device__ __forceinline__ double df_dinv(const DataflowArgs<T>& A, const double* Z, int64_t g, int r) {
    const int64_t n = A.n;
    const double y = Z[g + r * n];
    if (A.diag_mode == 0) return y;
    if (A.diag_mode == 1) return y / A.d[g];
    const int kk = A.kind[g];
    if (kk == KIND_2X2_FIRST) {
        const double a = A.d[g], b = A.d[n + g], c = A.d[g + 1];
        const double det = a * c - b * b;
        return (c * y - b * Z[g + 1 + r * n]) / det;
    }
    if (kk == KIND_2X2_SECOND) {
        const double a = A.d[g - 1], b = A.d[n + g - 1], c = A.d[g];
        const double det = a * c - b * b;
        return (a * y - b * Z[g - 1 + r * n]) / det;
    }
    return y / A.d[g];
}

// L2 prefetch of bytes [p, p + bytes), one 128-byte line per step of `step` threads starting at t0
__device__ __forceinline__ void df_prefetch_l2(const void* p, int64_t bytes, int t0, int step) {
    const char* c = static_cast<const char*>(p);
    for (int64_t o = (int64_t)t0 * 128; o < bytes; o += (int64_t)step * 128)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(c + o));
}

// The contributions of the children to one front row, read before the children are done: the row's
// range in the contribution lists and its first four sources (global update rows)
struct RowPull {
    int32_t e0, e1;
    int32_t g[4];
};

__device__ __forceinline__ RowPull df_row_pull_prep(const int32_t* rptr, const int32_t* csrc, int64_t at) {
    RowPull rp;
    rp.e0 = rptr[at];
    rp.e1 = rptr[at + 1];
#pragma unroll
    for (int k = 0; k < 4; ++k) rp.g[k] = rp.e0 + k < rp.e1 ? csrc[rp.e0 + k] : -1;
    return rp;
}

// acc[r] -= sum of the row's contributions (right-hand sides r < nrhs), in list order; the first four
// sources come from the preparation, the rest (rare) are read here
template <int NR>
__device__ __forceinline__ void df_row_pull(const RowPull& rp, const int32_t* csrc, const double* U, int nrhs,
                                            double* acc) {
    double v[4][NR];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int r = 0; r < NR; ++r) v[k][r] = (rp.g[k] >= 0 && r < nrhs) ? U[(int64_t)rp.g[k] * nrhs + r] : 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (rp.g[k] >= 0) {
#pragma unroll
            for (int r = 0; r < NR; ++r) acc[r] -= v[k][r];
        }
    for (int e = rp.e0 + 4; e < rp.e1; ++e) {
        const int64_t g = csrc[e];
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) acc[r] -= U[g * nrhs + r];
    }
}

// ---------------------------------------------------------------------------------------------------
// warp fronts (w <= 32, f <= DF_WARP_F); z: f x nrhs doubles of shared memory (ld f)

template <typename T, int NR>
__device__ __noinline__ void df_warp_forward(const DataflowArgs<T>& A, int s, double* z, int64_t* stamp) {
    const DFront fd = A.fronts[s];
    const DfFront q = A.df[s];
    const int f = fd.f, w = fd.w, m = f - w, nrhs = A.nrhs, lane = threadIdx.x & 31;
    const int64_t n = A.n;
    const T* L = A.facf + fd.panel;
    const T* Iv = A.invf + q.inv;
    // before the children are done: the inverse row, the right-hand side of the own row, the
    // contribution lists of the lane's rows, and the panel into L2
    double iv[DF_WARP_W];
#pragma unroll
    for (int j = 0; j < DF_WARP_W; ++j) iv[j] = (lane < w && j < w) ? (double)Iv[lane + (int64_t)w * j] : 0.0;
    double acc[4][NR];
    RowPull rp[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int p = lane + 32 * k;
        rp[k] = p < f ? df_row_pull_prep(A.rptr, A.csrc, (int64_t)q.rbase + p) : RowPull{0, 0, {-1, -1, -1, -1}};
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[k][r] = 0.0;
    }
    if (lane < w) {
        const int64_t src = A.perm[fd.c0 + lane];
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) acc[0][r] = A.in[src + r * A.ldin];
    }
    df_prefetch_l2(L + w, (int64_t)(f * w - w) * sizeof(T), lane, 32);
    if (q.fneed > 0) {
        if (lane == 0) df_wait(A.fcnt + s, (unsigned)q.fneed, A.status);
        __syncwarp();
    }
    if (stamp && lane == 0) *stamp = (int64_t)df_clock();
    // own rows z1 = b - children's updates, update rows u = sum of the children's updates (stored negated
    // like the own rows: z = -u, so that both take -= below); every row's loads before any store
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (lane + 32 * k < f) df_row_pull<NR>(rp[k], A.csrc, A.U, nrhs, acc[k]);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int p = lane + 32 * k;
        if (p < f) {
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) z[p + r * f] = acc[k][r];
        }
    }
    __syncwarp();
    double x[NR];
    if (A.reorder_fw) {
        const int src = lane < w ? A.piv[fd.c0 + lane] - 1 - fd.c0 : 0;
#pragma unroll
        for (int r = 0; r < NR; ++r) x[r] = (lane < w && r < nrhs) ? z[src + r * f] : 0.0;
        __syncwarp();
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (lane < w && r < nrhs) z[lane + r * f] = x[r];
        __syncwarp();
    }
    // x1 = L11^-1 z1 (lane i: row i)
#pragma unroll
    for (int r = 0; r < NR; ++r) x[r] = 0.0;
#pragma unroll
    for (int j = 0; j < DF_WARP_W; ++j) {
        if (j < w) {
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) x[r] += iv[j] * z[j + r * f];
        }
    }
    __syncwarp();
    if (lane < w) {
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) {
                z[lane + r * f] = x[r];
                A.Y[fd.c0 + lane + r * n] = x[r];
            }
    }
    __syncwarp();
    // u = (children's updates) + L21 x1: z holds -u, so u = -(z - L21 x1). The lane's rows (up to four)
    // take the panel in column groups of 8 with no store in between, so the loads of every group can be
    // in flight together; the results are stored at the end.
    if (m > 0) {
        double* u = A.U + (int64_t)q.urow * nrhs;
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int r = 0; r < NR; ++r)
                acc[k][r] = (lane + 32 * k < m && r < nrhs) ? -z[w + lane + 32 * k + r * f] : 0.0;
        for (int j = 0; j < w; j += 8) {
            double lv[4][8];
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int e = 0; e < 8; ++e)
                    lv[k][e] = (lane + 32 * k < m && j + e < w) ? (double)L[w + lane + 32 * k + (int64_t)(j + e) * f] : 0.0;
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int e = 0; e < 8; ++e)
                    if (j + e < w) {
#pragma unroll
                        for (int r = 0; r < NR; ++r)
                            if (r < nrhs) acc[k][r] += lv[k][e] * z[j + e + r * f];
                    }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (lane + 32 * k < m) {
#pragma unroll
                for (int r = 0; r < NR; ++r)
                    if (r < nrhs) u[(int64_t)(lane + 32 * k) * nrhs + r] = acc[k][r];
            }
    }
    __syncwarp();
    if (lane == 0) df_release_add(A.fcnt + (fd.parent >= 0 ? fd.parent : s));
    __syncwarp();
}

template <typename T, int NR>
__device__ __noinline__ void df_warp_backward(const DataflowArgs<T>& A, int s, double* z, int64_t* stamp) {
    const DFront fd = A.fronts[s];
    const DfFront q = A.df[s];
    const int f = fd.f, w = fd.w, m = f - w, nrhs = A.nrhs, lane = threadIdx.x & 31;
    const int64_t n = A.n;
    const T* L = A.facb + fd.panel;
    const T* Iv = A.invb + q.inv;
    // before the parent is done: column `lane` of the inverse (x1 = L11^-T y: x1[j] = sum_i inv[i, j]
    // y[i]), the rows of x2 this lane gathers, the first 16 entries of its panel column, and the panel
    // into L2
    double iv[DF_WARP_W];
#pragma unroll
    for (int i = 0; i < DF_WARP_W; ++i) iv[i] = (lane < w && i < w) ? (double)Iv[i + (int64_t)w * lane] : 0.0;
    const int32_t* rows = A.rowval + fd.row_begin + w;
    int32_t ridx[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) ridx[k] = lane + 32 * k < m ? rows[lane + 32 * k] : 0;
    df_prefetch_l2(L + w, (int64_t)(f * w - w) * sizeof(T), lane, 32);
    const T* Lc = L + w + (int64_t)lane * f;
    double lv0[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) lv0[e] = (lane < w && e < m) ? (double)Lc[e] : 0.0;
    const unsigned pbsig = fd.parent >= 0 ? (unsigned)A.df[fd.parent].bsig : 0u;
    if (lane == 0) {
        if (fd.parent >= 0) df_wait(A.bdone + fd.parent, pbsig, A.status);
        else df_wait(A.fcnt + s, (unsigned)(q.fneed + q.fsig), A.status);
        if (stamp) *stamp = (int64_t)df_clock();
    }
    __syncwarp();
    double y[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) y[r] = (lane < w && r < nrhs) ? df_dinv(A, A.Y, fd.c0 + lane, r) : 0.0;
    // x2: the solution at the rows below the front's columns (final: every ancestor is done)
    double* x2 = z;                 // m x nrhs
    double* ys = z + m * nrhs;      // w x nrhs
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (lane + 32 * k < m) {
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) x2[lane + 32 * k + r * m] = A.Y[ridx[k] + r * n];
        }
    __syncwarp();
    // y1 -= L21^T x2 (lane j: column j, contiguous); the first 16 rows were read before the wait
    if (lane < w && m > 0) {
#pragma unroll
        for (int e = 0; e < 16; ++e)
            if (e < m) {
#pragma unroll
                for (int r = 0; r < NR; ++r)
                    if (r < nrhs) y[r] -= lv0[e] * x2[e + r * m];
            }
        for (int i = 16; i < m; i += 32) {
            double lv[32];
#pragma unroll
            for (int e = 0; e < 32; ++e) lv[e] = i + e < m ? (double)Lc[i + e] : 0.0;
#pragma unroll
            for (int e = 0; e < 32; ++e)
                if (i + e < m) {
#pragma unroll
                    for (int r = 0; r < NR; ++r)
                        if (r < nrhs) y[r] -= lv[e] * x2[i + e + r * m];
                }
        }
    }
#pragma unroll
    for (int r = 0; r < NR; ++r)
        if (lane < w && r < nrhs) ys[lane + r * w] = y[r];
    __syncwarp();
    double x[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) x[r] = 0.0;
#pragma unroll
    for (int i = 0; i < DF_WARP_W; ++i) {
        if (i < w) {
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) x[r] += iv[i] * ys[i + r * w];
        }
    }
    if (lane < w) {
        const int64_t dst = A.reorder_bw ? A.piv[fd.c0 + lane] - 1 : fd.c0 + lane;
        const int64_t o = A.perm[dst];
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) {
                A.Y[dst + r * n] = x[r];
                double* op = A.out + o + r * A.ldout;
                if (A.mode == 2) *op += x[r];
                else *op = x[r];
            }
    }
    __syncwarp();
    if (lane == 0) df_release(A.bdone + s, 1u);
    __syncwarp();
}

// ---------------------------------------------------------------------------------------------------
// tiled fronts; 256 threads: thread (i = tid / 4, qq = tid % 4) owns row i of a 64-row tile (or column
// i of a 64-column block) and one quarter (16 entries) of each 64-entry dot product. Shared memory:
// xs and zs (64 x NR each), x2 (DF_CHUNK x NR) doubles.

template <typename T, int NR>
__device__ __noinline__ void df_tile_forward(const DataflowArgs<T>& A, int s, int t, double* sm, int64_t* stamp) {
    const DFront fd = A.fronts[s];
    const DfFront q = A.df[s];
    const int f = fd.f, w = fd.w, nrhs = A.nrhs, tid = threadIdx.x;
    const int64_t n = A.n;
    const int K = q.nblk;
    const int i = tid >> 2, qq = tid & 3, lane = tid & 31;
    const int row = DF_BLK * t + i;
    const bool valid = row < f;
    const T* L = A.facf + fd.panel;
    const T* Iv = A.invf + q.inv;
    double* xs = sm;
    double* zs = sm + DF_BLK * NR;
    const bool recompute = K == 1 && t > 0;   // one block: every tile recomputes x_0 from the own rows
    // before the children are done: the inverse (block t, or block 0 to recompute x_0), the tile row's
    // right-hand side and contribution lists (qq == 0), the own row's for the recompute (qq == 1)
    const int ivb = t < K ? t : 0;
    const int ivw = min(DF_BLK, w - DF_BLK * ivb);
    double iv[16];
#pragma unroll
    for (int jj = 0; jj < 16; ++jj)
        iv[jj] = ((t < K || recompute) && i < ivw && 16 * qq + jj < ivw)
                     ? (double)Iv[(int64_t)ivb * DF_BLK * DF_BLK + i + DF_BLK * (16 * qq + jj)] : 0.0;
    double val[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) val[r] = 0.0;
    RowPull rp{0, 0, {-1, -1, -1, -1}};
    const int prow = qq == 0 ? row : i;   // qq == 1 with the recompute: own row i
    const bool puller = (qq == 0 && valid) || (qq == 1 && recompute && i < w);
    if (puller) {
        // an own row in the local pivot order takes the natural row piv[c0 + k] - 1 - c0
        const int srow = (prow < w && A.reorder_fw) ? A.piv[fd.c0 + prow] - 1 - fd.c0 : prow;
        rp = df_row_pull_prep(A.rptr, A.csrc, (int64_t)q.rbase + srow);
        if (srow < w) {
            const int64_t src = A.perm[fd.c0 + srow];
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) val[r] = A.in[src + r * A.ldin];
        }
    }
    // row `row`'s 16 entries (this thread's quarter) of block k below the block's own rows; block 0's
    // are read before the wait, each later block's before the wait for its solution
    auto load_lv = [&](int k, double* lv) {
        const int bwk = min(DF_BLK, w - DF_BLK * k);
        const int col0 = DF_BLK * k + 16 * qq;
#pragma unroll
        for (int jj = 0; jj < 16; ++jj)
            lv[jj] = (valid && row >= DF_BLK * k + bwk && 16 * qq + jj < bwk) ? (double)L[row + (int64_t)(col0 + jj) * f] : 0.0;
    };
    double lv[16];
    load_lv(0, lv);
    if (tid == 0 && q.fneed > 0) df_wait(A.fcnt + s, (unsigned)q.fneed, A.status);
    __syncthreads();
    if (stamp && tid == 0) *stamp = (int64_t)df_clock();
    if (puller) df_row_pull<NR>(rp, A.csrc, A.U, nrhs, val);
    if (qq == 1 && recompute) {
#pragma unroll
        for (int r = 0; r < NR; ++r) zs[i + DF_BLK * r] = (i < w && r < nrhs) ? val[r] : 0.0;
    }
    // the tile's values: own rows z (to be solved), update rows -u (so that every row takes -= L x)
#pragma unroll
    for (int r = 0; r < NR; ++r) val[r] = __shfl_sync(0xffffffffu, val[r], lane & ~3);
    const int kmax = min(t, K - 1);
    for (int k = 0; k <= kmax; ++k) {
        const int bw = min(DF_BLK, w - DF_BLK * k);
        if (k > 0) load_lv(k, lv);
        if (k == t) {
            // the diagonal block: x_t = inv_tt z_t
            if (qq == 0) {
#pragma unroll
                for (int r = 0; r < NR; ++r) zs[i + DF_BLK * r] = (i < bw) ? val[r] : 0.0;
            }
            __syncthreads();
            double x[NR];
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                double acc = 0.0;
                if (r < nrhs) {
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) acc += iv[jj] * zs[16 * qq + jj + DF_BLK * r];
                }
                x[r] = quad_sum(acc);
            }
            if (qq == 0) {
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    xs[i + DF_BLK * r] = (i < bw) ? x[r] : 0.0;
                    if (i < bw && r < nrhs) {
                        A.Y[fd.c0 + DF_BLK * t + i + r * n] = x[r];
                        if (K > 1) A.xtmp[fd.c0 + DF_BLK * t + i + r * n] = x[r];
                    }
                }
            }
            if (K > 1) df_publish_cta(A.xflag + q.blk + t, 1u, false);
            else __syncthreads();
            // update rows of this tile below the front's columns (a tile that straddles w)
            if (DF_BLK * t + DF_BLK > w) {
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    double acc = 0.0;
                    if (r < nrhs) {
#pragma unroll
                        for (int jj = 0; jj < 16; ++jj) acc += lv[jj] * xs[16 * qq + jj + DF_BLK * r];
                    }
                    acc = quad_sum(acc);
                    if (row >= w) val[r] -= acc;
                }
            }
            __syncthreads();
        } else {
            if (recompute) {
                __syncthreads();   // zs complete
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    double acc = 0.0;
                    if (r < nrhs) {
#pragma unroll
                        for (int jj = 0; jj < 16; ++jj) acc += iv[jj] * zs[16 * qq + jj + DF_BLK * r];
                    }
                    acc = quad_sum(acc);
                    if (qq == 0) xs[i + DF_BLK * r] = (i < bw) ? acc : 0.0;
                }
            } else {
                if (tid == 0) df_wait(A.xflag + q.blk + k, 1u, A.status);
                __syncthreads();
                for (int idx = tid; idx < DF_BLK * NR; idx += blockDim.x) {
                    const int jr = idx % DF_BLK, r = idx / DF_BLK;
                    xs[idx] = (jr < bw && r < nrhs) ? A.xtmp[fd.c0 + DF_BLK * k + jr + r * n] : 0.0;
                }
            }
            __syncthreads();
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                double acc = 0.0;
                if (r < nrhs) {
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) acc += lv[jj] * xs[16 * qq + jj + DF_BLK * r];
                }
                val[r] -= quad_sum(acc);
            }
            __syncthreads();
        }
    }
    if (qq == 0 && valid && row >= w) {
        double* u = A.U + ((int64_t)q.urow + row - w) * nrhs;
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) u[r] = -val[r];
    }
    df_publish_cta(A.fcnt + (fd.parent >= 0 ? fd.parent : s), 0u, true);
}

// -L21^T x2 of block b over the update rows [r0, r0 + cnt) into `acc` (thread: column j of the block,
// rows 4 ii + qq of the chunk); x2 staged in shared memory (ld DF_CHUNK)
template <typename T, int NR>
__device__ __forceinline__ void df_block_l21t(const T* L, int f, int w, int b, int bw, int r0, int cnt, const double* x2,
                                              int nrhs, double* acc) {
    const int j = threadIdx.x >> 2, qq = threadIdx.x & 3;
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = 0.0;
    if (j < bw) {
        const T* Lc = L + w + r0 + (int64_t)(DF_BLK * b + j) * f;
        for (int i0 = qq; i0 < cnt; i0 += 64) {
            double lv[16];
#pragma unroll
            for (int e = 0; e < 16; ++e) lv[e] = (i0 + 4 * e < cnt) ? (double)Lc[i0 + 4 * e] : 0.0;
#pragma unroll
            for (int e = 0; e < 16; ++e)
#pragma unroll
                for (int r = 0; r < NR; ++r)
                    if (r < nrhs && i0 + 4 * e < cnt) acc[r] += lv[e] * x2[i0 + 4 * e + DF_CHUNK * r];
        }
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = quad_sum(acc[r]);
}

// L2 prefetch of the rows [r0, r0 + cnt) below the front's columns of block b's columns
template <typename T>
__device__ __forceinline__ void df_prefetch_block_rows(const T* L, int f, int w, int b, int bw, int r0, int cnt) {
    const int j = threadIdx.x >> 2, qq = threadIdx.x & 3;
    if (j < bw) df_prefetch_l2(L + w + r0 + (int64_t)(DF_BLK * b + j) * f, (int64_t)cnt * sizeof(T), qq, 4);
}

template <typename T, int NR>
__device__ __noinline__ void df_tiled_part(const DataflowArgs<T>& A, int s, int b, int c, double* sm, int64_t* stamp) {
    const DFront fd = A.fronts[s];
    const DfFront q = A.df[s];
    const int f = fd.f, w = fd.w, m = f - w, nrhs = A.nrhs, tid = threadIdx.x;
    const int64_t n = A.n;
    const int bw = min(DF_BLK, w - DF_BLK * b), r0 = DF_CHUNK * c, cnt = min(DF_CHUNK, m - r0);
    const int j = tid >> 2, qq = tid & 3;
    const T* L = A.facb + fd.panel;
    double* x2 = sm + 2 * DF_BLK * NR;
    // before the parent is done: this thread's 32 entries of column j of the block (rows qq + 4 e of
    // the chunk) and the chunk's row indices
    double lv[DF_CHUNK / 4];
    const T* Lc = L + w + r0 + (int64_t)(DF_BLK * b + j) * f;
#pragma unroll
    for (int e = 0; e < DF_CHUNK / 4; ++e) lv[e] = (j < bw && qq + 4 * e < cnt) ? (double)Lc[qq + 4 * e] : 0.0;
    const int32_t ridx = tid < cnt ? A.rowval[fd.row_begin + w + r0 + tid] : 0;
    const unsigned pbsig = (unsigned)A.df[fd.parent].bsig;
    if (tid == 0) {
        df_wait(A.bdone + fd.parent, pbsig, A.status);
        if (stamp) *stamp = (int64_t)df_clock();
    }
    __syncthreads();
    if (tid < DF_CHUNK) {
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) x2[tid + DF_CHUNK * r] = tid < cnt ? A.Y[ridx + r * n] : 0.0;
    }
    __syncthreads();
    double acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        double a = 0.0;
        if (r < nrhs) {
#pragma unroll
            for (int e = 0; e < DF_CHUNK / 4; ++e) a += lv[e] * x2[qq + 4 * e + DF_CHUNK * r];
        }
        acc[r] = quad_sum(a);
    }
    if (qq == 0 && j < bw) {
        double* p = A.part + ((int64_t)q.part + (int64_t)b * q.nchunk + c) * (DF_BLK * NR);
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) p[j + DF_BLK * r] = acc[r];
    }
    df_publish_cta(A.pcnt + q.blk + b, 0u, true);
}

template <typename T, int NR>
__device__ __noinline__ void df_tiled_owner(const DataflowArgs<T>& A, int s, int b, double* sm, int64_t* stamp) {
    const DFront fd = A.fronts[s];
    const DfFront q = A.df[s];
    const int f = fd.f, w = fd.w, m = f - w, nrhs = A.nrhs, tid = threadIdx.x, nt = blockDim.x;
    const int64_t n = A.n;
    const int K = q.nblk, C = q.nchunk;
    const int bw = min(DF_BLK, w - DF_BLK * b);
    const int j = tid >> 2, qq = tid & 3;
    const T* L = A.facb + fd.panel;
    const T* Ib = A.invb + q.inv + (int64_t)b * DF_BLK * DF_BLK;
    double* xs = sm;
    double* ys = sm + DF_BLK * NR;
    double* x2 = sm + 2 * DF_BLK * NR;
    // before the wait: column j of inv_bb, rows 4 ii + qq (x_b = inv_bb^T y_b); the later blocks' rows
    // of this block's columns into L2; with the update rows summed here (m <= DF_CHUNK), their indices
    // and their rows of this block's columns
    double iv[16];
#pragma unroll
    for (int ii = 0; ii < 16; ++ii)
        iv[ii] = (j < bw && 4 * ii + qq < bw) ? (double)Ib[4 * ii + qq + (int64_t)DF_BLK * j] : 0.0;
    if (j < bw)
        for (int tt = b + 1; tt < K; ++tt)
            df_prefetch_l2(L + DF_BLK * tt + (int64_t)(DF_BLK * b + j) * f, (int64_t)min(DF_BLK, f - DF_BLK * tt) * sizeof(T),
                           qq, 4);
    const bool inline_part = C == 0 && m > 0;
    const int32_t ridx = (inline_part && tid < m) ? A.rowval[fd.row_begin + w + tid] : 0;
    if (inline_part) df_prefetch_block_rows(L, f, w, b, bw, 0, m);
    const unsigned pbsig = fd.parent >= 0 ? (unsigned)A.df[fd.parent].bsig : 0u;
    if (tid == 0) {
        if (C > 0) df_wait(A.pcnt + q.blk + b, (unsigned)C, A.status);
        else if (fd.parent >= 0) df_wait(A.bdone + fd.parent, pbsig, A.status);
        else df_wait(A.fcnt + s, (unsigned)(q.fneed + q.fsig), A.status);
        if (stamp) *stamp = (int64_t)df_clock();
    }
    __syncthreads();
    // y_b = D^-1 (forward result) - L21^T x2 of the block
    for (int idx = tid; idx < DF_BLK * NR; idx += nt) {
        const int jr = idx % DF_BLK, r = idx / DF_BLK;
        double v = 0.0;
        if (jr < bw && r < nrhs) {
            v = df_dinv(A, A.Y, fd.c0 + DF_BLK * b + jr, r);
            for (int c = 0; c < C; ++c)
                v -= A.part[((int64_t)q.part + (int64_t)b * C + c) * (DF_BLK * NR) + jr + DF_BLK * r];
        }
        ys[idx] = v;
    }
    if (inline_part) {
        if (tid < DF_CHUNK) {
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) x2[tid + DF_CHUNK * r] = tid < m ? A.Y[ridx + r * n] : 0.0;
        }
        __syncthreads();
        double acc[NR];
        df_block_l21t<T, NR>(L, f, w, b, bw, 0, m, x2, nrhs, acc);
        if (qq == 0 && j < bw) {
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) ys[j + DF_BLK * r] -= acc[r];
        }
    }
    __syncthreads();
    // the later blocks of the front, as their owners publish them
    for (int tt = K - 1; tt > b; --tt) {
        const int bwt = min(DF_BLK, w - DF_BLK * tt);
        double lv[16];
#pragma unroll
        for (int ii = 0; ii < 16; ++ii)
            lv[ii] = (j < bw && 4 * ii + qq < bwt) ? (double)L[DF_BLK * tt + 4 * ii + qq + (int64_t)(DF_BLK * b + j) * f] : 0.0;
        if (tid == 0) df_wait(A.xflag + q.blk + tt, 2u, A.status);
        __syncthreads();
        for (int idx = tid; idx < DF_BLK * NR; idx += nt) {
            const int ir = idx % DF_BLK, r = idx / DF_BLK;
            xs[idx] = (ir < bwt && r < nrhs) ? A.xtmp[fd.c0 + DF_BLK * tt + ir + r * n] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            double acc = 0.0;
            if (r < nrhs) {
#pragma unroll
                for (int ii = 0; ii < 16; ++ii) acc += lv[ii] * xs[4 * ii + qq + DF_BLK * r];
            }
            acc = quad_sum(acc);
            if (qq == 0 && j < bw && r < nrhs) ys[j + DF_BLK * r] -= acc;
        }
        __syncthreads();
    }
    // x_b = inv_bb^T y_b
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        double acc = 0.0;
        if (r < nrhs) {
#pragma unroll
            for (int ii = 0; ii < 16; ++ii) acc += iv[ii] * ys[4 * ii + qq + DF_BLK * r];
        }
        acc = quad_sum(acc);
        if (qq == 0 && j < bw && r < nrhs) A.xtmp[fd.c0 + DF_BLK * b + j + r * n] = acc;
    }
    if (b > 0) {
        df_publish_cta(A.xflag + q.blk + b, 2u, false);
        return;
    }
    __syncthreads();
    // block 0 ends the front's chain (every later block was acquired above): the front's solution
    // goes into Y (local pivot order undone) and into X
    for (int idx = tid; idx < w * nrhs; idx += nt) {
        const int k = idx % w, r = idx / w;
        const double v = A.xtmp[fd.c0 + k + (int64_t)r * n];
        const int64_t dst = A.reorder_bw ? A.piv[fd.c0 + k] - 1 : fd.c0 + k;
        A.Y[dst + r * n] = v;
        double* op = A.out + A.perm[dst] + r * A.ldout;
        if (A.mode == 2) *op += v;
        else *op = v;
    }
    df_publish_cta(A.bdone + s, 1u, false);
}

// ---------------------------------------------------------------------------------------------------
// inverse-panel fronts: P = [L11^-1; L21 L11^-1] (f x w, ld f) of the front's panel; the part of L11^-1
// above its diagonal is never read (masked by index)

// Called by every thread after the CTA wrote its partial product: the counter of the tile (or block)
// counts the tasks done (one acquire-release increment per task); true in the CTA that arrived last,
// after the other tasks' partials are visible
__device__ __forceinline__ bool df_last_arrival(unsigned int* cnt, unsigned count, int* flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned old;
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(cnt) : "memory");
        *flag = old + 1 == count;
    }
    __syncthreads();
    return *flag != 0;
}

// one halving step of a cross-lane reduction of NV values: lanes with bit O set keep the upper half
template <int NV, int O>
__device__ __forceinline__ void df_fold(double* v, int lane) {
    const bool upper = (lane & O) != 0;
#pragma unroll
    for (int i = 0; i < NV / 2; ++i) {
        const double send = upper ? v[i] : v[i + NV / 2];
        const double keep = upper ? v[i + NV / 2] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, O);
    }
}

// the warp sums of NV (a power of two, <= 32) values per lane: lane l returns the sum over the warp of
// value l / (32 / NV), in a fixed order
template <int NV>
__device__ __forceinline__ double df_lane_reduce(double* v, int lane) {
    if constexpr (NV >= 2) df_fold<NV, 16>(v, lane); else v[0] += __shfl_xor_sync(0xffffffffu, v[0], 16);
    if constexpr (NV >= 4) df_fold<NV / 2, 8>(v, lane); else v[0] += __shfl_xor_sync(0xffffffffu, v[0], 8);
    if constexpr (NV >= 8) df_fold<NV / 4, 4>(v, lane); else v[0] += __shfl_xor_sync(0xffffffffu, v[0], 4);
    if constexpr (NV >= 16) df_fold<NV / 8, 2>(v, lane); else v[0] += __shfl_xor_sync(0xffffffffu, v[0], 2);
    if constexpr (NV >= 32) df_fold<NV / 16, 1>(v, lane); else v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
    return v[0];
}

// Forward of an inverse-panel front, row tile t (64 rows) times column chunk kc of P:
// [x1; u] = P z1 + [0; children's updates], z1 = the own rows' right-hand side minus the children's
// updates (local pivot order). 256 threads: thread (i = tid % 64, g = tid / 64) takes row i of the tile
// over 32 columns of the chunk; the four groups' sums add in order. With several chunks the tasks write
// partial products and the last one sums them in chunk order. x1 goes to xtmp (the backward reads it
// there), u to the update vectors.
template <typename T, int NR>
__device__ __noinline__ void df_pinv_forward(const DataflowArgs<T>& A, int s, int t, int cc, double* sm, int64_t* stamp) {
    __shared__ int last;
    const DFront fd = A.fronts[s];
    const DfFront q = A.df[s];
    const int f = fd.f, w = fd.w, nrhs = A.nrhs, tid = threadIdx.x;
    const int64_t n = A.n;
    const int kc = cc & 255, slot0 = cc >> 8;
    const int nkc = df_pf_chunks(w, t);
    const int i = tid & (DF_BLK - 1), g = tid >> 6;
    const int row = DF_BLK * t + i;
    const int col0 = DF_PCOLS * kc;
    const int ncol = min(DF_PCOLS, w - col0);
    const T* Pm = A.invf + q.inv;
    double* zs = sm;                          // DF_PCOLS x NR: z1 over the chunk's columns
    double* red = zs + DF_PCOLS * NR;         // NR x 4 x 64: the column groups' sums
    double* pass = red + 4 * DF_BLK * NR;     // 64 x NR: the tile's update rows, minus the children's updates
    // before the children are done: the thread's 32 entries of P, the chunk's own rows' right-hand side
    // and contribution lists (threads < ncol), with the first chunk the contribution lists of the tile's
    // update rows (threads DF_PCOLS + i)
    T pv[32];
#pragma unroll
    for (int e = 0; e < 32; ++e) {
        const int col = col0 + 32 * g + e;
        pv[e] = (row < f && col < w && (row >= w || col <= row)) ? Pm[row + (int64_t)col * f] : T(0);
    }
    const int prow = tid < DF_PCOLS ? col0 + tid : DF_BLK * t + (tid - DF_PCOLS);
    const bool own = tid < ncol;
    const bool thru = kc == 0 && tid >= DF_PCOLS && tid < DF_PCOLS + DF_BLK && prow >= w && prow < f;
    RowPull rp{0, 0, {-1, -1, -1, -1}};
    double val[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) val[r] = 0.0;
    if (own) {
        const int srow = A.reorder_fw ? A.piv[fd.c0 + prow] - 1 - fd.c0 : prow;
        rp = df_row_pull_prep(A.rptr, A.csrc, (int64_t)q.rbase + srow);
        const int64_t src = A.perm[fd.c0 + srow];
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) val[r] = A.in[src + r * A.ldin];
    } else if (thru) {
        rp = df_row_pull_prep(A.rptr, A.csrc, (int64_t)q.rbase + prow);
    }
    if (tid == 0 && q.fneed > 0) df_wait(A.fcnt + s, (unsigned)q.fneed, A.status);
    __syncthreads();
    if (stamp && tid == 0) *stamp = (int64_t)df_clock();
    if (own || thru) df_row_pull<NR>(rp, A.csrc, A.U, nrhs, val);
    if (tid < DF_PCOLS) {
#pragma unroll
        for (int r = 0; r < NR; ++r) zs[tid + DF_PCOLS * r] = own ? val[r] : 0.0;
    } else if (tid < DF_PCOLS + DF_BLK) {
#pragma unroll
        for (int r = 0; r < NR; ++r) pass[(tid - DF_PCOLS) + DF_BLK * r] = thru ? val[r] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        double acc = 0.0;
        if (r < nrhs) {
#pragma unroll
            for (int e = 0; e < 32; ++e) acc += (double)pv[e] * zs[32 * g + e + DF_PCOLS * r];
        }
        red[(r * 4 + g) * DF_BLK + i] = acc;
    }
    __syncthreads();
    double v[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r)
        v[r] = tid < DF_BLK ? red[(r * 4) * DF_BLK + tid] + red[(r * 4 + 1) * DF_BLK + tid] +
                                  red[(r * 4 + 2) * DF_BLK + tid] + red[(r * 4 + 3) * DF_BLK + tid] -
                                  pass[tid + DF_BLK * r]
                            : 0.0;
    if (nkc > 1) {
        double* p = A.part + (int64_t)(slot0 + kc) * (DF_BLK * DF_MAX_NRHS);
        if (tid < DF_BLK) {
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) p[tid + DF_BLK * r] = v[r];
        }
        if (!df_last_arrival(A.tcnt + q.tcnt + t, (unsigned)nkc, &last)) return;
        // the partials in parallel: thread (i, kq) sums chunks kq, kq + 4, ... of row i; then the four
        // groups add in order
        {
            const int kq = tid >> 6;
            double acc[NR];
#pragma unroll
            for (int r = 0; r < NR; ++r) acc[r] = 0.0;
            for (int k = kq; k < nkc; k += 4) {
                const double* pk = A.part + (int64_t)(slot0 + k) * (DF_BLK * DF_MAX_NRHS);
#pragma unroll
                for (int r = 0; r < NR; ++r)
                    if (r < nrhs) acc[r] += __ldcg(pk + i + DF_BLK * r);
            }
#pragma unroll
            for (int r = 0; r < NR; ++r) red[(r * 4 + kq) * DF_BLK + i] = acc[r];
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < NR; ++r)
            v[r] = tid < DF_BLK ? red[(r * 4) * DF_BLK + tid] + red[(r * 4 + 1) * DF_BLK + tid] +
                                      red[(r * 4 + 2) * DF_BLK + tid] + red[(r * 4 + 3) * DF_BLK + tid]
                                : 0.0;
    }
    if (tid < DF_BLK && row < f) {
        if (row < w) {
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) A.xtmp[fd.c0 + row + r * n] = v[r];
        } else {
            double* u = A.U + ((int64_t)q.urow + row - w) * nrhs;
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) u[r] = v[r];
        }
    }
    df_publish_cta(A.fcnt + (fd.parent >= 0 ? fd.parent : s), 0u, true);
}

// Backward of an inverse-panel front, column block b (DF_PBCOLS columns) times row chunk rc of P:
// x1 = P^T [y1; -x2], y1 = D^-1 (the forward result), x2 = the solution at the front's update rows.
// Warp wp takes columns 4 wp .. 4 wp + 3 of the block, lane l the chunk's rows l + 32 e; the lanes' sums
// reduce across the warp. With several chunks the last task sums the partials in chunk order and
// writes the block's solution (local pivot order undone) into Y and X; every block signals bdone.
template <typename T, int NR>
__device__ __noinline__ void df_pinv_backward(const DataflowArgs<T>& A, int s, int b, int cc, double* sm, int64_t* stamp) {
    __shared__ int last;
    const DFront fd = A.fronts[s];
    const DfFront q = A.df[s];
    const int f = fd.f, w = fd.w, nrhs = A.nrhs, tid = threadIdx.x;
    const int64_t n = A.n;
    const int rc = cc & 255, slot0 = cc >> 8;
    const int first = df_pb_first(b), nrc = df_pb_chunks(f, b);
    const int j0 = DF_PBCOLS * b, i0 = DF_PROWS * rc;
    const int wp = tid >> 5, lane = tid & 31;
    const T* Pm = A.invb + q.inv;
    double* zs = sm;                          // DF_PROWS x NR: [y1; -x2] over the chunk's rows
    double* xs = zs + DF_PROWS * NR;          // DF_PBCOLS x NR: the block's sums (then 8 x that: the
                                              // finisher's partial sums)
    static_assert(DF_PBCOLS == 4 * (DF_THREADS / 32) && DF_PROWS == 4 * 32 && DF_THREADS / DF_PBCOLS == 8,
                  "backward task shape");
    // before the parent is done: the thread's 16 entries of P and the chunk's update-row indices
    T pv[4][4];
#pragma unroll
    for (int c4 = 0; c4 < 4; ++c4)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int row = i0 + lane + 32 * e, col = j0 + 4 * wp + c4;
            pv[c4][e] = (row < f && col < w && (row >= w || row >= col)) ? Pm[row + (int64_t)col * f] : T(0);
        }
    const int zrow = i0 + tid;
    const bool zin = tid < DF_PROWS && zrow < f;
    const int32_t ridx = (zin && zrow >= w) ? A.rowval[fd.row_begin + zrow] : 0;
    const unsigned pbsig = fd.parent >= 0 ? (unsigned)A.df[fd.parent].bsig : 0u;
    if (tid == 0) {
        if (fd.parent >= 0) df_wait(A.bdone + fd.parent, pbsig, A.status);
        else df_wait(A.fcnt + s, (unsigned)(q.fneed + q.fsig), A.status);
        if (stamp) *stamp = (int64_t)df_clock();
    }
    __syncthreads();
    if (tid < DF_PROWS) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            double z = 0.0;
            if (zin && r < nrhs) z = zrow < w ? df_dinv(A, A.xtmp, fd.c0 + zrow, r) : -A.Y[ridx + r * n];
            zs[tid + DF_PROWS * r] = z;
        }
    }
    __syncthreads();
    constexpr int NV = 4 * NR, G = 32 / NV;
    double v[NV];
#pragma unroll
    for (int c4 = 0; c4 < 4; ++c4)
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            double acc = 0.0;
            if (r < nrhs) {
#pragma unroll
                for (int e = 0; e < 4; ++e) acc += (double)pv[c4][e] * zs[lane + 32 * e + DF_PROWS * r];
            }
            v[c4 * NR + r] = acc;
        }
    const double red = df_lane_reduce<NV>(v, lane);
    if (lane % G == 0) {
        const int idx = lane / G;
        xs[4 * wp + idx / NR + DF_PBCOLS * (idx % NR)] = red;
    }
    __syncthreads();
    double x[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) x[r] = tid < DF_PBCOLS ? xs[tid + DF_PBCOLS * r] : 0.0;
    if (nrc > 1) {
        double* p = A.part + (int64_t)(slot0 + rc - first) * (DF_BLK * DF_MAX_NRHS);
        if (tid < DF_PBCOLS) {
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) p[tid + DF_PBCOLS * r] = x[r];
        }
        if (!df_last_arrival(A.ccnt + q.ccnt + b, (unsigned)nrc, &last)) return;
        // the partials in parallel: thread (jj, kq) sums chunks kq, kq + 8, ... of column jj; then the
        // eight groups add in order
        double* grp = xs + DF_PBCOLS * NR;    // 8 x DF_PBCOLS x NR
        {
            const int jj = tid & (DF_PBCOLS - 1), kq = tid / DF_PBCOLS;
            double acc[NR];
#pragma unroll
            for (int r = 0; r < NR; ++r) acc[r] = 0.0;
            for (int k = kq; k < nrc; k += DF_THREADS / DF_PBCOLS) {
                const double* pk = A.part + (int64_t)(slot0 + k) * (DF_BLK * DF_MAX_NRHS);
#pragma unroll
                for (int r = 0; r < NR; ++r)
                    if (r < nrhs) acc[r] += __ldcg(pk + jj + DF_PBCOLS * r);
            }
#pragma unroll
            for (int r = 0; r < NR; ++r) grp[(r * 8 + kq) * DF_PBCOLS + jj] = acc[r];
        }
        __syncthreads();
        if (tid < DF_PBCOLS) {
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                double sum = 0.0;
#pragma unroll
                for (int kq = 0; kq < 8; ++kq) sum += grp[(r * 8 + kq) * DF_PBCOLS + tid];
                x[r] = sum;
            }
        }
    }
    const int k = j0 + tid;
    if (tid < DF_PBCOLS && k < w) {
        const int64_t dst = A.reorder_bw ? A.piv[fd.c0 + k] - 1 : fd.c0 + k;
        const int64_t o = A.perm[dst];
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) {
                A.Y[dst + r * n] = x[r];
                double* op = A.out + o + r * A.ldout;
                if (A.mode == 2) *op += x[r];
                else *op = x[r];
            }
    }
    df_publish_cta(A.bdone + s, 0u, true);
}

}  // namespace

// the arguments of one batch member: the member-dependent arrays advanced by its strides
template <typename T>
__device__ __forceinline__ void df_member_args(const DataflowArgs<T>& A, int member, DataflowArgs<T>& B) {
    B = A;
    const int64_t q = member;
    B.facf += q * A.s_fac;
    B.facb += q * A.s_fac;
    B.invf += q * A.s_inv;
    B.invb += q * A.s_inv;
    if (B.piv) B.piv += q * A.s_piv;
    if (B.d) B.d += q * A.s_d;
    if (B.kind) B.kind += q * A.s_piv;
    B.in += q * A.s_in;
    B.out += q * A.s_out;
    B.Y += q * A.s_y;
    B.xtmp += q * A.s_y;
    B.U += q * A.s_u;
    B.part += q * A.s_part;
    B.fcnt += q * A.s_flags;
    B.bdone += q * A.s_flags;
    B.xflag += q * A.s_flags;
    B.pcnt += q * A.s_flags;
    B.tcnt += q * A.s_flags;
    B.ccnt += q * A.s_flags;
}

template <typename T, int NR>
__global__ void __launch_bounds__(DF_THREADS, 2) dataflow_solve_kernel(DataflowArgs<T> A0) {
    extern __shared__ double dsm[];
    __shared__ int task_k, bundle_next;
    __shared__ DataflowArgs<T> A;   // this task's member's arguments
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = A0.ntasks * A0.nmembers;
    while (true) {
        if (threadIdx.x == 0) {
            task_k = atomicAdd(A0.head, 1u);
            bundle_next = 0;
            if (*(volatile int32_t*)A0.status != 0) task_k = total;   // a wait gave up: stop
        }
        __syncthreads();
        if (task_k >= total) break;
        const int k = task_k / A0.nmembers, j = task_k - k * A0.nmembers;
        if (threadIdx.x == 0) df_member_args(A0, A0.members ? A0.members[j] : j, A);
        __syncthreads();
        const DfTask tk = A.tasks[k];
        if (A.trace && threadIdx.x == 0) {
            A.trace[6 * k] = (int64_t)df_clock();
            A.trace[6 * k + 1] = 0;
            A.trace[6 * k + 3] = blockIdx.x;
            A.trace[6 * k + 4] = tk.kind;
            A.trace[6 * k + 5] = (int64_t)tk.a | ((int64_t)tk.b << 32);
        }
        int64_t* stamp = A.trace ? A.trace + 6 * k + 1 : nullptr;
        switch (tk.kind) {
            case DF_FW_BUNDLE:
            case DF_BW_BUNDLE: {
                double* z = dsm + (int64_t)warp * A.warp_smem;
                while (true) {
                    int i = 0;
                    if (lane == 0) i = atomicAdd(&bundle_next, 1);
                    i = __shfl_sync(0xffffffffu, i, 0);
                    if (i >= tk.b) break;
                    const int s = A.bundles[tk.a + i];
                    int64_t* st = i == 0 ? stamp : nullptr;
                    if (tk.kind == DF_FW_BUNDLE) df_warp_forward<T, NR>(A, s, z, st);
                    else df_warp_backward<T, NR>(A, s, z, st);
                }
                break;
            }
            case DF_FW_TILE: df_tile_forward<T, NR>(A, tk.a, tk.b, dsm, stamp); break;
            case DF_BW_PART: df_tiled_part<T, NR>(A, tk.a, tk.b, tk.c, dsm, stamp); break;
            case DF_BW_OWNER: df_tiled_owner<T, NR>(A, tk.a, tk.b, dsm, stamp); break;
            case DF_FW_PINV: df_pinv_forward<T, NR>(A, tk.a, tk.b, tk.c, dsm, stamp); break;
            case DF_BW_PINV: df_pinv_backward<T, NR>(A, tk.a, tk.b, tk.c, dsm, stamp); break;
            default: break;
        }
        __syncthreads();
        if (A.trace && threadIdx.x == 0) A.trace[6 * k + 2] = (int64_t)df_clock();
    }
}

// the right-hand-side group width the kernel is instantiated for: the smallest of 1, 2, 4, 8 >= nrhs
inline int df_nr(int nrhs) { return nrhs <= 1 ? 1 : nrhs <= 2 ? 2 : nrhs <= 4 ? 4 : 8; }

template <typename T>
const void* df_kernel_ptr(int nr) {
    switch (nr) {
        case 1: return (const void*)dataflow_solve_kernel<T, 1>;
        case 2: return (const void*)dataflow_solve_kernel<T, 2>;
        case 4: return (const void*)dataflow_solve_kernel<T, 4>;
        default: return (const void*)dataflow_solve_kernel<T, 8>;
    }
}

template <typename T>
int dataflow_solve_grid(int nrhs, size_t smem) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, df_kernel_ptr<T>(df_nr(nrhs)), DF_THREADS, smem) != cudaSuccess)
        return 0;
    return sms * std::min(per, 2);
}

template <typename T>
cudaError_t launch_dataflow_solve(const DataflowArgs<T>& a, int grid, size_t smem, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(DF_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    switch (df_nr(a.nrhs)) {
        case 1: return cudaLaunchKernelEx(&cfg, dataflow_solve_kernel<T, 1>, a);
        case 2: return cudaLaunchKernelEx(&cfg, dataflow_solve_kernel<T, 2>, a);
        case 4: return cudaLaunchKernelEx(&cfg, dataflow_solve_kernel<T, 4>, a);
        default: return cudaLaunchKernelEx(&cfg, dataflow_solve_kernel<T, 8>, a);
    }
}

template cudaError_t launch_dataflow_solve<double>(const DataflowArgs<double>&, int, size_t, cudaStream_t);
template cudaError_t launch_dataflow_solve<float>(const DataflowArgs<float>&, int, size_t, cudaStream_t);
template int dataflow_solve_grid<double>(int, size_t);
template int dataflow_solve_grid<float>(int, size_t);

cudaError_t prepare_dataflow_kernels(int max_smem) {
    for (int nr : {1, 2, 4, 8})
        for (const void* k : {df_kernel_ptr<double>(nr), df_kernel_ptr<float>(nr)}) {
            cudaFuncAttributes fa;
            cudaError_t e = cudaFuncGetAttributes(&fa, k);
            if (e != cudaSuccess) return e;
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem - (int)fa.sharedSizeBytes);
            if (e != cudaSuccess) return e;
        }
    return cudaSuccess;
}

}  // namespace sds

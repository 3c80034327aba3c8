// Fused per-front kernels of the numeric phase.
//
// small_front_kernel: one CTA per front of one level, the whole f x f front in
// shared memory: zero, assemble A, extend-add the children's contribution
// blocks (children in child_list order, so every sum has a fixed order and the
// result is bitwise reproducible), the dense partial factorization of the w
// fully-summed columns (Cholesky; Bunch-Kaufman LDLT; threshold-pivoting LU),
// the Schur update of the contribution block, and the write-out of the panel,
// D, pivots, statistics and contribution block. It replaces the reference's
// regime B kernels (front_cholesky_kernel! src/numeric/front.jl:154-206,
// front_ldlt_kernel! src/numeric/ldlt.jl:992-1111, front_lu_kernel!
// src/numeric/lu.jl:264-330); the in-front arithmetic follows the CPU reference
// (src/reference/*.jl) step by step.
//
// subtree_kernel: the same per-front body run by one CTA over a whole leaf
// subtree of such fronts in postorder (the reference's regime A).
//
// warp_front_kernel: Cholesky fronts of at most 32 rows, one warp per front, for
// level launches of many such fronts (batches of small systems).
//
// assemble_large_kernel: column-owner assembly of the fronts too large for
// shared memory: one warp per (front, parent index p) builds the column it
// owns in row chunks from the entries of A of that column and every child's
// contribution, in child order. No atomics.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "common.cuh"
#include "kernels.cuh"
#include "front_factor.cuh"
#include "pivot.cuh"

namespace sds {

// One front by the whole CTA, in shared memory (smem_raw holds at least small_front_smem(f)). The CTA's
// threads all call it; it ends with the front's outputs written to global memory.
template <typename T, int STRUCT>
__device__ __forceinline__ void small_front(const SmallArgs<T>& A, const int s, const int member,
                                            unsigned char* smem_raw) {
    const DFront fd = A.maps.fronts[s];
    const int f = fd.f, w = fd.w, m = f - w;
    const int ld = f | 1;
    T* F = reinterpret_cast<T*>(smem_raw);
    size_t off = ((size_t)ld * f * sizeof(T) + 15) & ~size_t(15);
    double* dd = reinterpret_cast<double*>(smem_raw + off);  // w
    double* ee = dd + w;                                     // w
    double* lvec = ee + w;                                   // 2 f (multipliers)
    int* lp = reinterpret_cast<int*>(lvec + 2 * f);          // w
    int* ri = lp + w;                                        // relind of the current child (<= f)
    int* ctl = ri + f;                                       // control words
    signed char* kd = reinterpret_cast<signed char*>(ctl + 16);

    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    const double* nz = A.nzval + (int64_t)member * A.nnz;
    T* factor = A.factor + (int64_t)member * A.factor_len;
    T* cbar = A.cb + (int64_t)member * A.cb_len;

    for (int q = tid; q < ld * f; q += nt) F[q] = T(0);
    if (tid < 16) ctl[tid] = 0;
    __syncthreads();
    // assembly of A: each run of equal destinations is summed by one thread, in entry order
    for (int k = fd.am_begin + tid; k < fd.am_end; k += nt) {
        int code = A.maps.am_loc[k];
        if (k > fd.am_begin && A.maps.am_loc[k - 1] == code) continue;
        T acc = T(0);
        for (int q = k; q < fd.am_end && A.maps.am_loc[q] == code; ++q) acc += T(nz[A.maps.am_src[q]]);
        int loc = (code > 0 ? code : -code) - 1;
        int i = loc % f, j = loc / f;
        if (code > 0) F[i + j * ld] += acc;
        else F[j + i * ld] += acc;
    }
    __syncthreads();
    // extend-add, children in order
    for (int q = fd.ch_begin; q < fd.ch_end; ++q) {
        const int c = A.maps.child_list[q];
        const DFront cd = A.maps.fronts[c];
        const int mc = cd.f - cd.w;
        if (mc <= 0 || cd.cb < 0) continue;
        for (int t = tid; t < mc; t += nt) ri[t] = A.maps.relind[cd.ri_begin + t];
        __syncthreads();
        const T* C = cbar + cd.cb;
        for (int jj = warp; jj < mc; jj += nwarps) {
            const int pj = ri[jj];
            const int i0 = STRUCT == STRUCT_G ? 0 : jj;
            batched_add<8, T>(i0 + lane, 32, mc, [&](int ii) { return (double)C[ii + (int64_t)jj * mc]; },
                              [&](int ii) -> T* { return F + ri[ii] + pj * ld; });
        }
        __syncthreads();
    }
    if (STRUCT == STRUCT_S) {  // the pivoting reads both triangles of the fully-summed block
        for (int q = tid; q < w * w; q += nt) {
            int i = q % w, j = q / w;
            if (i > j) F[j + i * ld] = F[i + j * ld];
        }
        __syncthreads();
    }
    int64_t st[NSTAT] = {0, 0, 0, 0, 0, 0};
    int status = 0;
    const double eps = A.eps;

    if (STRUCT == STRUCT_SPD) {
        for (int j = 0; j < w; ++j) {
            double ajj = (double)F[j + j * ld];
            bool ok = ajj > eps || (eps > 0 && ajj >= 0);
            if (!ok) { status = j + 1; break; }
            double djj = sqrt(fmax(ajj, eps));
            T inv = T(1.0 / djj);
            __syncthreads();
            for (int i = j + 1 + tid; i < f; i += nt) F[i + j * ld] *= inv;
            if (tid == 0) F[j + j * ld] = T(djj);
            __syncthreads();
            for (int l = j + 1 + warp; l < f; l += nwarps) {
                const T flj = F[l + j * ld];
                for (int i = l + lane; i < f; i += 32) F[i + l * ld] -= F[i + j * ld] * flj;
            }
            __syncthreads();
        }
        st[ST_NPOS] = status ? status - 1 : w;
        st[ST_INFO] = status;
    } else if (STRUCT == STRUCT_S) {
        SmemStore<T> store{F, ld, f, w};
        FrontScratch sc{lvec, dd, ee, lp, kd, ctl};
        ldlt_front_steps<T>(store, sc, f, w, A.pivot, A.u, eps, A.psign, A.maps.perm, fd.c0, st);
        // F22 -= (L21 D) L21^T, lower triangle, kk in order (ldlt.jl:184-191)
        for (int jj = warp; jj < m; jj += nwarps)
            for (int ii = jj + lane; ii < m; ii += 32) {
                T acc = F[w + ii + (w + jj) * ld];
                int q = 0;
                while (q < w) {
                    if (kd[q] == KIND_2X2_FIRST) {
                        double x1 = (double)F[w + ii + q * ld], x2 = (double)F[w + ii + (q + 1) * ld];
                        T w1 = T(x1 * dd[q] + x2 * ee[q]), w2 = T(x1 * ee[q] + x2 * dd[q + 1]);
                        acc -= w1 * F[w + jj + q * ld];
                        acc -= w2 * F[w + jj + (q + 1) * ld];
                        q += 2;
                    } else {
                        acc -= T((double)F[w + ii + q * ld] * dd[q]) * F[w + jj + q * ld];
                        q += 1;
                    }
                }
                F[w + ii + (w + jj) * ld] = acc;
            }
        __syncthreads();
    } else {  // STRUCT_G: LU with row interchanges inside the fully-summed rows
        SmemStore<T> store{F, ld, f, w};
        FrontScratch sc{lvec, dd, ee, lp, kd, ctl};
        lu_front_steps<T>(store, sc, f, w, A.lu_pivot != 0, A.u, eps, st);
        // F22 -= (L21 D) U12, summed over k in order (lu.jl:142-150)
        for (int jj = warp; jj < m; jj += nwarps)
            for (int ii = lane; ii < m; ii += 32) {
                T acc = T(0);
                for (int q = 0; q < w; ++q) acc += F[w + ii + q * ld] * T(dd[q]) * F[q + (w + jj) * ld];
                F[w + ii + (w + jj) * ld] -= acc;
            }
        __syncthreads();
    }

    // write-out: panel (and U^T panel), D / pivots, statistics, contribution block
    T* P = factor + fd.panel;
    const bool unit = STRUCT != STRUCT_SPD;
    for (int j = warp; j < w; j += nwarps)
        for (int i = lane; i < f; i += 32) {
            T v = i < j ? T(0) : (i == j && unit ? T(1) : F[i + j * ld]);
            P[i + (int64_t)j * f] = v;
        }
    if (STRUCT == STRUCT_G) {
        T* U = A.ufactor + (int64_t)member * A.factor_len + fd.panel;
        for (int j = warp; j < w; j += nwarps)
            for (int i = lane; i < f; i += 32) U[i + (int64_t)j * f] = i < j ? T(0) : (i == j ? T(1) : F[j + i * ld]);
    }
    if (STRUCT != STRUCT_SPD) {
        const int64_t n = A.n;
        for (int q = tid; q < w; q += nt) {
            const int64_t g = fd.c0 + q;
            A.piv[member * n + g] = fd.c0 + lp[q] + 1;
            A.kind[member * n + g] = kd[q];
            A.d[member * 2 * n + g] = dd[q];
            A.d[member * 2 * n + n + g] = STRUCT == STRUCT_S ? ee[q] : 0.0;
        }
    }
    if (tid == 0) {
        int64_t* S = A.stats + ((int64_t)member * A.ns + s) * NSTAT;
        for (int q = 0; q < NSTAT; ++q) S[q] = st[q];
        A.finfo[(int64_t)member * A.ns + s] = (int32_t)st[ST_INFO];
    }
    if (fd.cb >= 0 && m > 0 && status == 0) {
        T* C = cbar + fd.cb;
        for (int jj = warp; jj < m; jj += nwarps)
            for (int ii = (STRUCT == STRUCT_G ? 0 : jj) + lane; ii < m; ii += 32)
                C[ii + (int64_t)jj * m] = F[w + ii + (w + jj) * ld];
    }
}

template <typename T, int STRUCT>
__global__ void __launch_bounds__(256) small_front_kernel(SmallArgs<T> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    small_front<T, STRUCT>(A, A.list[blockIdx.x], member, smem_raw);
}

// Fused subtrees: one CTA factors a whole subtree of shared-memory fronts, front after front in the
// subtree's postorder (A.list[A.sub_ptr[b] .. A.sub_ptr[b + 1]) for CTA b), in one launch for every
// subtree of its size class instead of one launch per level. A child's contribution block goes to
// global memory (the subtree's stack region of the arena, hot in L2) and its parent, later in the same
// CTA, reads it back after the barrier between the two fronts, which makes the CTA's global writes
// visible to all its threads. Each front's arithmetic is small_front's, so the factor is bit for bit
// the level launches'. Replaces the reference's regime-A kernels (subtree_cholesky_kernel!
// src/numeric/subtree.jl:274-316, subtree_ldlt_kernel! src/numeric/ldlt.jl:1133-1228,
// subtree_lu_kernel! src/numeric/lu.jl:424-493).
template <typename T, int STRUCT>
__global__ void __launch_bounds__(256) subtree_kernel(SmallArgs<T> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    const int q0 = A.sub_ptr[blockIdx.x], q1 = A.sub_ptr[blockIdx.x + 1];
    for (int q = q0; q < q1; ++q) {
        small_front<T, STRUCT>(A, A.list[q], member, smem_raw);
        __syncthreads();   // the front's shared memory is read out before the next front zeroes it
    }
}

// One Cholesky front of at most WARP_FRONT_F rows by one warp, in its own shared-memory slice F: the
// lower triangle packed by columns (column j holds rows j .. f - 1 from offset j f - j (j - 1) / 2),
// since a Cholesky front reads and writes nothing above its diagonal. The arithmetic of every entry is
// small_front's, in the same order (assembly runs summed in entry order by the run's first lane;
// children's contributions added in child order; per column the scaling by the reciprocal square
// root and the rank-1 update in column order), so the results are bit for bit the CTA kernel's; only
// the mapping of entries to threads differs. Batches of small systems have hundreds of thousands of
// such fronts, and a warp per front keeps eight of them in flight per CTA instead of one; a launch of
// few fronts keeps the CTA kernel, whose 128 threads shorten each front's chain (lap2d 64^2: 1.04
// against 1.35 ms per factorization). Fused subtrees keep the CTA kernel too: one warp per subtree was
// slower (1024 uneven systems: 6.79 against 5.93 ms).
constexpr int WARP_FRONT_F = 32;
constexpr int WARP_FRONTS_PER_CTA = 8;
constexpr int WARP_FRONT_LEN = WARP_FRONT_F * (WARP_FRONT_F + 1) / 2;   // packed entries per warp
constexpr int64_t WARP_FRONT_MIN_LAUNCH = 4096;   // fronts x members of a launch for the warp kernel

template <typename T>
__device__ __forceinline__ void warp_front_spd(const SmallArgs<T>& A, const int s, const int member, T* F) {
    const DFront fd = A.maps.fronts[s];
    const int f = fd.f, w = fd.w, m = f - w;
    const int lane = threadIdx.x & 31;
    auto at = [&](int i, int j) -> T& { return F[j * f - ((j * (j - 1)) >> 1) + (i - j)]; };   // i >= j
    const double* nz = A.nzval + (int64_t)member * A.nnz;
    for (int q = lane; q < (f * (f + 1)) / 2; q += 32) F[q] = T(0);
    __syncwarp();
    for (int k = fd.am_begin + lane; k < fd.am_end; k += 32) {
        const int code = A.maps.am_loc[k];
        if (k > fd.am_begin && A.maps.am_loc[k - 1] == code) continue;
        T acc = T(0);
        for (int q = k; q < fd.am_end && A.maps.am_loc[q] == code; ++q) acc += T(nz[A.maps.am_src[q]]);
        const int loc = (code > 0 ? code : -code) - 1;
        const int i = loc % f, j = loc / f;
        // (an entry above the diagonal is never read by a Cholesky front: the CTA kernel's square
        // slice holds it unused)
        if (code > 0 && i >= j) at(i, j) += acc;
        else if (code < 0 && j >= i) at(j, i) += acc;
    }
    __syncwarp();
    const T* cbar = A.cb + (int64_t)member * A.cb_len;
    for (int q = fd.ch_begin; q < fd.ch_end; ++q) {
        const DFront cd = A.maps.fronts[A.maps.child_list[q]];
        const int mc = cd.f - cd.w;
        if (mc <= 0 || cd.cb < 0) continue;
        const int32_t* ri = A.maps.relind + cd.ri_begin;
        const T* C = cbar + cd.cb;
        for (int jj = 0; jj < mc; ++jj) {
            const int pj = ri[jj];
            batched_add<4, T>(jj + lane, 32, mc, [&](int ii) { return (double)C[ii + (int64_t)jj * mc]; },
                              [&](int ii) -> T* { return &at(ri[ii], pj); });
        }
        __syncwarp();
    }
    int status = 0;
    const double eps = A.eps;
    for (int j = 0; j < w; ++j) {
        const double ajj = (double)at(j, j);
        const bool ok = ajj > eps || (eps > 0 && ajj >= 0);
        if (!ok) { status = j + 1; break; }
        const double djj = sqrt(fmax(ajj, eps));
        const T inv = T(1.0 / djj);
        __syncwarp();
        for (int i = j + 1 + lane; i < f; i += 32) at(i, j) *= inv;
        if (lane == 0) at(j, j) = T(djj);
        __syncwarp();
        for (int l = j + 1; l < f; ++l) {
            const T flj = at(l, j);
            for (int i = l + lane; i < f; i += 32) at(i, l) -= at(i, j) * flj;
        }
        __syncwarp();
    }
    T* P = A.factor + (int64_t)member * A.factor_len + fd.panel;
    for (int j = 0; j < w; ++j)
        for (int i = lane; i < f; i += 32) P[i + (int64_t)j * f] = i < j ? T(0) : at(i, j);
    if (lane == 0) {
        int64_t* S = A.stats + ((int64_t)member * A.ns + s) * NSTAT;
        S[ST_NPOS] = status ? status - 1 : w;
        for (int q = 1; q < NSTAT; ++q) S[q] = q == ST_INFO ? status : 0;
        A.finfo[(int64_t)member * A.ns + s] = status;
    }
    if (fd.cb >= 0 && m > 0 && status == 0) {
        T* C = A.cb + (int64_t)member * A.cb_len + fd.cb;
        for (int jj = 0; jj < m; ++jj)
            for (int ii = jj + lane; ii < m; ii += 32) C[ii + (int64_t)jj * m] = at(w + ii, w + jj);
    }
    __syncwarp();
}

// Level launches of Cholesky fronts of at most 32 rows: one warp per front, eight per CTA.
template <typename T>
__global__ void __launch_bounds__(256) warp_front_kernel(SmallArgs<T> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int wi = blockIdx.x * WARP_FRONTS_PER_CTA + (threadIdx.x >> 5);
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    if (wi >= A.count) return;
    T* F = reinterpret_cast<T*>(smem_raw) + (threadIdx.x >> 5) * WARP_FRONT_LEN;
    warp_front_spd<T>(A, A.list[wi], member, F);
}

size_t small_front_smem(int fmax, int elsize) {
    size_t ld = fmax | 1;
    size_t b = (ld * fmax * elsize + 15) & ~size_t(15);
    b += sizeof(double) * (2 * fmax + 2 * fmax);  // dd, ee (w <= f), lvec (2 f)
    b += sizeof(int) * (fmax + fmax + 16);        // lp, ri, ctl
    b += fmax + 16;                               // kind
    return (b + 15) & ~size_t(15);
}

template <typename T>
cudaError_t launch_small(int structure, const SmallArgs<T>& a, int count, int nmembers, int fmax, cudaStream_t st) {
    const bool sub = a.sub_ptr != nullptr;
    if (structure == STRUCT_SPD && fmax <= WARP_FRONT_F && !sub &&
        (int64_t)count * nmembers >= WARP_FRONT_MIN_LAUNCH) {   // a warp per front
        const size_t wsmem = sizeof(T) * WARP_FRONTS_PER_CTA * WARP_FRONT_LEN;
        dim3 wgrid((count + WARP_FRONTS_PER_CTA - 1) / WARP_FRONTS_PER_CTA, nmembers);
        SmallArgs<T> b = a;
        b.count = count;
        warp_front_kernel<T><<<wgrid, 32 * WARP_FRONTS_PER_CTA, wsmem, st>>>(b);
        return cudaGetLastError();
    }
    size_t smem = small_front_smem(fmax, sizeof(T));
    int threads = fmax <= 48 ? 128 : 256;
    dim3 grid(count, nmembers);
    switch (structure) {
        case STRUCT_SPD:
            if (sub) subtree_kernel<T, STRUCT_SPD><<<grid, threads, smem, st>>>(a);
            else small_front_kernel<T, STRUCT_SPD><<<grid, threads, smem, st>>>(a);
            break;
        case STRUCT_S:
            if (sub) subtree_kernel<T, STRUCT_S><<<grid, threads, smem, st>>>(a);
            else small_front_kernel<T, STRUCT_S><<<grid, threads, smem, st>>>(a);
            break;
        default:
            if (sub) subtree_kernel<T, STRUCT_G><<<grid, threads, smem, st>>>(a);
            else small_front_kernel<T, STRUCT_G><<<grid, threads, smem, st>>>(a);
    }
    return cudaGetLastError();
}

// the opt-in shared-memory limit of every kernel with a dynamic allocation, set once at plan creation
// (outside any stream capture)
cudaError_t prepare_factor_kernels(int max_smem) {
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* k) {
        if (e != cudaSuccess) return;
        cudaFuncAttributes fa;
        e = cudaFuncGetAttributes(&fa, k);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem - (int)fa.sharedSizeBytes);
    };
    set((const void*)small_front_kernel<double, STRUCT_SPD>);
    set((const void*)small_front_kernel<double, STRUCT_S>);
    set((const void*)small_front_kernel<double, STRUCT_G>);
    set((const void*)small_front_kernel<float, STRUCT_SPD>);
    set((const void*)small_front_kernel<float, STRUCT_S>);
    set((const void*)small_front_kernel<float, STRUCT_G>);
    set((const void*)subtree_kernel<double, STRUCT_SPD>);
    set((const void*)subtree_kernel<double, STRUCT_S>);
    set((const void*)subtree_kernel<double, STRUCT_G>);
    set((const void*)subtree_kernel<float, STRUCT_SPD>);
    set((const void*)subtree_kernel<float, STRUCT_S>);
    set((const void*)subtree_kernel<float, STRUCT_G>);
    set((const void*)warp_front_kernel<double>);
    set((const void*)warp_front_kernel<float>);
    return e;
}

template cudaError_t launch_small<double>(int, const SmallArgs<double>&, int, int, int, cudaStream_t);
template cudaError_t launch_small<float>(int, const SmallArgs<float>&, int, int, int, cudaStream_t);

// ---------------------------------------------------------------------------
// Column-owner assembly of large fronts (one warp per task).
// Storage of a large front: the panel (f x w, ld f) holds F[:, 0:w] -- for "S"
// both triangles of the fully-summed block -- ; "G" keeps F[j, i] (i > j, j < w)
// in the U^T panel at ufactor[panel + i + j f]; the contribution block
// F[w:f, w:f] lives at cb (ld m).
//
// A warp builds its column ASM_ROWS rows at a time in shared memory: the chunk
// starts at zero, takes the column's entries of A, then the rows of every
// child's contribution that land in it (the child's row-chunk table gives their
// range, relind being increasing) in the order of the column's extend-add list,
// and is written once. Every entry receives the same additions in the same
// order as a zero fill followed by accumulation in place, at one write of the
// entry instead of a write, a read and a write.
constexpr int ASM_WARPS = 8;
constexpr int ASM_KIDS = 8;   // child descriptors a warp keeps in shared memory per column

template <typename T>
struct AsmChild {
    const T* col;      // column t of the child's contribution block
    const int* ri;     // the child's relind
    const int* rc;     // the child's row-chunk starts
    int t, mc;
};

// buf[ri[q] - r0] += val(q) for q in [q0, q1) (lanes strided; the targets of one call are distinct);
// eight loads in flight per lane before the shared-memory updates
template <class T, class VAL>
__device__ __forceinline__ void chunk_add(T* buf, int r0, int q0, int q1, const int* ri, int lane, VAL val) {
    constexpr int U = ASM_ROWS / 32;
    for (int qb = q0 + lane; qb < q1; qb += 32 * U) {
        int pos[U];
        double v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int q = qb + 32 * u;
            pos[u] = q < q1 ? ri[q] - r0 : -1;
            v[u] = q < q1 ? val(q) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (pos[u] >= 0) buf[pos[u]] = T((double)buf[pos[u]] + v[u]);
    }
}

template <typename T, int STRUCT>
__global__ void __launch_bounds__(ASM_WARPS * 32) assemble_large_kernel(LargeAsmArgs<T> A) {
    constexpr bool GEN = STRUCT == STRUCT_G;
    __shared__ T lbuf[ASM_WARPS][ASM_ROWS];
    __shared__ T ubuf[GEN ? ASM_WARPS : 1][GEN ? ASM_ROWS : 1];
    __shared__ AsmChild<T> kids[ASM_WARPS][ASM_KIDS];
    const int wid = threadIdx.x >> 5;
    const int task = blockIdx.x * ASM_WARPS + wid;
    const int lane = threadIdx.x & 31;
    if (task >= A.count) return;
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    const ColTask ct = A.tasks[task];
    const DFront fd = A.maps.fronts[ct.front];
    const int f = fd.f, w = fd.w, m = f - w, p = ct.p;
    const bool panel = p < w;
    if (!panel && fd.cb < 0) return;
    const double* nz = A.nzval + (int64_t)member * A.nnz;
    const T* cbar = A.cb + (int64_t)member * A.cb_len;
    // the column indexed by front row: panel rows 0..f-1; contribution-block rows w..f-1 (from p for
    // the lower triangle of "SPD" and "S")
    T* lcol = panel ? A.factor + (int64_t)member * A.factor_len + fd.panel + (int64_t)p * f
                    : A.cb + (int64_t)member * A.cb_len + fd.cb + (int64_t)(p - w) * m - w;
    T* ucol = GEN && panel ? A.ufactor + (int64_t)member * A.factor_len + fd.panel + (int64_t)p * f : nullptr;
    const int rfirst = panel ? 0 : (GEN ? w : p);
    const int a0 = panel ? A.maps.amcol[fd.amcol_begin + p] : 0;
    const int a1 = panel ? A.maps.amcol[fd.amcol_begin + p + 1] : 0;
    const int e0 = A.maps.eacol[fd.eacol_begin + p], e1 = A.maps.eacol[fd.eacol_begin + p + 1];
    AsmChild<T>* kd = kids[wid];
    auto child = [&](int e) {
        AsmChild<T> k;
        const int c = A.maps.ea[2 * e];
        k.t = A.maps.ea[2 * e + 1];
        const DFront cd = A.maps.fronts[c];
        k.mc = cd.f - cd.w;
        k.col = cbar + cd.cb + (int64_t)k.t * k.mc;
        k.ri = A.maps.relind + cd.ri_begin;
        k.rc = A.maps.rchunk + cd.rc_begin;
        return k;
    };
    if (lane < ASM_KIDS && e0 + lane < e1) kd[lane] = child(e0 + lane);
    T* lb = lbuf[wid];
    T* ub = GEN ? ubuf[wid] : nullptr;
    __syncwarp();
    for (int r0 = rfirst; r0 < f;) {
        const int k = r0 / ASM_ROWS;
        const int r1 = min(f, (k + 1) * ASM_ROWS);
        const int len = r1 - r0;
        for (int i = lane; i < len; i += 32) {
            lb[i] = T(0);
            if (GEN && panel) ub[i] = T(0);
        }
        __syncwarp();
        // entries of A (runs of one location summed first, as the reference's assembly map lists them)
        for (int q = a0 + lane; q < a1; q += 32) {
            const int code = A.maps.am_loc[q];
            if (q > a0 && A.maps.am_loc[q - 1] == code) continue;
            const int row = (code > 0 ? code : -code) - 1 - p * f;
            if (row < r0 || row >= r1) continue;
            T acc = T(0);
            for (int z = q; z < a1 && A.maps.am_loc[z] == code; ++z) acc += T(nz[A.maps.am_src[z]]);
            if (code > 0) lb[row - r0] += acc;
            else ub[row - r0] += acc;
        }
        __syncwarp();
        for (int e = e0; e < e1; ++e) {
            const AsmChild<T> c = e - e0 < ASM_KIDS ? kd[e - e0] : child(e);
            const int lo = c.rc[k], hi = c.rc[k + 1];
            // column t of the child: its rows from the diagonal down land in column p; "G" contribution
            // block columns also take the rows above the diagonal (those below front row w are skipped by
            // the chunk bounds: they belong to the U^T panel)
            const int qb = (GEN && !panel) ? lo : max(lo, c.t);
            const T* col = c.col;
            chunk_add(lb, r0, qb, hi, c.ri, lane, [&](int q) { return (double)col[q]; });
            if (GEN && panel) {
                // row t of the child right of its diagonal: F[p, ri[jj]], the U^T panel column p
                const T* row = col - (int64_t)c.t * c.mc + c.t;
                const int64_t mcl = c.mc;
                chunk_add(ub, r0, max(lo, c.t + 1), hi, c.ri, lane, [&](int q) { return (double)row[q * mcl]; });
            }
            __syncwarp();
        }
        for (int i = lane; i < len; i += 32) {
            lcol[r0 + i] = lb[i];
            if (GEN && panel) ucol[r0 + i] = ub[i];
        }
        __syncwarp();
        r0 = r1;
    }
}

template <typename T>
cudaError_t launch_assemble_large(int structure, const LargeAsmArgs<T>& a, int nmembers, cudaStream_t st) {
    dim3 grid((a.count + ASM_WARPS - 1) / ASM_WARPS, nmembers);
    switch (structure) {
        case STRUCT_SPD: assemble_large_kernel<T, STRUCT_SPD><<<grid, ASM_WARPS * 32, 0, st>>>(a); break;
        case STRUCT_S: assemble_large_kernel<T, STRUCT_S><<<grid, ASM_WARPS * 32, 0, st>>>(a); break;
        default: assemble_large_kernel<T, STRUCT_G><<<grid, ASM_WARPS * 32, 0, st>>>(a);
    }
    return cudaGetLastError();
}

template cudaError_t launch_assemble_large<double>(int, const LargeAsmArgs<double>&, int, cudaStream_t);
template cudaError_t launch_assemble_large<float>(int, const LargeAsmArgs<float>&, int, cudaStream_t);

// ---------------------------------------------------------------------------
// Totals of the per-front statistics and the smallest failed factor column
// (reduce_stats! src/numeric/ldlt.jl:1276-1340, _cholesky_stats_kernel!
// src/numeric/factorize.jl:13-45): one CTA per member, no atomics.
__global__ void stats_kernel(StatsArgs A) {
    const int member = A.members ? A.members[blockIdx.x] : blockIdx.x;
    __shared__ int64_t red[NSTAT + 1][256];
    int64_t acc[NSTAT] = {0, 0, 0, 0, 0, 0};
    int64_t best = INT64_MAX;
    const int64_t* S = A.stats + (int64_t)member * A.ns * NSTAT;
    for (int s = threadIdx.x; s < A.ns; s += blockDim.x) {
        for (int q = 0; q < NSTAT - 1; ++q) acc[q] += S[(int64_t)s * NSTAT + q];
        int64_t fi = S[(int64_t)s * NSTAT + ST_INFO];
        if (fi != 0) {
            acc[ST_INFO] += 1;
            best = min(best, (int64_t)A.super_ptr0[s] + fi - 1);
        }
    }
    for (int q = 0; q < NSTAT; ++q) red[q][threadIdx.x] = acc[q];
    red[NSTAT][threadIdx.x] = best;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            for (int q = 0; q < NSTAT; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + h];
            red[NSTAT][threadIdx.x] = min(red[NSTAT][threadIdx.x], red[NSTAT][threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int q = 0; q < NSTAT; ++q) A.totals[(int64_t)member * NSTAT + q] = red[q][0];
        int64_t b = red[NSTAT][0];
        A.info[member] = b == INT64_MAX ? 0 : (int64_t)A.perm0[b] + 1;  // original column, 1-based
    }
}

cudaError_t launch_stats(const StatsArgs& a, int nmembers, cudaStream_t st) {
    stats_kernel<<<nmembers, 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace sds

// Pivoting kernels of the wide LDLT / LU fronts: the reference's in-front steps (front_factor.cuh,
// pivot.cuh) on the global panels, by one CTA (large_pivot_kernel, batched plans) or by a group of
// co-resident CTAs (large_pivot_coop_kernel, one-member plans).
//
// This file is compiled without floating-point contraction (--fmad=false), like the small-front
// kernels: the reference computes a - b c as a rounded product and a rounded difference
// (src/reference/ldlt.jl, src/reference/lu.jl, and its KernelAbstractions front kernels), and a
// fused multiply-add can leave a tiny residue where that arithmetic cancels to exactly zero, which
// changes the sign of a statically perturbed pivot and with it the inertia.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "common.cuh"
#include "front_factor.cuh"
#include "kernels.cuh"

namespace sds {

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

static_assert(COOP_ROWS == COOP_THREADS, "an update item holds one row per thread");

// Multipliers of one elimination step of the cooperative kernel
struct CoopStep {
    double dk;                    // LDLT 1x1 pivot
    double e11, e12, e21, e22;    // LDLT 2x2: the inverse of the pivot block
    double b;                     // LDLT 2x2: its subdiagonal entry
};

// Eight values per lane (columns u = 0..7 of the lane's row) -> the warp's maximum of column
// (lane >> 2) & 7 in every lane: a butterfly that halves the columns a lane keeps (7 exchanges), then
// two plain ones. jmax is exact in any order.
__device__ __forceinline__ double transpose_jmax8(double (&v)[8], int lane) {
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        const int o = 16 >> s, n = 4 >> s;
        const bool hi = (lane & o) != 0;
#pragma unroll
        for (int u = 0; u < n; ++u) {
            const double keep = hi ? v[u + n] : v[u];
            const double send = hi ? v[u] : v[u + n];
            v[u] = jmax(keep, __shfl_xor_sync(0xffffffffu, send, o));
        }
    }
    double r = v[0];
    r = jmax(r, __shfl_xor_sync(0xffffffffu, r, 2));
    r = jmax(r, __shfl_xor_sync(0xffffffffu, r, 1));
    return r;
}

// One update item of the cooperative kernel over the panel: row i = q COOP_ROWS + tid of chunk q
// (when i >= ilo), columns [jb, je) (at most COOP_COLS, all < w); for "G" only entries on or below
// the diagonal (the others are the U^T part). KIND 0 only reads (the first maxima), 1 is an LDLT 1x1
// step, 2 an LDLT 2x2 step, 3 an LU step. The arithmetic is the sequential update's:
//   1x1  F[i, j] -= T(F[i, k] / dk) F[k, j]
//   2x2  F[i, j] -= T(l1) F[k, j] + T(l2) F[k + 1, j],  (l1, l2) = (F[i, k], F[i, k + 1]) E
//   LU   F[i, j] -= F[i, k] / T(dk) F[k, j]
// Loads go out eight columns at a time. The maxima of the first nmax columns over the item's rows
// >= w go to part[j nch + q] (all threads of the CTA call this with the same arguments).
template <int KIND, typename T, bool GEN>
__device__ void coop_panel_item(const CoopStore<T, GEN>& F, int k, int q, int ilo, int jb, int je, int nmax,
                                const CoopStep& cs, T tdk, double (*pred)[COOP_COLS], int tid) {
    const int warp = tid >> 5, lane = tid & 31;
    const int i = q * COOP_ROWS + tid;
    const bool live = i >= ilo && i < F.f;
    const bool below = live && i >= F.w;
    T l1 = T(0), l2 = T(0);
    if (KIND != 0 && live) {
        if (KIND == 1) {
            l1 = T(F.get(i, k) / cs.dk);
        } else if (KIND == 2) {
            const double x1 = F.get(i, k), x2 = F.get(i, k + 1);
            l1 = T(x1 * cs.e11 + x2 * cs.e21);
            l2 = T(x1 * cs.e12 + x2 * cs.e22);
        } else {
            l1 = F.at(i, k) / tdk;
        }
    }
    for (int u0 = 0; jb + u0 < je; u0 += 8) {
        T a[8], b1[8], b2[8];
        double mx[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int j = jb + u0 + u;
            const bool ok = live && j < je && (!GEN || i >= j);
            if (KIND != 0) b1[u] = j < je ? F.at(k, j) : T(0);
            if (KIND == 2) b2[u] = j < je ? F.at(k + 1, j) : T(0);
            a[u] = ok ? F.at(i, j) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int j = jb + u0 + u;
            const bool ok = live && j < je && (!GEN || i >= j);
            T v = a[u];
            if (KIND != 0 && ok) {
                if (KIND == 2) v -= l1 * b1[u] + l2 * b2[u];
                else v -= l1 * b1[u];
                F.at(i, j) = v;
            }
            mx[u] = ok && below ? fabs((double)v) : 0.0;
        }
        if (u0 < nmax) {
            const double r = transpose_jmax8(mx, lane);
            if ((lane & 3) == 0) pred[warp][u0 + ((lane >> 2) & 7)] = r;
        }
    }
    if (nmax > 0) {
        __syncthreads();
        if (tid < nmax) {
            double m = pred[0][tid];
            for (int x = 1; x < COOP_THREADS / 32; ++x) m = jmax(m, pred[x][tid]);
            F.part[(int64_t)(jb + tid) * F.nch + q] = m;
        }
        __syncthreads();
    }
}

// The U^T part of an LU step: rows [rb, re) (fully-summed, > k) against column j = cb + tid (one per
// thread, i < j < f), F[i, j] -= F[i, k] / T(dk) F[k, j]; coalesced in the U^T panel (U[j + i f])
template <typename T>
__device__ void coop_u_item(const CoopStore<T, true>& F, int k, int rb, int re, int cb, T tdk, int tid) {
    const int j = cb + tid;
    if (j >= F.f || j <= rb) return;
    const int64_t f = F.f;
    const T fkj = F.U[j + k * f];
    for (int i0 = rb; i0 < re; i0 += 8) {
        T l[8], a[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + u;
            const bool ok = i < re && i < j;
            l[u] = ok ? F.P[i + k * f] / tdk : T(0);
            a[u] = ok ? F.U[j + i * f] : T(0);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + u;
            if (i < re && i < j) F.U[j + i * f] = a[u] - l[u] * fkj;
        }
    }
}

// Wide LDLT / LU fronts on a group of co-resident CTAs (one group per front of the launch, barriers
// over the group). A step: CTA 0 takes the pivot decision while every CTA writes the previous step's
// multipliers into its column (the update needs them unscaled until then); barrier; the interchange
// (one phase) and a barrier when there is one; the update, which also leaves the maxima of the updated
// fully-summed columns over each chunk of rows below the block, so that the next decision scans only
// the w fully-summed rows; barrier. The decisions and the arithmetic are those of the sequential
// kernel.
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
    const int tid = threadIdx.x, nt = blockDim.x;
    const int gt = rank * nt + tid, GT = gs * nt;
    const bool lead = rank == 0 && tid == 0;
    const int nch = (f + COOP_ROWS - 1) / COOP_ROWS;
    const CoopStore<T, GEN> F{{P, U, f, w}, scr + pivot_scratch_base(f, w), nch, w / COOP_ROWS};
    __shared__ double team_red[COOP_THREADS / 32];
    __shared__ int team_redi[COOP_THREADS / 32];
    __shared__ double pred[COOP_THREADS / 32][COOP_COLS];
    const CtaTeam team{tid, nt, team_red, team_redi};
    if (STRUCT == STRUCT_S) {
        for (int q = gt; q < w * w; q += GT) {
            const int i = q % w, j = q / w;
            if (i > j) P[j + (int64_t)i * f] = P[i + (int64_t)j * f];
        }
    }
    for (int q = gt; q < w; q += GT) sc.lp[q] = q;
    {   // maxima below the block of the columns the first decision may scan (all for "S", column 0 for "G")
        const int nq = nch - F.q0, ncg = GEN ? 1 : (w + COOP_COLS - 1) / COOP_COLS;
        for (int it = rank; it < nq * ncg; it += gs) {
            const int q = F.q0 + it % nq, jb = (it / nq) * COOP_COLS;
            const int je = GEN ? 1 : min(w, jb + COOP_COLS);
            coop_panel_item<0>(F, 0, q, w, jb, je, je - jb, CoopStep{}, T(1), pred, tid);
        }
    }
    group_barrier(bar, epoch, gs, G.status);
    int64_t st[NSTAT] = {0, 0, 0, 0, 0, 0};
    if constexpr (STRUCT == STRUCT_S) {
        int pk = -1, pkind = 0;   // the step whose multipliers are still to be written (1: 1x1, 2: 2x2)
        CoopStep pc{};
        // write the multipliers of step pk into its column(s); the pivot block's own entries (which the
        // final pass overwrites) only before the last step
        auto flush = [&](bool last) {
            if (pkind == 1) {
                for (int i = pk + 1 + gt; i < f; i += GT) F.at(i, pk) = T(F.get(i, pk) / pc.dk);
                if (lead && !last) F.at(pk, pk) = T(pc.dk);
            } else if (pkind == 2) {
                for (int i = pk + 2 + gt; i < f; i += GT) {
                    const double x1 = F.get(i, pk), x2 = F.get(i, pk + 1);
                    F.at(i, pk) = T(x1 * pc.e11 + x2 * pc.e21);
                    F.at(i, pk + 1) = T(x1 * pc.e12 + x2 * pc.e22);
                }
                if (lead) {
                    if (!last) F.at(pk, pk + 1) = T(pc.b);
                    F.at(pk + 1, pk) = T(0);
                }
            }
        };
        int k = 0;
        while (k < w) {
            flush(false);
            if (rank == 0) {   // the whole first CTA takes the decision (row scans split over its threads)
                int c, r;
                choose_pivot(F, k, w, A.pivot, A.u, A.eps, team, c, r);
                if (tid == 0) { sc.ctl[0] = c; sc.ctl[1] = r; }
            }
            group_barrier(bar, epoch, gs, G.status);
            const int c = sc.ctl[0], r = sc.ctl[1];
            const int p = r < 0 ? k : k + 1, qsw = r < 0 ? c : r;
            if (p != qsw) {
                // the symmetric interchange of p and qsw: columns (rows other than p, qsw), rows (columns
                // other than p, qsw) and the 2x2 block they share, in one phase
                for (int i = gt; i < f; i += GT) {
                    if (i == p || i == qsw) continue;
                    T t = F.at(i, p); F.at(i, p) = F.at(i, qsw); F.at(i, qsw) = t;
                }
                for (int j = gt; j < w; j += GT) {
                    if (j == p || j == qsw) continue;
                    T t = F.at(p, j); F.at(p, j) = F.at(qsw, j); F.at(qsw, j) = t;
                }
                if (lead) {
                    T t = F.at(p, p); F.at(p, p) = F.at(qsw, qsw); F.at(qsw, qsw) = t;
                    t = F.at(p, qsw); F.at(p, qsw) = F.at(qsw, p); F.at(qsw, p) = t;
                    int tl = sc.lp[p]; sc.lp[p] = sc.lp[qsw]; sc.lp[qsw] = tl;
                }
                group_barrier(bar, epoch, gs, G.status);
            }
            CoopStep cs{};
            const int nb = r < 0 ? 1 : 2;
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
                if (lead) { sc.dd[k] = dk; sc.ee[k] = 0.0; sc.kd[k] = kk; }
                cs.dk = dk;
            } else {
                const double a = F.get(k, k), b = F.get(k + 1, k), c2 = F.get(k + 1, k + 1);
                const double det = a * c2 - b * b;
                cs.e11 = c2 / det; cs.e12 = -b / det; cs.e21 = -b / det; cs.e22 = a / det;
                cs.b = b;
                st[ST_N2X2]++;
                if (det < 0) { st[ST_NPOS]++; st[ST_NNEG]++; }
                else if (a > 0) st[ST_NPOS] += 2;
                else st[ST_NNEG] += 2;
                if (lead) {
                    sc.dd[k] = a; sc.dd[k + 1] = c2; sc.ee[k] = b; sc.ee[k + 1] = 0.0;
                    sc.kd[k] = KIND_2X2_FIRST; sc.kd[k + 1] = KIND_2X2_SECOND;
                }
            }
            const int j0 = k + nb, qa = j0 / COOP_ROWS, nq = nch - qa;
            const int ncg = (w - j0 + COOP_COLS - 1) / COOP_COLS;
            for (int it = rank; it < nq * ncg; it += gs) {
                const int q = qa + it % nq, jb = j0 + (it / nq) * COOP_COLS, je = min(w, jb + COOP_COLS);
                const int nmax = q >= F.q0 ? je - jb : 0;
                if (r < 0) coop_panel_item<1>(F, k, q, j0, jb, je, nmax, cs, T(1), pred, tid);
                else coop_panel_item<2>(F, k, q, j0, jb, je, nmax, cs, T(1), pred, tid);
            }
            group_barrier(bar, epoch, gs, G.status);
            pk = k; pkind = nb; pc = cs;
            k += nb;
        }
        flush(true);
    } else {
        const bool pivoting = A.lu_pivot != 0;
        int pk = -1;
        T ptdk = T(1);
        double pdk = 0.0;
        // scale column pk into L and row pk into U (the update reads them unscaled); D into the pivot
        // entry before the last step (the final pass overwrites it)
        auto flush = [&](bool last) {
            if (pk < 0) return;
            for (int i = pk + 1 + gt; i < f; i += GT) F.at(i, pk) /= ptdk;
            for (int j = pk + 1 + gt; j < f; j += GT) F.at(pk, j) /= ptdk;
            if (lead && !last) F.at(pk, pk) = T(pdk);
        };
        for (int k = 0; k < w; ++k) {
            flush(false);
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
            if (lead) { sc.dd[k] = dk; sc.kd[k] = kk; }
            const T tdk = T(dk);
            const int qa = (k + 1) / COOP_ROWS, nq = nch - qa;
            const int ncg = (w - k - 1 + COOP_COLS - 1) / COOP_COLS;       // column groups; also row groups of U^T
            const int nct = (f - k - 1 + COOP_ROWS - 1) / COOP_ROWS;       // column tiles of U^T
            const int nl = nq * ncg;
            for (int it = rank; it < nl + ncg * nct; it += gs) {
                if (it < nl) {
                    const int q = qa + it % nq, g = it / nq;
                    const int jb = k + 1 + g * COOP_COLS, je = min(w, jb + COOP_COLS);
                    coop_panel_item<3>(F, k, q, k + 1, jb, je, (g == 0 && q >= F.q0) ? 1 : 0, CoopStep{}, tdk, pred,
                                       tid);
                } else {
                    const int u = it - nl, rg = u % ncg, ct = u / ncg;
                    const int rb = k + 1 + rg * COOP_COLS, re = min(w, rb + COOP_COLS);
                    coop_u_item(F, k, rb, re, k + 1 + ct * COOP_ROWS, tdk, tid);
                }
            }
            group_barrier(bar, epoch, gs, G.status);
            pk = k; ptdk = tdk; pdk = dk;
        }
        flush(true);
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

}  // namespace sds

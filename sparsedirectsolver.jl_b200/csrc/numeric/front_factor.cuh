// In-front dense factorization steps of LDLT (Bunch-Kaufman) and LU (threshold
// partial pivoting), written once over a front-storage abstraction so that the
// same arithmetic runs on shared-memory fronts (small fronts) and on the
// global-memory panels of large fronts. One CTA runs a front; warp 0 takes the
// pivot decisions (pivot.cuh), the CTA applies interchanges and updates.
// Restates _ldlt_front! (src/reference/ldlt.jl:384-454) and _lu_front!
// (src/reference/lu.jl:174-212) of the reference: the updates touch only the
// w fully-summed columns (and, for LU, the fully-summed rows); the contribution
// block is updated afterwards by the caller.
#pragma once
#include "common.cuh"
#include "pivot.cuh"

namespace sds {

// Scratch of one front: multipliers (2 f), D (w + w), local order (w), kinds (w), control (16)
struct FrontScratch {
    double* lvec;
    double* dd;
    double* ee;
    int* lp;
    signed char* kd;
    int* ctl;
};

template <typename T>
struct SmemStore {
    T* a;
    int ld, f, w;
    __device__ T& at(int i, int j) const { return a[i + j * ld]; }
    __device__ double get(int i, int j) const { return (double)a[i + j * ld]; }
    __device__ int scan_rows() const { return f; }
    __device__ double part_max(int, int, int) const { return 0.0; }
};

// Large-front storage: F[:, 0:w] in the panel P (ld f); for "G" the strict upper
// part F[i, j] (i < j, i < w) in the U^T panel U at U[j + i f].
template <typename T, bool GEN>
struct GlobalStore {
    T* P;
    T* U;
    int f, w;
    __device__ T& at(int i, int j) const {
        if (!GEN || (i >= j && j < w)) return P[i + (int64_t)j * f];
        return U[j + (int64_t)i * f];
    }
    __device__ double get(int i, int j) const { return (double)at(i, j); }
    __device__ int scan_rows() const { return f; }
    __device__ double part_max(int, int, int) const { return 0.0; }
};

// Large-front storage of the cooperative kernel: column scans read the fully-summed rows and take
// the rows below from per-chunk maxima that the update phase leaves behind.
template <typename T, bool GEN>
struct CoopStore : GlobalStore<T, GEN> {
    double* part;   // part[c nch + q]: max |F[i, c]| over the rows i >= w of row chunk q (COOP_ROWS rows)
    int nch, q0;    // row chunks of the front; q0: the first that holds a row >= w
    __device__ int scan_rows() const { return this->w; }
    __device__ double part_max(int c, int rank, int size) const {
        double m = 0.0;
        for (int q = q0 + rank; q < nch; q += size) m = jmax(m, part[(int64_t)c * nch + q]);
        return m;
    }
};

__device__ __forceinline__ double perturb_sign_of(double d, int requested) {
    if (requested != 0) return (double)requested;
    return d < 0 ? -1.0 : 1.0;
}

// LDLT of the fully-summed columns. psign_row(local column) gives the requested sign.
// st[] accumulates the statistics (all threads hold identical copies).
template <typename T, class Store>
__device__ void ldlt_front_steps(const Store& F, const FrontScratch& S, int f, int w, int pivot, double u, double eps,
                                 const signed char* psign, const int* perm, int c0, int64_t* st) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    for (int q = tid; q < w; q += nt) S.lp[q] = q;
    __syncthreads();
    int k = 0;
    while (k < w) {
        if (warp == 0) {
            int c, r;
            choose_pivot_w(F, k, w, pivot, u, eps, lane, c, r);
            if (lane == 0) { S.ctl[0] = c; S.ctl[1] = r; }
        }
        __syncthreads();
        const int c = S.ctl[0], r = S.ctl[1];
        const int p = r < 0 ? k : k + 1, qsw = r < 0 ? c : r;
        if (p != qsw) {
            for (int i = tid; i < f; i += nt) {
                T t = F.at(i, p); F.at(i, p) = F.at(i, qsw); F.at(i, qsw) = t;
            }
            __syncthreads();
            for (int j = tid; j < w; j += nt) {
                T t = F.at(p, j); F.at(p, j) = F.at(qsw, j); F.at(qsw, j) = t;
            }
            if (tid == 0) { int t = S.lp[p]; S.lp[p] = S.lp[qsw]; S.lp[qsw] = t; }
            __syncthreads();
        }
        if (r < 0) {
            double dk = F.get(k, k);
            signed char kk = KIND_1X1;
            if (!(fabs(dk) >= eps) || dk == 0.0) {
                if (dk == 0.0) st[ST_NZERO]++;
                int req = psign ? (int)psign[perm[c0 + S.lp[k]]] : 0;
                dk = perturb_sign_of(dk, req) * eps;
                kk = KIND_PERTURBED;
                st[ST_NPERT]++;
                if (dk == 0.0 && st[ST_INFO] == 0) st[ST_INFO] = S.lp[k] + 1;
            }
            if (dk > 0) st[ST_NPOS]++;
            else if (dk < 0) st[ST_NNEG]++;
            __syncthreads();
            for (int i = k + 1 + tid; i < f; i += nt) S.lvec[i] = F.get(i, k) / dk;
            if (tid == 0) { F.at(k, k) = T(dk); S.dd[k] = dk; S.ee[k] = 0.0; S.kd[k] = kk; }
            __syncthreads();
            for (int j = k + 1 + warp; j < w; j += nwarps) {
                const T fkj = F.at(k, j);
                for (int i = k + 1 + lane; i < f; i += 32) F.at(i, j) -= T(S.lvec[i]) * fkj;
            }
            __syncthreads();
            for (int i = k + 1 + tid; i < f; i += nt) F.at(i, k) = T(S.lvec[i]);
            __syncthreads();
            k += 1;
        } else {
            double a = F.get(k, k), b = F.get(k + 1, k), c2 = F.get(k + 1, k + 1);
            double det = a * c2 - b * b;
            double e11 = c2 / det, e12 = -b / det, e21 = -b / det, e22 = a / det;
            st[ST_N2X2]++;
            if (det < 0) { st[ST_NPOS]++; st[ST_NNEG]++; }
            else if (a > 0) st[ST_NPOS] += 2;
            else st[ST_NNEG] += 2;
            __syncthreads();
            for (int i = k + 2 + tid; i < f; i += nt) {
                double x1 = F.get(i, k), x2 = F.get(i, k + 1);
                S.lvec[i] = x1 * e11 + x2 * e21;
                S.lvec[f + i] = x1 * e12 + x2 * e22;
            }
            if (tid == 0) {
                F.at(k, k + 1) = T(b);
                S.dd[k] = a; S.dd[k + 1] = c2; S.ee[k] = b; S.ee[k + 1] = 0.0;
                S.kd[k] = KIND_2X2_FIRST; S.kd[k + 1] = KIND_2X2_SECOND;
            }
            __syncthreads();
            for (int j = k + 2 + warp; j < w; j += nwarps) {
                const T fkj = F.at(k, j), fk1j = F.at(k + 1, j);
                for (int i = k + 2 + lane; i < f; i += 32)
                    F.at(i, j) -= T(S.lvec[i]) * fkj + T(S.lvec[f + i]) * fk1j;
            }
            __syncthreads();
            for (int i = k + 2 + tid; i < f; i += nt) {
                F.at(i, k) = T(S.lvec[i]);
                F.at(i, k + 1) = T(S.lvec[f + i]);
            }
            if (tid == 0) F.at(k + 1, k) = T(0);
            __syncthreads();
            k += 2;
        }
    }
}

// LU of the fully-summed columns with row interchanges among the fully-summed rows.
template <typename T, class Store>
__device__ void lu_front_steps(const Store& F, const FrontScratch& S, int f, int w, bool pivoting, double u,
                               double eps, int64_t* st) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    for (int q = tid; q < w; q += nt) S.lp[q] = q;
    __syncthreads();
    for (int k = 0; k < w; ++k) {
        if (warp == 0) {
            int r = pivoting ? lu_choose_row_w(F, k, w, u, lane) : k;
            if (lane == 0) S.ctl[0] = r;
        }
        __syncthreads();
        const int r = S.ctl[0];
        if (r != k) {
            for (int j = tid; j < f; j += nt) {
                T t = F.at(k, j); F.at(k, j) = F.at(r, j); F.at(r, j) = t;
            }
            if (tid == 0) { int t = S.lp[k]; S.lp[k] = S.lp[r]; S.lp[r] = t; }
            __syncthreads();
        }
        double dk = F.get(k, k);
        signed char kk = KIND_1X1;
        if (!(fabs(dk) >= eps) || dk == 0.0) {
            if (dk == 0.0) st[ST_NZERO]++;
            dk = perturb_sign_of(dk, 0) * eps;
            kk = KIND_PERTURBED;
            st[ST_NPERT]++;
            if (dk == 0.0 && st[ST_INFO] == 0) st[ST_INFO] = k + 1;
        }
        __syncthreads();
        if (tid == 0) { F.at(k, k) = T(dk); S.dd[k] = dk; S.kd[k] = kk; }
        const T tdk = T(dk);
        for (int j = k + 1 + warp; j < f; j += nwarps) {
            const T fkj = F.at(k, j);
            const int iend = j < w ? f : w;
            for (int i = k + 1 + lane; i < iend; i += 32) F.at(i, j) -= F.at(i, k) / tdk * fkj;
        }
        __syncthreads();
        for (int i = k + 1 + tid; i < f; i += nt) F.at(i, k) /= tdk;
        for (int j = k + 1 + tid; j < f; j += nt) F.at(k, j) /= tdk;
        __syncthreads();
    }
}

}  // namespace sds

// Pivot decisions of the in-front LDLT (Bunch-Kaufman) and LU (threshold partial
// pivoting), run by one warp or one CTA over a front accessor. They restate the reference's
// decision sequence exactly (SparseDirectSolver.jl src/reference/ldlt.jl:254-355,
// src/reference/lu.jl:216-231), including its NaN semantics: Julia's max
// propagates NaN, so a NaN in a scanned column fails the threshold tests, and a
// strict `>` arg-max never selects a NaN. All comparisons are made in FP64 on the
// front's values (exact for FP32 fronts).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace sds {

__device__ __forceinline__ double jmax(double a, double b) {  // Julia max: NaN if either is NaN
    return (a != a || b != b) ? (a + b) : (a > b ? a : b);
}

__device__ __forceinline__ double warp_jmax(double v) {
    for (int o = 16; o > 0; o >>= 1) v = jmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// arg-max with strict > (first index on ties, NaN never wins); returns index (-1 none) in all lanes
__device__ __forceinline__ void warp_argmax(double& v, int& idx) {
    for (int o = 16; o > 0; o >>= 1) {
        double ov = __shfl_xor_sync(0xffffffffu, v, o);
        int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        bool take = (ov > v) || (ov == v && oi >= 0 && (idx < 0 || oi < idx));
        if (take) { v = ov; idx = oi; }
    }
}

// Teams: the threads that take a pivot decision together. Every thread of a team runs the same
// decision sequence on the same values; only the scans over rows are split among them and reduced.
// Max and first-index arg-max are exact in any order (jmax propagates NaN whatever the order), so a
// warp team and a CTA team take identical decisions.
struct WarpTeam {
    int rank;                      // lane
    static constexpr int size = 32;
    __device__ double reduce_jmax(double v) const { return warp_jmax(v); }
    __device__ void reduce_argmax(double& v, int& idx) const { warp_argmax(v, idx); }
};

// all threads of a CTA (every thread must take part in every reduction); red, redi: shared scratch
// of blockDim.x / 32 entries
struct CtaTeam {
    int rank, size;
    double* red;
    int* redi;
    __device__ double reduce_jmax(double v) const {
        v = warp_jmax(v);
        __syncthreads();
        if ((rank & 31) == 0) red[rank >> 5] = v;
        __syncthreads();
        double r = red[0];
        for (int w = 1; w < (size >> 5); ++w) r = jmax(r, red[w]);
        return r;
    }
    __device__ void reduce_argmax(double& v, int& idx) const {
        warp_argmax(v, idx);
        __syncthreads();
        if ((rank & 31) == 0) {
            red[rank >> 5] = v;
            redi[rank >> 5] = idx;
        }
        __syncthreads();
        double bv = red[0];
        int bi = redi[0];
        for (int w = 1; w < (size >> 5); ++w) {
            const double ov = red[w];
            const int oi = redi[w];
            if ((ov > bv) || (ov == bv && oi >= 0 && (bi < 0 || oi < bi))) {
                bv = ov;
                bi = oi;
            }
        }
        v = bv;
        idx = bi;
    }
};

// Front accessor interface: F(i, j) returns the current value (double) of entry (i, j).
// Acc must provide: double get(int i, int j) const; int f; int w; int scan_rows() const (the rows
// 0..scan_rows()-1 a column scan reads); double part_max(int c, int rank, int size) const (this
// team member's share of max |F[i, c]| over the rows from scan_rows() on, kept by the accessor;
// 0.0 when scan_rows() == f).

// max |F[i, c]| over rows k..f-1, skipping c and skip (Julia max semantics); c and skip are
// fully-summed rows, so they are never among the rows the accessor keeps maxima for
template <class Acc, class Team>
__device__ double colmax(const Acc& F, int c, int k, int skip, const Team& tm) {
    double m = 0.0;
    for (int i = k + tm.rank; i < F.scan_rows(); i += tm.size) {
        if (i == c || i == skip) continue;
        m = jmax(m, fabs(F.get(i, c)));
    }
    m = jmax(m, F.part_max(c, tm.rank, tm.size));
    return tm.reduce_jmax(m);
}

// d >= u * max_{i != c, i >= k} |F[i, c]| with the reference's early-exit semantics
// (equivalent to: no NaN in the column and the test on the maximum)
template <class Acc, class Team>
__device__ bool threshold_ok(const Acc& F, int c, int k, double u, double d, const Team& tm) {
    double m = colmax(F, c, k, -1, tm);
    return d >= u * m;
}

template <class Acc, class Team>
__device__ bool accept_1x1(const Acc& F, int c, int k, double u, double eps, const Team& tm) {
    double d = fabs(F.get(c, c));
    if (!(d >= eps)) return false;
    return threshold_ok(F, c, k, u, d, tm);
}

template <class Acc>
__device__ bool nonsingular_2x2_w(const Acc& F, int k, int r, double eps) {
    double akk = F.get(k, k), arr = F.get(r, r), akr = F.get(k, r), ark = F.get(r, k);
    double det = akk * arr - akr * ark;
    double mx = jmax(jmax(fabs(akk), fabs(ark)), fabs(arr));
    return det != 0.0 && isfinite(det) && mx >= eps;
}

template <class Acc, class Team>
__device__ bool accept_2x2(const Acc& F, int k, int r, double u, double eps, const Team& tm) {
    if (!nonsingular_2x2_w(F, k, r, eps)) return false;
    double akk = F.get(k, k), arr = F.get(r, r), akr = F.get(k, r), ark = F.get(r, k);
    double det = akk * arr - akr * ark;
    double e11 = fabs(arr / det), e12 = fabs(akr / det), e21 = fabs(ark / det), e22 = fabs(akk / det);
    double m1 = colmax(F, k, k, r, tm), m2 = colmax(F, r, k, k, tm);
    return u * (e11 * m1 + e21 * m2) <= 1.0 && u * (e12 * m1 + e22 * m2) <= 1.0;
}

// acceptable 1x1 pivot of the block k..w-1 with the largest |a_jj|, first on ties; -1 if none
template <class Acc, class Team>
__device__ int best_1x1(const Acc& F, int k, int w, double u, double eps, const Team& tm) {
    int best = -1;
    double bv = 0.0;
    for (int j = k; j < w; ++j) {
        double a = fabs(F.get(j, j));
        if (!(a >= eps)) continue;
        if (best >= 0 && !(a > bv)) continue;
        if (!threshold_ok(F, j, k, u, a, tm)) continue;
        best = j;
        bv = a;
    }
    return best;
}

// Pivot choice at column k: sets c (1x1 at c, r = -1) or the 2x2 on (k, r). Team-uniform result.
template <class Acc, class Team>
__device__ void choose_pivot(const Acc& F, int k, int w, int pivot, double u, double eps, const Team& tm,
                             int& c_out, int& r_out) {
    r_out = -1;
    if (pivot == PIVOT_NONE) { c_out = k; return; }
    if (pivot == PIVOT_DIAGONAL) {
        if (accept_1x1(F, k, k, u, eps, tm)) { c_out = k; return; }
        int best = best_1x1(F, k, w, u, eps, tm);
        if (best >= 0) { c_out = best; return; }
        int big = k;
        for (int j = k + 1; j < w; ++j)
            if (fabs(F.get(j, j)) > fabs(F.get(big, big))) big = j;
        c_out = fabs(F.get(big, big)) >= eps ? big : k;
        return;
    }
    const double alpha = (1.0 + sqrt(17.0)) / 8.0;
    double lambda = 0.0;
    int r = -1;
    for (int i = k + 1 + tm.rank; i < w; i += tm.size) {
        double a = fabs(F.get(i, k));
        if (a > lambda) { lambda = a; r = i; }
    }
    tm.reduce_argmax(lambda, r);
    double akk = fabs(F.get(k, k));
    int bc = k, br = -1;
    if (r < 0 || akk >= alpha * lambda) {
        bc = k;
    } else {
        double sigma = 0.0;
        for (int i = k + tm.rank; i < w; i += tm.size)
            if (i != r) sigma = jmax(sigma, fabs(F.get(i, r)));
        sigma = tm.reduce_jmax(sigma);
        if (akk * sigma >= alpha * lambda * lambda) bc = k;
        else if (fabs(F.get(r, r)) >= alpha * sigma) bc = r;
        else { bc = k; br = r; }
    }
    bool acc = br < 0 ? accept_1x1(F, bc, k, u, eps, tm) : accept_2x2(F, k, br, u, eps, tm);
    if (acc) { c_out = bc; r_out = br; return; }
    int best = best_1x1(F, k, w, u, eps, tm);
    if (best >= 0) { c_out = best; return; }
    if (br >= 0 && nonsingular_2x2_w(F, k, br, eps)) { c_out = bc; r_out = br; return; }
    c_out = bc;
}

// LU row choice (lu.jl:216-231): the diagonal if |F[k,k]| >= u max_{i>=k} |F[i,k]|,
// else the first fully-summed row with the largest |F[r,k]|.
template <class Acc, class Team>
__device__ int lu_choose_row(const Acc& F, int k, int w, double u, const Team& tm) {
    double g = 0.0;
    for (int i = k + tm.rank; i < F.scan_rows(); i += tm.size) g = jmax(g, fabs(F.get(i, k)));
    g = jmax(g, F.part_max(k, tm.rank, tm.size));
    g = tm.reduce_jmax(g);
    double akk = fabs(F.get(k, k));
    if (akk >= u * g) return k;
    double best = -1.0;
    int r = -1;
    for (int i = k + 1 + tm.rank; i < w; i += tm.size) {
        double a = fabs(F.get(i, k));
        if (a > best) { best = a; r = i; }
    }
    tm.reduce_argmax(best, r);
    // the reference starts from (k, akk) and takes a row only when strictly larger
    if (r >= 0 && best > akk) return r;
    return k;
}

// one-warp entry points (lane = the calling thread's lane)
template <class Acc>
__device__ void choose_pivot_w(const Acc& F, int k, int w, int pivot, double u, double eps, int lane, int& c_out,
                               int& r_out) {
    choose_pivot(F, k, w, pivot, u, eps, WarpTeam{lane}, c_out, r_out);
}

template <class Acc>
__device__ int lu_choose_row_w(const Acc& F, int k, int w, double u, int lane) {
    return lu_choose_row(F, k, w, u, WarpTeam{lane});
}

}  // namespace sds

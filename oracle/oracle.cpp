// CPU oracle of the numeric phase -- TEST INFRASTRUCTURE ONLY (see oracle.h).
//
// Restates SparseDirectSolver.jl's CPU reference factorizations:
//   ref_factorize!  src/reference/cholesky.jl:44-111
//   ref_ldlt!       src/reference/ldlt.jl:121-202, _choose_pivot :314-355, _ldlt_front! :384-454
//   ref_lu!         src/reference/lu.jl:84-165, _lu_front! :174-212, _lu_choose_row :216-231
//   ref_solve!      src/reference/cholesky.jl:127-170, ref_solve_ldlt! ldlt.jl:467-539,
//   ref_solve_lu!   lu.jl:278-294 (written here as the equivalent supernodal sweeps)
// Fronts are dense column-major f x f host matrices; the dense kernels are plain
// loops in the order of the reference's (LAPACK potrf / BLAS trsm and syrk for
// Cholesky; the explicit loops of the LDLT and LU oracles).
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

using std::vector;
typedef int64_t i64;

namespace {

const int NF = 6;  // per-front statistics: npos, nneg, nzero, nperturbed, n2x2, info
enum { ST_NPOS = 0, ST_NNEG, ST_NZERO, ST_NPERT, ST_N2X2, ST_INFO };
enum { KIND_1X1 = 1, KIND_2X2_FIRST = 2, KIND_2X2_SECOND = 3, KIND_PERTURBED = 4 };
enum { PIV_AUTO = 0, PIV_NONE = 1, PIV_DIAGONAL = 4, PIV_LOCAL = 5, PIV_BK = 6 };

struct Front {
    i64 f, w;
    vector<double> a;  // f x f column-major
    double& operator()(i64 i, i64 j) { return a[i + j * f]; }  // 0-based
};

struct Ctx {
    const oracle_symbolic* S;
    i64 ns;
    i64 f(i64 s) const { return S->rowptr[s] - S->rowptr[s - 1]; }             // s 1-based
    i64 w(i64 s) const { return S->super_ptr[s] - S->super_ptr[s - 1]; }
    i64 base(i64 s) const { return S->front_ptr[s - 1]; }
};

// Host threads for the fronts (oracle_set_threads); 1 = the serial postorder of the reference.
int g_threads = 1;
thread_local bool t_worker = false;   // inside a level-parallel worker: the dense loops stay serial

// fn(i) for i in [lo, hi) on the host threads, when the loop is worth it (work in multiply-adds) and
// the caller is not itself a worker; each i is one thread's, so every entry sees the serial arithmetic
template <class Fn>
void parallel_for(i64 lo, i64 hi, double work, Fn fn) {
    const i64 nt = std::min<i64>(g_threads, hi - lo);
    if (nt <= 1 || t_worker || work < 5.0e5) {
        for (i64 i = lo; i < hi; ++i) fn(i);
        return;
    }
    std::atomic<i64> next(lo);
    vector<std::thread> pool;
    for (i64 k = 0; k < nt; ++k)
        pool.emplace_back([&]() {
            t_worker = true;
            for (i64 i = next++; i < hi; i = next++) fn(i);
        });
    for (std::thread& th : pool) th.join();
}

// Runs body(s) for every supernode, children before parents. Serially it follows the postorder and
// stops at the first nonzero return (a failed Cholesky pivot). With several threads, the fronts of
// one elimination-tree level run concurrently: a front reads only its children's contribution
// blocks and writes its own panel, statistics and block, so the results are those of the serial
// order. Every front is processed, and the first nonzero return in postorder is returned, which is
// the serial return value.
template <class Body>
i64 run_fronts(const Ctx& C, Body body) {
    const oracle_symbolic* S = C.S;
    if (g_threads <= 1 || C.ns < 2) {
        for (i64 t = 0; t < C.ns; ++t) {
            i64 r = body(S->snpost[t]);
            if (r) return r;
        }
        return 0;
    }
    vector<i64> level(C.ns + 1, 0);
    i64 nlev = 0;
    for (i64 t = 0; t < C.ns; ++t) {          // postorder: children first
        i64 s = S->snpost[t], p = S->snparent[s - 1];
        if (p != 0) level[p] = std::max(level[p], level[s] + 1);
        nlev = std::max(nlev, level[s] + 1);
    }
    vector<vector<i64>> bylevel(nlev);
    for (i64 t = 0; t < C.ns; ++t) bylevel[level[S->snpost[t]]].push_back(S->snpost[t]);
    vector<i64> ret(C.ns + 1, 0);
    for (const vector<i64>& fronts : bylevel) {
        const int nt = (int)std::min<i64>(g_threads, (i64)fronts.size());
        if (nt <= 1) {
            for (i64 s : fronts) ret[s] = body(s);
            continue;
        }
        std::atomic<i64> next(0);
        vector<std::thread> pool;
        for (int k = 0; k < nt; ++k)
            pool.emplace_back([&]() {
                t_worker = true;
                for (i64 q = next++; q < (i64)fronts.size(); q = next++) ret[fronts[q]] = body(fronts[q]);
            });
        for (std::thread& th : pool) th.join();
    }
    for (i64 t = 0; t < C.ns; ++t)
        if (ret[S->snpost[t]]) return ret[S->snpost[t]];
    return 0;
}

// assembly of A and extend-add of the children (cholesky.jl:67-84; lu.jl:115-131)
void assemble(const Ctx& C, i64 s, const double* nz, Front& F, vector<vector<double>>& cbs, vector<i64>& cbm,
              bool general) {
    const oracle_symbolic* S = C.S;
    i64 f = F.f, base = C.base(s);
    for (i64 k = S->amap_ptr[s - 1]; k < S->amap_ptr[s]; ++k) {
        i64 p = S->amap_src[k - 1];
        i64 off = S->amap[p - 1];
        i64 loc = std::llabs(off) - base;
        i64 i = loc % f, j = loc / f;
        if (general && off < 0) F(j, i) += nz[p - 1];
        else F(i, j) += nz[p - 1];  // real values: conj is the identity
    }
    for (i64 k = S->child_ptr[s - 1]; k < S->child_ptr[s]; ++k) {
        i64 c = S->child_list[k - 1];
        if (cbm[c] < 0) continue;
        i64 m = cbm[c];
        const i64* ri = S->relind + (S->relind_ptr[c - 1] - 1);
        vector<double>& Cb = cbs[c];
        for (i64 jj = 0; jj < m; ++jj)
            for (i64 ii = general ? 0 : jj; ii < m; ++ii) F(ri[ii] - 1, ri[jj] - 1) += Cb[ii + jj * m];
        vector<double>().swap(Cb);
        cbm[c] = -1;
    }
}

// Schur complement mode (assemble_schur!, src/numeric/schur.jl:15-98): the root supernode S->schur is
// assembled and not factored. Its panel keeps the assembled front: the lower triangle in `factor`, and
// for LU the strict upper triangle transposed in `ufactor`; its columns get the identity local order,
// unit 1x1 pivots (d = 1, no 2x2 part) and zero statistics.
void store_schur(const Ctx& C, i64 s, Front& F, bool general, double* factor, double* ufactor, double* d,
                 int32_t* piv, int8_t* kind) {
    const oracle_symbolic* S = C.S;
    const i64 f = F.f, base = C.base(s), c0 = S->super_ptr[s - 1];
    for (i64 j = 0; j < f; ++j)
        for (i64 i = j; i < f; ++i) {
            factor[base - 1 + j * f + i] = F(i, j);
            if (general && i > j) ufactor[base - 1 + j * f + i] = F(j, i);
        }
    if (!piv) return;
    for (i64 k = 0; k < f; ++k) {
        piv[c0 - 1 + k] = (int32_t)(c0 + k);
        kind[c0 - 1 + k] = KIND_1X1;
        d[c0 - 1 + k] = 1.0;
        d[S->n + c0 - 1 + k] = 0.0;
    }
}

// ---------------------------------------------------------------------------
// Cholesky (cholesky.jl:44-111). eps > 0 adds the device path's static clamp
// (src/numeric/front.jl:38-53): a pivot in [0, eps] is raised to eps.
i64 factor_cholesky(const Ctx& C, const double* nz, double eps, double* factor, int64_t* stats) {
    const oracle_symbolic* S = C.S;
    vector<vector<double>> cbs(C.ns + 1);
    vector<i64> cbm(C.ns + 1, -1);
    return run_fronts(C, [&](i64 s) -> i64 {
        i64 f = C.f(s), w = C.w(s), m = f - w, base = C.base(s);
        Front F{f, w, vector<double>(f * f, 0.0)};
        assemble(C, s, nz, F, cbs, cbm, false);
        if (s == S->schur) {
            store_schur(C, s, F, false, factor, nullptr, nullptr, nullptr, nullptr);
            return 0;
        }
        // potrf on F11 (right-looking, lower), in panels of 64 columns: a panel's columns are factored
        // in order with the updates among them, then every later column takes the panel's updates in
        // increasing j. Each entry receives the updates of j = 0, 1, ... in order, as in the unblocked
        // loop; the later columns of a panel run on the host threads.
        constexpr i64 PB = 64;
        for (i64 j0 = 0; j0 < w; j0 += PB) {
            const i64 j1 = std::min(w, j0 + PB);
            for (i64 j = j0; j < j1; ++j) {
                double ajj = F(j, j);
                bool ok = ajj > eps || (eps > 0 && ajj >= 0);
                if (!ok) {
                    stats[(s - 1) * NF + ST_NPOS] = j;
                    stats[(s - 1) * NF + ST_INFO] = j + 1;
                    return S->perm[S->super_ptr[s - 1] + j - 1];
                }
                double djj = std::sqrt(std::max(ajj, eps));
                F(j, j) = djj;
                for (i64 i = j + 1; i < w; ++i) F(i, j) /= djj;
                for (i64 k = j + 1; k < j1; ++k) {
                    double l = F(k, j);
                    for (i64 i = k; i < w; ++i) F(i, k) -= F(i, j) * l;
                }
            }
            const double rest = (double)(w - j1);
            parallel_for(j1, w, 0.5 * rest * rest * (double)(j1 - j0), [&](i64 k) {
                for (i64 j = j0; j < j1; ++j) {
                    double l = F(k, j);
                    for (i64 i = k; i < w; ++i) F(i, k) -= F(i, j) * l;
                }
            });
        }
        if (m > 0) {
            // trsm R,L,T: F21 <- F21 L11^-T, row by row (each entry takes the updates of columns j < k, in
            // order, then its division, as in the column-by-column form)
            parallel_for(w, f, 0.5 * (double)m * w * w, [&](i64 i) {
                for (i64 j = 0; j < w; ++j) {
                    F(i, j) /= F(j, j);
                    const double x = F(i, j);
                    for (i64 k = j + 1; k < w; ++k) F(i, k) -= x * F(k, j);
                }
            });
            // syrk: F22 -= F21 F21^T (lower), column by column (each entry takes k = 0..w-1 in order)
            parallel_for(w, f, 0.5 * (double)m * m * w, [&](i64 jj) {
                for (i64 k = 0; k < w; ++k) {
                    double l = F(jj, k);
                    for (i64 ii = jj; ii < f; ++ii) F(ii, jj) -= F(ii, k) * l;
                }
            });
            if (S->snparent[s - 1] != 0) {
                cbs[s].assign(m * m, 0.0);
                for (i64 jj = 0; jj < m; ++jj)
                    for (i64 ii = jj; ii < m; ++ii) cbs[s][ii + jj * m] = F(w + ii, w + jj);
                cbm[s] = m;
            }
        }
        for (i64 j = 0; j < w; ++j)
            for (i64 i = j; i < f; ++i) factor[base - 1 + j * f + i] = F(i, j);
        stats[(s - 1) * NF + ST_NPOS] = w;
        return 0;
    });
}

// ---------------------------------------------------------------------------
// LDL^T (ldlt.jl:121-454), real symmetric (herm = true)
struct LdltParams {
    int pivot;  // PIV_NONE, PIV_DIAGONAL or PIV_BK
    double u, eps;
};

// all index arguments 0-based; "k" is the first remaining row/column
double colmax(Front& F, i64 c, i64 k, i64 skip) {
    double m = 0.0;
    for (i64 i = k; i < F.f; ++i) {
        if (i == c || i == skip) continue;
        m = std::max(m, std::fabs(F(i, c)));
    }
    return m;
}

bool threshold_ok(Front& F, i64 c, i64 k, double u, double d) {
    double m = 0.0;
    for (i64 i = k; i < F.f; ++i) {
        if (i == c) continue;
        m = std::max(m, std::fabs(F(i, c)));
        if (!(d >= u * m)) return false;
    }
    return d >= u * m;
}

bool accept_1x1(Front& F, i64 c, i64 k, const LdltParams& p) {
    double d = std::fabs(F(c, c));
    return d >= p.eps && threshold_ok(F, c, k, p.u, d);
}

bool nonsingular_2x2(Front& F, i64 k, i64 r, const LdltParams& p) {
    double det = F(k, k) * F(r, r) - F(k, r) * F(r, k);
    return det != 0.0 && std::isfinite(det) &&
           std::max(std::max(std::fabs(F(k, k)), std::fabs(F(r, k))), std::fabs(F(r, r))) >= p.eps;
}

bool accept_2x2(Front& F, i64 k, i64 r, const LdltParams& p) {
    if (!nonsingular_2x2(F, k, r, p)) return false;
    double det = F(k, k) * F(r, r) - F(k, r) * F(r, k);
    double e11 = std::fabs(F(r, r) / det), e12 = std::fabs(F(k, r) / det), e21 = std::fabs(F(r, k) / det),
           e22 = std::fabs(F(k, k) / det);
    double m1 = colmax(F, k, k, r), m2 = colmax(F, r, k, k);
    return p.u * (e11 * m1 + e21 * m2) <= 1 && p.u * (e12 * m1 + e22 * m2) <= 1;
}

i64 best_1x1(Front& F, i64 k, i64 w, const LdltParams& p) {  // -1 if none
    i64 best = -1;
    double bv = 0.0;
    for (i64 j = k; j < w; ++j) {
        double a = std::fabs(F(j, j));
        if (!(a >= p.eps)) continue;
        if (best >= 0 && !(a > bv)) continue;
        if (!threshold_ok(F, j, k, p.u, a)) continue;
        best = j;
        bv = a;
    }
    return best;
}

// returns (c, r): r < 0 for a 1x1 pivot at c, else the 2x2 on (k, r)
void choose_pivot(Front& F, i64 k, i64 w, const LdltParams& p, i64& c_out, i64& r_out) {
    r_out = -1;
    if (p.pivot == PIV_NONE) { c_out = k; return; }
    if (p.pivot == PIV_DIAGONAL) {
        if (accept_1x1(F, k, k, p)) { c_out = k; return; }
        i64 best = best_1x1(F, k, w, p);
        if (best >= 0) { c_out = best; return; }
        i64 big = k;
        for (i64 j = k + 1; j < w; ++j)
            if (std::fabs(F(j, j)) > std::fabs(F(big, big))) big = j;
        c_out = std::fabs(F(big, big)) >= p.eps ? big : k;
        return;
    }
    const double alpha = (1.0 + std::sqrt(17.0)) / 8.0;
    double lambda = 0.0;
    i64 r = -1;
    for (i64 i = k + 1; i < w; ++i) {
        double a = std::fabs(F(i, k));
        if (a > lambda) { lambda = a; r = i; }
    }
    double akk = std::fabs(F(k, k));
    i64 bc = k, br = -1;
    if (r < 0 || akk >= alpha * lambda) {
        bc = k;
    } else {
        double sigma = 0.0;
        for (i64 i = k; i < w; ++i)
            if (i != r) sigma = std::max(sigma, std::fabs(F(i, r)));
        if (akk * sigma >= alpha * lambda * lambda) bc = k;
        else if (std::fabs(F(r, r)) >= alpha * sigma) bc = r;
        else { bc = k; br = r; }
    }
    bool acc = br < 0 ? accept_1x1(F, bc, k, p) : accept_2x2(F, k, br, p);
    if (acc) { c_out = bc; r_out = br; return; }
    i64 best = best_1x1(F, k, w, p);
    if (best >= 0) { c_out = best; return; }
    if (br >= 0 && nonsingular_2x2(F, k, br, p)) { c_out = bc; r_out = br; return; }
    c_out = bc;
}

void swap_front(Front& F, i64 p, i64 q, i64 w, vector<i64>& lp) {
    if (p == q) return;
    for (i64 i = 0; i < F.f; ++i) std::swap(F(i, p), F(i, q));
    for (i64 j = 0; j < w; ++j) std::swap(F(p, j), F(q, j));
    std::swap(lp[p], lp[q]);
}

i64 factor_ldlt(const Ctx& C, const double* nz, const LdltParams& prm, const int8_t* psign, double* factor,
                double* d, int32_t* piv, int8_t* kind, int64_t* stats) {
    const oracle_symbolic* S = C.S;
    i64 n = S->n;
    vector<vector<double>> cbs(C.ns + 1);
    vector<i64> cbm(C.ns + 1, -1);
    return run_fronts(C, [&](i64 s) -> i64 {
        i64 f = C.f(s), w = C.w(s), m = f - w, base = C.base(s);
        i64 c0 = S->super_ptr[s - 1];
        Front F{f, w, vector<double>(f * f, 0.0)};
        assemble(C, s, nz, F, cbs, cbm, false);
        if (s == S->schur) {
            store_schur(C, s, F, false, factor, nullptr, d, piv, kind);
            return 0;
        }
        for (i64 j = 0; j < w; ++j)
            for (i64 i = j + 1; i < w; ++i) F(j, i) = F(i, j);
        vector<i64> lp(w);
        for (i64 k = 0; k < w; ++k) lp[k] = k;  // 0-based local columns
        vector<int8_t> kd(w, 0);
        vector<double> dd(w, 0.0), ee(w, 0.0);
        i64 st[NF] = {0, 0, 0, 0, 0, 0};
        i64 k = 0;
        while (k < w) {
            i64 c, r;
            choose_pivot(F, k, w, prm, c, r);
            if (r < 0) {
                swap_front(F, k, c, w, lp);
                double dk = F(k, k);
                kd[k] = KIND_1X1;
                if (!(std::fabs(dk) >= prm.eps) || dk == 0.0) {
                    if (dk == 0.0) st[ST_NZERO]++;
                    int req = psign ? (int)psign[S->perm[c0 + lp[k] - 1] - 1] : 0;
                    double sg = req != 0 ? (double)req : (dk < 0 ? -1.0 : 1.0);
                    dk = sg * prm.eps;
                    kd[k] = KIND_PERTURBED;
                    st[ST_NPERT]++;
                    if (dk == 0.0 && st[ST_INFO] == 0) st[ST_INFO] = lp[k] + 1;
                }
                F(k, k) = dk;
                dd[k] = dk;
                if (dk > 0) st[ST_NPOS]++;
                else if (dk < 0) st[ST_NNEG]++;
                for (i64 i = k + 1; i < f; ++i) {
                    double l = F(i, k) / dk;
                    for (i64 j = k + 1; j < w; ++j) F(i, j) -= l * F(k, j);
                    F(i, k) = l;
                }
                k += 1;
            } else {
                swap_front(F, k + 1, r, w, lp);
                double a = F(k, k), b = F(k + 1, k), c2 = F(k + 1, k + 1);
                double up = b;
                F(k, k) = a; F(k + 1, k + 1) = c2; F(k, k + 1) = up;
                double det = a * c2 - up * b;
                double e11 = c2 / det, e12 = -up / det, e21 = -b / det, e22 = a / det;
                kd[k] = KIND_2X2_FIRST;
                kd[k + 1] = KIND_2X2_SECOND;
                dd[k] = a; dd[k + 1] = c2; ee[k] = b;
                st[ST_N2X2]++;
                if (det < 0) { st[ST_NPOS]++; st[ST_NNEG]++; }
                else if (a > 0) st[ST_NPOS] += 2;
                else st[ST_NNEG] += 2;
                for (i64 i = k + 2; i < f; ++i) {
                    double x1 = F(i, k), x2 = F(i, k + 1);
                    double l1 = x1 * e11 + x2 * e21;
                    double l2 = x1 * e12 + x2 * e22;
                    for (i64 j = k + 2; j < w; ++j) F(i, j) -= l1 * F(k, j) + l2 * F(k + 1, j);
                    F(i, k) = l1; F(i, k + 1) = l2;
                }
                F(k + 1, k) = 0.0;
                k += 2;
            }
        }
        for (i64 q = 0; q < w; ++q) {
            i64 g = c0 + q;  // 1-based factor column
            piv[g - 1] = (int32_t)(c0 + lp[q]);
            kind[g - 1] = kd[q];
            d[g - 1] = dd[q];
            d[n + g - 1] = ee[q];
        }
        for (int q = 0; q < NF; ++q) stats[(s - 1) * NF + q] = st[q];
        if (m > 0) {
            // W = L21 D, then F22 -= W L21^T (ldlt.jl:184-191)
            vector<double> W(m * w);
            i64 q = 0;
            while (q < w) {
                if (kd[q] == KIND_2X2_FIRST) {
                    double a = dd[q], b = ee[q], c = dd[q + 1];
                    for (i64 i = 0; i < m; ++i) {
                        double x1 = F(w + i, q), x2 = F(w + i, q + 1);
                        W[i + q * m] = x1 * a + x2 * b;
                        W[i + (q + 1) * m] = x1 * b + x2 * c;
                    }
                    q += 2;
                } else {
                    for (i64 i = 0; i < m; ++i) W[i + q * m] = F(w + i, q) * dd[q];
                    q += 1;
                }
            }
            for (i64 jj = 0; jj < m; ++jj)
                for (i64 kk = 0; kk < w; ++kk) {
                    double l = F(w + jj, kk);
                    for (i64 ii = 0; ii < m; ++ii) F(w + ii, w + jj) -= W[ii + kk * m] * l;
                }
            if (S->snparent[s - 1] != 0) {
                cbs[s].assign(m * m, 0.0);
                for (i64 jj = 0; jj < m; ++jj)
                    for (i64 ii = jj; ii < m; ++ii) cbs[s][ii + jj * m] = F(w + ii, w + jj);
                cbm[s] = m;
            }
        }
        for (i64 j = 0; j < w; ++j) {
            factor[base - 1 + j * f + j] = 1.0;
            for (i64 i = j + 1; i < f; ++i) factor[base - 1 + j * f + i] = F(i, j);
        }
        return 0;
    });
}

// ---------------------------------------------------------------------------
// LU (lu.jl:84-231)
i64 lu_choose_row(Front& F, i64 k, i64 w, double u) {
    double g = 0.0;
    for (i64 i = k; i < F.f; ++i) g = std::max(g, std::fabs(F(i, k)));
    double akk = std::fabs(F(k, k));
    if (akk >= u * g) return k;
    i64 r = k;
    double best = akk;
    for (i64 i = k + 1; i < w; ++i) {
        double a = std::fabs(F(i, k));
        if (a > best) { r = i; best = a; }
    }
    return r;
}

i64 factor_lu(const Ctx& C, const double* nz, bool pivot, double u, double eps, double* factor, double* ufactor,
              double* d, int32_t* piv, int8_t* kind, int64_t* stats) {
    const oracle_symbolic* S = C.S;
    vector<vector<double>> cbs(C.ns + 1);
    vector<i64> cbm(C.ns + 1, -1);
    return run_fronts(C, [&](i64 s) -> i64 {
        i64 f = C.f(s), w = C.w(s), m = f - w, base = C.base(s);
        i64 c0 = S->super_ptr[s - 1];
        Front F{f, w, vector<double>(f * f, 0.0)};
        assemble(C, s, nz, F, cbs, cbm, true);
        if (s == S->schur) {
            store_schur(C, s, F, true, factor, ufactor, d, piv, kind);
            return 0;
        }
        vector<i64> lp(w);
        for (i64 k = 0; k < w; ++k) lp[k] = k;
        vector<int8_t> kd(w, KIND_1X1);
        vector<double> dd(w, 0.0);
        i64 st[NF] = {0, 0, 0, 0, 0, 0};
        for (i64 k = 0; k < w; ++k) {
            i64 r = pivot ? lu_choose_row(F, k, w, u) : k;
            if (r != k) {
                for (i64 j = 0; j < f; ++j) std::swap(F(k, j), F(r, j));
                std::swap(lp[k], lp[r]);
            }
            double dk = F(k, k);
            if (!(std::fabs(dk) >= eps) || dk == 0.0) {
                if (dk == 0.0) st[ST_NZERO]++;
                dk = (dk < 0 ? -1.0 : 1.0) * eps;
                kd[k] = KIND_PERTURBED;
                st[ST_NPERT]++;
                if (dk == 0.0 && st[ST_INFO] == 0) st[ST_INFO] = k + 1;
            }
            F(k, k) = dk;
            dd[k] = dk;
            for (i64 j = k + 1; j < w; ++j)
                for (i64 i = k + 1; i < f; ++i) F(i, j) -= F(i, k) / dk * F(k, j);
            for (i64 j = w; j < f; ++j)
                for (i64 i = k + 1; i < w; ++i) F(i, j) -= F(i, k) / dk * F(k, j);
            for (i64 i = k + 1; i < f; ++i) F(i, k) /= dk;
            for (i64 j = k + 1; j < f; ++j) F(k, j) /= dk;
        }
        for (i64 q = 0; q < w; ++q) {
            i64 g = c0 + q;
            piv[g - 1] = (int32_t)(c0 + lp[q]);
            kind[g - 1] = kd[q];
            d[g - 1] = dd[q];
        }
        for (int q = 0; q < NF; ++q) stats[(s - 1) * NF + q] = st[q];
        if (m > 0) {
            for (i64 jj = 0; jj < m; ++jj)
                for (i64 ii = 0; ii < m; ++ii) {
                    double acc = 0.0;
                    for (i64 k = 0; k < w; ++k) acc += F(w + ii, k) * dd[k] * F(k, w + jj);
                    F(w + ii, w + jj) -= acc;
                }
            if (S->snparent[s - 1] != 0) {
                cbs[s].assign(m * m, 0.0);
                for (i64 jj = 0; jj < m; ++jj)
                    for (i64 ii = 0; ii < m; ++ii) cbs[s][ii + jj * m] = F(w + ii, w + jj);
                cbm[s] = m;
            }
        }
        for (i64 j = 0; j < w; ++j) {
            factor[base - 1 + j * f + j] = 1.0;
            ufactor[base - 1 + j * f + j] = 1.0;
            for (i64 i = j + 1; i < f; ++i) {
                factor[base - 1 + j * f + i] = F(i, j);
                ufactor[base - 1 + j * f + i] = F(j, i);
            }
        }
        return 0;
    });
}

i64 host_info(const Ctx& C, const int64_t* stats) {  // ldlt.jl:206-214
    i64 best = 0;
    for (i64 s = 1; s <= C.ns; ++s) {
        i64 fi = stats[(s - 1) * NF + ST_INFO];
        if (fi > 0) {
            i64 col = C.S->super_ptr[s - 1] + fi - 1;
            best = best == 0 ? col : std::min(best, col);
        }
    }
    return best == 0 ? 0 : C.S->perm[best - 1];
}

// ---------------------------------------------------------------------------
// Solves. Panels of front s: P(i, j) = panel[base + j f + i], rows = rowval[rowptr[s]..].
struct Panel {
    const double* p;
    i64 f, w;
    double operator()(i64 i, i64 j) const { return p[i + j * f]; }
};

// forward with unit (unit=true) or non-unit lower panels; reorder: apply the local pivot order
void forward(const Ctx& C, const double* fac, const int32_t* piv, bool unit, bool reorder, double* Y, i64 n,
             i64 nrhs) {
    const oracle_symbolic* S = C.S;
    vector<double> blk, t;
    for (i64 q = 0; q < C.ns; ++q) {
        i64 s = S->snpost[q];
        i64 f = C.f(s), w = C.w(s), c0 = S->super_ptr[s - 1];
        Panel P{fac + C.base(s) - 1, f, w};
        const i64* rows = S->rowval + S->rowptr[s - 1] - 1;
        for (i64 r = 0; r < nrhs; ++r) {
            double* y = Y + r * n;
            if (reorder) {
                blk.assign(w, 0.0);
                for (i64 k = 0; k < w; ++k) blk[k] = y[piv[c0 + k - 1] - 1];
                for (i64 k = 0; k < w; ++k) y[c0 + k - 1] = blk[k];
            }
            double* yc = y + c0 - 1;
            for (i64 j = 0; j < w; ++j) {
                if (!unit) yc[j] /= P(j, j);
                for (i64 i = j + 1; i < w; ++i) yc[i] -= P(i, j) * yc[j];
            }
            for (i64 i = w; i < f; ++i) {
                double acc = 0.0;
                for (i64 j = 0; j < w; ++j) acc += P(i, j) * yc[j];
                y[rows[i] - 1] -= acc;
            }
        }
    }
}

void backward(const Ctx& C, const double* fac, const int32_t* piv, bool unit, bool reorder, double* Y, i64 n,
              i64 nrhs) {
    const oracle_symbolic* S = C.S;
    vector<double> blk;
    for (i64 q = C.ns - 1; q >= 0; --q) {
        i64 s = S->snpost[q];
        i64 f = C.f(s), w = C.w(s), c0 = S->super_ptr[s - 1];
        Panel P{fac + C.base(s) - 1, f, w};
        const i64* rows = S->rowval + S->rowptr[s - 1] - 1;
        for (i64 r = 0; r < nrhs; ++r) {
            double* y = Y + r * n;
            double* yc = y + c0 - 1;
            for (i64 j = 0; j < w; ++j) {
                double acc = 0.0;
                for (i64 i = w; i < f; ++i) acc += P(i, j) * y[rows[i] - 1];
                yc[j] -= acc;
            }
            for (i64 j = w - 1; j >= 0; --j) {
                double acc = yc[j];
                for (i64 i = j + 1; i < w; ++i) acc -= P(i, j) * yc[i];
                yc[j] = unit ? acc : acc / P(j, j);
            }
            if (reorder) {
                blk.assign(yc, yc + w);
                for (i64 k = 0; k < w; ++k) y[piv[c0 + k - 1] - 1] = blk[k];
            }
        }
    }
}

void diagonal(const oracle_symbolic* S, const double* d, const int8_t* kind, bool twobytwo, double* Y, i64 nrhs) {
    i64 n = S->n;
    for (i64 r = 0; r < nrhs; ++r) {
        double* y = Y + r * n;
        i64 k = 0;
        while (k < n) {
            if (twobytwo && kind[k] == KIND_2X2_FIRST) {
                double a = d[k], b = d[n + k], c = d[k + 1];
                double det = a * c - b * b;
                double y1 = y[k], y2 = y[k + 1];
                y[k] = (c * y1 - b * y2) / det;
                y[k + 1] = (a * y2 - b * y1) / det;
                k += 2;
            } else {
                y[k] /= d[k];
                k += 1;
            }
        }
    }
}

}  // namespace

extern "C" {

int64_t oracle_factor(const oracle_symbolic* S, const double* nzval, int structure, int pivot_type, double u,
                      double eps, int eps_scaled, const int8_t* psign, double* factor, double* ufactor, double* d,
                      int32_t* piv, int8_t* kind, int64_t* stats) {
    Ctx C{S, S->ns};
    i64 flen = S->ns > 0 ? S->front_ptr[S->ns] - 1 : 0;
    std::fill(factor, factor + flen, 0.0);
    std::fill(stats, stats + NF * S->ns, (int64_t)0);
    if (structure == 3) return factor_cholesky(C, nzval, eps, factor, stats);
    if (eps_scaled) {
        double amax = 0.0;
        for (i64 p = 0; p < S->nnz; ++p) amax = std::max(amax, std::fabs(nzval[p]));
        if (amax > 0) eps *= amax;
    }
    std::fill(d, d + 2 * S->n, 0.0);
    std::fill(piv, piv + S->n, 0);
    std::fill(kind, kind + S->n, (int8_t)0);
    if (structure == 1) {
        LdltParams prm;
        if (pivot_type == PIV_NONE) prm.pivot = PIV_NONE;
        else if (pivot_type == PIV_DIAGONAL) prm.pivot = PIV_DIAGONAL;
        else if (pivot_type == PIV_AUTO || pivot_type == PIV_BK || pivot_type == PIV_LOCAL) prm.pivot = PIV_BK;
        else return -1;
        prm.u = u;
        prm.eps = eps;
        factor_ldlt(C, nzval, prm, psign, factor, d, piv, kind, stats);
        return host_info(C, stats);
    }
    if (structure == 0) {
        bool pv;
        if (pivot_type == PIV_NONE || pivot_type == PIV_DIAGONAL) pv = false;
        else if (pivot_type == PIV_AUTO || pivot_type == PIV_BK || pivot_type == PIV_LOCAL) pv = true;
        else return -1;
        std::fill(ufactor, ufactor + flen, 0.0);
        factor_lu(C, nzval, pv, u, eps, factor, ufactor, d, piv, kind, stats);
        return host_info(C, stats);
    }
    return -1;
}

// Host threads for the factorizations (1, the default: the reference's serial postorder).
void oracle_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

int oracle_solve(const oracle_symbolic* S, int structure, const double* factor, const double* ufactor,
                 const double* d, const int32_t* piv, const int8_t* kind, double* X, const double* B, int64_t nrhs,
                 int transpose) {
    Ctx C{S, S->ns};
    i64 n = S->n;
    vector<double> Y(n * nrhs);
    for (i64 r = 0; r < nrhs; ++r)
        for (i64 k = 0; k < n; ++k) Y[k + r * n] = B[S->perm[k] - 1 + r * n];
    if (structure == 3) {
        forward(C, factor, nullptr, false, false, Y.data(), n, nrhs);
        backward(C, factor, nullptr, false, false, Y.data(), n, nrhs);
    } else if (structure == 1) {
        forward(C, factor, piv, true, true, Y.data(), n, nrhs);
        diagonal(S, d, kind, true, Y.data(), nrhs);
        backward(C, factor, piv, true, true, Y.data(), n, nrhs);
    } else if (structure == 0) {
        if (!transpose) {
            forward(C, factor, piv, true, true, Y.data(), n, nrhs);
            diagonal(S, d, kind, false, Y.data(), nrhs);
            backward(C, ufactor, piv, true, false, Y.data(), n, nrhs);
        } else {
            forward(C, ufactor, piv, true, false, Y.data(), n, nrhs);
            diagonal(S, d, kind, false, Y.data(), nrhs);
            backward(C, factor, piv, true, true, Y.data(), n, nrhs);
        }
    } else {
        return -1;
    }
    for (i64 r = 0; r < nrhs; ++r)
        for (i64 k = 0; k < n; ++k) X[S->perm[k] - 1 + r * n] = Y[k + r * n];
    return 0;
}

}  // extern "C"

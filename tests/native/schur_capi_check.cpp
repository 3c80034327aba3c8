// Schur complement mode and the solve sub-phases through the C ABI alone (no Python, no torch):
// for each case of the input file (written by tests/test_schur_capi_gpu.py with dense expectations),
// the Schur analysis (sdsa_analyze with user_schur_indices), sdsb200_factor, sdsb200_schur_matrix
// against the dense Schur complement, "solve_fwd_schur" / "solve_diag" / "solve_bwd_schur" as
// sdsb200_solve_phase sequences around a host solve of the condensed system, and on a plain plan the
// five sub-phases against sdsb200_solve (bit for bit with the per-level engine). Exit status 0 = pass.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "sdsb200.h"
#include "sdsb200_analysis.h"

using std::vector;
static int fails = 0;
#define CHECK(cond, ...)                      \
    do {                                      \
        if (!(cond)) {                        \
            printf("FAIL: " __VA_ARGS__);     \
            printf("\n");                     \
            ++fails;                          \
        }                                     \
    } while (0)
#define CU(x)                                                                        \
    do {                                                                             \
        cudaError_t e_ = (x);                                                        \
        if (e_ != cudaSuccess) { printf("cuda %s: %s\n", #x, cudaGetErrorString(e_)); return 2; } \
    } while (0)
#define API(x)                                                                    \
    do {                                                                          \
        int r_ = (x);                                                             \
        if (r_ != 0) { printf("api %s: %d %s\n", #x, r_, sdsb200_last_error()); return 3; } \
    } while (0)

template <class T>
static vector<T> rd(FILE* f, size_t n) {
    vector<T> v(n);
    if (n && fread(v.data(), sizeof(T), n, f) != n) { printf("short read\n"); exit(4); }
    return v;
}

struct Sym {
    vector<vector<int64_t>> keep;
    sdsb200_symbolic s{};
    int64_t schur = 0;
};

static int analyze(int64_t n, const vector<int64_t>& rp, const vector<int64_t>& cv, const vector<double>& nz,
                   int structure, const int8_t* flags, Sym& out) {
    sdsa_options o;
    sdsa_default_options(&o, structure);
    o.index_base = 0;
    o.user_schur_indices = flags;
    sdsa_result* R = nullptr;
    if (sdsa_analyze(n, rp.data(), cv.data(), nz.data(), &o, &R) != 0) {
        printf("analysis: %s\n", sdsa_last_error());
        return 5;
    }
    const char* names[] = {"perm", "super_ptr", "snparent", "rowptr", "rowval", "front_ptr", "child_ptr",
                           "child_list", "relind_ptr", "relind", "amap", "amap_ptr", "amap_src"};
    const void** dst[] = {&out.s.perm, &out.s.super_ptr, &out.s.snparent, &out.s.rowptr, &out.s.rowval,
                          &out.s.front_ptr, &out.s.child_ptr, &out.s.child_list, &out.s.relind_ptr, &out.s.relind,
                          &out.s.amap, &out.s.amap_ptr, &out.s.amap_src};
    out.keep.resize(13);
    for (int k = 0; k < 13; ++k) {
        int64_t len = sdsa_len(R, names[k]);
        out.keep[k].assign(len > 0 ? len : 1, 0);
        if (len > 0) sdsa_get(R, names[k], out.keep[k].data());
        *dst[k] = out.keep[k].data();
    }
    out.s.n = n;
    out.s.nnz = (int64_t)cv.size();
    out.s.ns = (int64_t)sdsa_stat(R, "ns");
    out.s.index_width = 8;
    out.s.structure = structure;
    out.s.schur = (int64_t)sdsa_stat(R, "schur");
    sdsa_free(R);
    return 0;
}

// dense solve with partial pivoting (column-major, n small)
static vector<double> dense_solve(vector<double> A, vector<double> b, int n) {
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (fabs(A[i + k * n]) > fabs(A[p + k * n])) p = i;
        for (int j = 0; j < n; ++j) std::swap(A[k + j * n], A[p + j * n]);
        std::swap(b[k], b[p]);
        for (int i = k + 1; i < n; ++i) {
            double l = A[i + k * n] / A[k + k * n];
            for (int j = k; j < n; ++j) A[i + j * n] -= l * A[k + j * n];
            b[i] -= l * b[k];
        }
    }
    for (int k = n - 1; k >= 0; --k) {
        double s = b[k];
        for (int j = k + 1; j < n; ++j) s -= A[k + j * n] * b[j];
        b[k] = s / A[k + k * n];
    }
    return b;
}

static double maxabs(const vector<double>& v) {
    double m = 0;
    for (double x : v) m = std::max(m, fabs(x));
    return m;
}

int main(int argc, char** argv) {
    FILE* f = fopen(argc > 1 ? argv[1] : "schur_cases.bin", "rb");
    if (!f) { printf("no input\n"); return 4; }
    int64_t ncase = rd<int64_t>(f, 1)[0];
    CU(cudaSetDevice(0));
    for (int64_t c = 0; c < ncase; ++c) {
        vector<int64_t> hdr = rd<int64_t>(f, 5);
        double u = rd<double>(f, 1)[0];
        const int64_t n = hdr[0], nnz = hdr[1], k = hdr[2], tr = hdr[4];
        const int structure = (int)hdr[3];
        vector<int64_t> rp = rd<int64_t>(f, n + 1), cv = rd<int64_t>(f, nnz);
        vector<double> nz = rd<double>(f, nnz);
        vector<int8_t> fl = rd<int8_t>(f, n);
        vector<double> Sd = rd<double>(f, k * k), b = rd<double>(f, n), bs = rd<double>(f, k), xe = rd<double>(f, n);
        printf("case %lld: structure %d n %lld ns %lld transpose %lld\n", (long long)c, structure, (long long)n,
               (long long)k, (long long)tr);
        double *d_nz, *d_b, *d_z, *d_x, *d_S;
        CU(cudaMalloc(&d_nz, sizeof(double) * nnz));
        CU(cudaMalloc(&d_b, sizeof(double) * n));
        CU(cudaMalloc(&d_z, sizeof(double) * n));
        CU(cudaMalloc(&d_x, sizeof(double) * n));
        CU(cudaMalloc(&d_S, sizeof(double) * k * k));
        CU(cudaMemcpy(d_nz, nz.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(d_b, b.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        sdsb200_opts o;
        sdsb200_default_opts(&o);
        o.pivot_threshold = u;
        o.solve_mode = (int32_t)tr;
        sdsb200_plan_options po{1, SDSB200_PRECISION_FP64, 1, 0};
        // Schur complement mode
        {
            Sym S;
            if (analyze(n, rp, cv, nz, structure, fl.data(), S)) return 5;
            CHECK(S.s.schur == S.s.ns, "schur root %lld of %lld", (long long)S.s.schur, (long long)S.s.ns);
            sdsb200_plan* P = nullptr;
            API(sdsb200_plan_create(&P, &S.s, &po, nullptr));
            int64_t info = -1;
            API(sdsb200_factor(P, d_nz, nullptr, &o, &info, nullptr));
            CHECK(info == 0, "info %lld", (long long)info);
            CHECK((int64_t)sdsb200_plan_stat(P, "schur_n") == k, "schur_n");
            int rc = sdsb200_solve(P, d_x, n, d_b, n, 1, nullptr, &o, nullptr, nullptr);
            CHECK(rc == SDSB200_NOT_SUPPORTED, "complete solve in Schur mode gave %d", rc);
            API(sdsb200_schur_matrix(P, 0, d_S, k, (int32_t)tr, nullptr));
            vector<double> Sg(k * k);
            CU(cudaMemcpy(Sg.data(), d_S, sizeof(double) * k * k, cudaMemcpyDeviceToHost));
            double dS = 0;
            for (int64_t q = 0; q < k * k; ++q) dS = std::max(dS, fabs(Sg[q] - Sd[q]));
            printf("  S vs dense: %.3e (rel)\n", dS / maxabs(Sd));
            CHECK(dS <= 1e-11 * maxabs(Sd), "S");
            // solve_fwd_schur
            API(sdsb200_solve_phase(P, SDSB200_PHASE_FWD_PERM, nullptr, n, d_b, n, 1, &o, nullptr));
            API(sdsb200_solve_phase(P, SDSB200_PHASE_FWD, nullptr, n, nullptr, n, 1, &o, nullptr));
            API(sdsb200_solve_phase(P, SDSB200_PHASE_STORE, d_z, n, nullptr, n, 1, &o, nullptr));
            vector<double> z(n);
            CU(cudaMemcpy(z.data(), d_z, sizeof(double) * n, cudaMemcpyDeviceToHost));
            double db = 0;
            for (int64_t q = 0; q < k; ++q) db = std::max(db, fabs(z[n - k + q] - bs[q]));
            printf("  condensed rhs: %.3e (rel)\n", db / maxabs(bs));
            CHECK(db <= 1e-12 * maxabs(bs), "condensed rhs");
            // solve_diag
            API(sdsb200_solve_phase(P, SDSB200_PHASE_LOAD, nullptr, n, d_z, n, 1, &o, nullptr));
            if (structure != SDSB200_STRUCTURE_G)
                API(sdsb200_solve_phase(P, SDSB200_PHASE_DIAG, nullptr, n, nullptr, n, 1, &o, nullptr));
            API(sdsb200_solve_phase(P, SDSB200_PHASE_STORE, d_z, n, nullptr, n, 1, &o, nullptr));
            CU(cudaMemcpy(z.data(), d_z, sizeof(double) * n, cudaMemcpyDeviceToHost));
            // the condensed system on the host (the exported matrix is already S^T for the transposed solve)
            vector<double> rhs(z.end() - k, z.end());
            vector<double> x2 = dense_solve(Sg, rhs, (int)k);
            for (int64_t q = 0; q < k; ++q) z[n - k + q] = x2[q];
            CU(cudaMemcpy(d_z, z.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
            // solve_bwd_schur
            API(sdsb200_solve_phase(P, SDSB200_PHASE_LOAD, nullptr, n, d_z, n, 1, &o, nullptr));
            if (structure == SDSB200_STRUCTURE_G)
                API(sdsb200_solve_phase(P, SDSB200_PHASE_DIAG, nullptr, n, nullptr, n, 1, &o, nullptr));
            API(sdsb200_solve_phase(P, SDSB200_PHASE_BWD, nullptr, n, nullptr, n, 1, &o, nullptr));
            API(sdsb200_solve_phase(P, SDSB200_PHASE_BWD_PERM, d_x, n, nullptr, n, 1, &o, nullptr));
            vector<double> x(n);
            CU(cudaMemcpy(x.data(), d_x, sizeof(double) * n, cudaMemcpyDeviceToHost));
            double dx = 0;
            for (int64_t q = 0; q < n; ++q) dx = std::max(dx, fabs(x[q] - xe[q]));
            printf("  Schur route x vs dense: %.3e (rel)\n", dx / maxabs(xe));
            CHECK(dx <= 1e-10 * maxabs(xe), "Schur route x");
            API(sdsb200_plan_destroy(P));
        }
        // the sub-phases of a plain plan against the complete solve
        {
            Sym S;
            if (analyze(n, rp, cv, nz, structure, nullptr, S)) return 5;
            sdsb200_plan* P = nullptr;
            API(sdsb200_plan_create(&P, &S.s, &po, nullptr));
            int64_t info = -1;
            API(sdsb200_factor(P, d_nz, nullptr, &o, &info, nullptr));
            int rc = sdsb200_solve_phase(P, SDSB200_PHASE_STORE, nullptr, n, nullptr, n, 1, &o, nullptr);
            CHECK(rc == SDSB200_INVALID_VALUE, "store without X gave %d", rc);
            vector<double> x1(n), x0(n), xp(n);
            API(sdsb200_solve(P, d_x, n, d_b, n, 1, nullptr, &o, nullptr, nullptr));
            CU(cudaMemcpy(x1.data(), d_x, sizeof(double) * n, cudaMemcpyDeviceToHost));
            API(sdsb200_set_persistent(P, 0));
            API(sdsb200_solve(P, d_x, n, d_b, n, 1, nullptr, &o, nullptr, nullptr));
            CU(cudaMemcpy(x0.data(), d_x, sizeof(double) * n, cudaMemcpyDeviceToHost));
            API(sdsb200_solve_phase(P, SDSB200_PHASE_FWD_PERM, nullptr, n, d_b, n, 1, &o, nullptr));
            API(sdsb200_solve_phase(P, SDSB200_PHASE_FWD, nullptr, n, nullptr, n, 1, &o, nullptr));
            API(sdsb200_solve_phase(P, SDSB200_PHASE_DIAG, nullptr, n, nullptr, n, 1, &o, nullptr));
            API(sdsb200_solve_phase(P, SDSB200_PHASE_BWD, nullptr, n, nullptr, n, 1, &o, nullptr));
            API(sdsb200_solve_phase(P, SDSB200_PHASE_BWD_PERM, d_z, n, nullptr, n, 1, &o, nullptr));
            CU(cudaMemcpy(xp.data(), d_z, sizeof(double) * n, cudaMemcpyDeviceToHost));
            CU(cudaDeviceSynchronize());
            CHECK(memcmp(xp.data(), x0.data(), sizeof(double) * n) == 0, "sub-phases differ from the level solve");
            double d1 = 0, de = 0;
            for (int64_t q = 0; q < n; ++q) {
                d1 = std::max(d1, fabs(xp[q] - x1[q]));
                de = std::max(de, fabs(xp[q] - xe[q]));
            }
            printf("  sub-phases vs persistent: %.3e, vs dense: %.3e (rel)\n", d1 / maxabs(x1), de / maxabs(xe));
            CHECK(d1 <= 1e-10 * maxabs(x1) && de <= 1e-10 * maxabs(xe), "sub-phases");
            API(sdsb200_plan_destroy(P));
        }
        cudaFree(d_nz); cudaFree(d_b); cudaFree(d_z); cudaFree(d_x); cudaFree(d_S);
    }
    printf("%s (%d failures)\n", fails ? "FAILED" : "ALL OK", fails);
    return fails ? 1 : 0;
}

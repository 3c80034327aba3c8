/*
 * oracle.h -- CPU oracle of the numeric phase. TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of the reference's CPU reference factorizations and
 * solves (SparseDirectSolver.jl, src/reference/cholesky.jl, ldlt.jl, lu.jl).
 * Only the tests, the smoke check and the benchmark's CPU-baseline leg load it,
 * as the checker; the product never links or calls it.
 *
 * Parity pins: the reference ships no golden vectors for this path (its tests
 * compare the device factor against these same CPU oracles and check
 * invariants), and Julia is absent here, so the reference cannot be run. This
 * oracle is pinned by the reference's own invariants (scaled backward error,
 * A[p,p] = L D L^T, eigenvalue inertia, residuals) on the reference's test
 * generators, checked in tests/test_oracle.py against numpy/scipy, and by the
 * hand-computed dense fixtures in tests/golden/.
 *
 * The Symbolic maps are the reference's (1-based, as `Symbolic` holds them).
 */
#ifndef SDS_ORACLE_H
#define SDS_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_symbolic {
    int64_t n, ns, nnz;
    const int64_t* perm;       /* n */
    const int64_t* super_ptr;  /* ns + 1 */
    const int64_t* snparent;   /* ns */
    const int64_t* snpost;     /* ns */
    const int64_t* rowptr;     /* ns + 1 */
    const int64_t* rowval;
    const int64_t* front_ptr;  /* ns + 1 (panel_ptr) */
    const int64_t* child_ptr;  /* ns + 1 */
    const int64_t* child_list;
    const int64_t* relind_ptr; /* ns + 1 */
    const int64_t* relind;
    const int64_t* amap;       /* nnz, signed offsets */
    const int64_t* amap_ptr;   /* ns + 1 */
    const int64_t* amap_src;
    int64_t schur;             /* Schur complement mode: the root supernode (1-based) that is assembled and
                                  not factored (src/numeric/schur.jl:15-98); 0 = none */
} oracle_symbolic;

/* structure: 0 "G" (LU), 1 "S" (LDL^T), 3 "SPD" (Cholesky)
 * pivot_type: the reference's PivotType codes: 0 auto, 1 none, 4 diagonal, 5 local block, 6 Bunch-Kaufman
 * u: pivot_threshold; eps: pivot_epsilon (already resolved, >= 0); eps_scaled: pivot_epsilon_alg = "algo1"
 * Outputs (caller-allocated): factor and ufactor (factor_len), d (2n), piv (n), kind (n), stats (6 ns).
 * Cholesky: eps is the cuDSS-style clamp of the device path (0 = the reference's unperturbed
 * ref_factorize!). Returns info (original column of the failed pivot, 0 = success) or -1 on bad input. */
int64_t oracle_factor(const oracle_symbolic* S, const double* nzval, int structure, int pivot_type, double u,
                      double eps, int eps_scaled, const int8_t* psign, double* factor, double* ufactor, double* d,
                      int32_t* piv, int8_t* kind, int64_t* stats);

/* Host threads of oracle_factor: 1 (the default) follows the reference's serial postorder; more run
 * the fronts of one elimination-tree level concurrently, with the same results. */
void oracle_set_threads(int n);

/* X = A^{-1} B (transpose != 0: A^T), B and X n x nrhs column-major (X == B allowed). */
int oracle_solve(const oracle_symbolic* S, int structure, const double* factor, const double* ufactor,
                 const double* d, const int32_t* piv, const int8_t* kind, double* X, const double* B, int64_t nrhs,
                 int transpose);

#ifdef __cplusplus
}
#endif
#endif

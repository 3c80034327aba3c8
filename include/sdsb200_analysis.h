/*
 * sdsb200_analysis.h -- host analysis that produces the Symbolic maps consumed by
 * the numeric phase (libsdsb200.so).
 *
 * The reference keeps its analysis in Julia (the files under src/symbolic/,
 * symbolic_analysis at src/symbolic/maps.jl:255-268); a Julia caller of the
 * numeric phase passes its own `Symbolic` maps and never needs this library.
 * It exists so that C, C++ and Python callers (and the tests and benchmark of
 * this repository) can build the same maps without Julia: every step restates
 * the reference's algorithm (pattern, 2x2 pivot pairs, etree, postorder, column
 * counts, fundamental supernodes, relaxed amalgamation, supernodal row
 * structure, panel layout, assembly map, extend-add maps) except the ordering,
 * whose reference implementation is third-party (AMD.jl / METIS through
 * CliqueTrees.jl) and is replaced by this library's own AMD and nested
 * dissection.
 *
 * All arrays returned by sdsa_get are int64, 1-based where the reference's maps
 * are 1-based (the values are exactly those a Julia `Symbolic` would hold).
 */
#ifndef SDSB200_ANALYSIS_H
#define SDSB200_ANALYSIS_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* structures: same codes as the numeric phase (sdsb200.h) */
#define SDSA_STRUCTURE_G 0
#define SDSA_STRUCTURE_S 1
#define SDSA_STRUCTURE_SPD 3

/* reordering algorithms (cuDSS names: "default", "algo3" AMD, "algo4" ND, "algo5" natural) */
#define SDSA_REORDER_DEFAULT 0 /* AMD and ND evaluated, the lower flops + 1e8 * sdepth wins */
#define SDSA_REORDER_AMD 1
#define SDSA_REORDER_ND 2
#define SDSA_REORDER_NATURAL 3

#define SDSA_PAIRS_NONE 0
#define SDSA_PAIRS_DEFAULT 1
#define SDSA_PAIRS_ALL 2

typedef struct sdsa_options {
    int structure;          /* SDSA_STRUCTURE_* */
    int view;               /* 'L', 'U' or 'F' */
    int index_base;         /* 0 or 1: base of rowptr/colval */
    int reordering;         /* SDSA_REORDER_* (ignored when user_perm != NULL) */
    const int64_t* user_perm; /* length n, 0- or 1-based, or NULL */
    int pivot_pairs;        /* SDSA_PAIRS_* (structure "S" only) */
    double pivot_pair_tolerance; /* 1e-6 */
    double pivot_threshold;      /* 0.01: partner threshold of the pairs */
    int use_superpanels;    /* 1: amalgamation on */
    int amalg_max_width;    /* 32 */
    double amalg_zero_fraction; /* 0.25 */
    int amalg_min_width;    /* 8 */
    const int64_t* user_pairs; /* structure "S": 2 x n_user_pairs 1-based (partner, candidate) pairs the
                                  ordering keeps adjacent instead of searching the values, or NULL */
    int64_t n_user_pairs;
    const int8_t* user_schur_indices; /* Schur complement mode (schur_mode = 1): n flags 0/1, 1 = the row and
                                  column belong to the Schur complement; NULL = off. The flagged indices are
                                  ordered last, in increasing order, as one dense root supernode that the
                                  factorization assembles and does not factor; no 2x2 pivot pairs. */
} sdsa_options;

typedef struct sdsa_result sdsa_result;

/* Fill `o` with the reference defaults (Options() of src/options.jl). */
void sdsa_default_options(sdsa_options* o, int structure);

/* Analyse the n x n CSR pattern (rowptr: n+1, colval: nnz). nzval (length nnz,
 * may be NULL) is read only for the 2x2 pivot pairs of structure "S".
 * Returns 0 or a negative error code; sdsa_last_error() gives the message. */
int sdsa_analyze(int64_t n, const int64_t* rowptr, const int64_t* colval, const double* nzval,
                 const sdsa_options* opts, sdsa_result** out);

/* Array accessors by name: length (or -1 for an unknown name), then copy. Names:
 * perm iperm super_ptr snparent snpost rowptr rowval front_ptr front_nrows front_ncols
 * child_ptr child_list relind_ptr relind amap amap_ptr amap_src counts
 * pairs (2*npairs: partner, candidate)
 * full_rowptr full_colval full_srcptr full_src full_conj  (residual map of the full matrix)
 * schur_rowptr schur_colval  (Schur complement mode: 1-based CSR pattern of S over the Schur indices in
 *                            increasing order, both triangles and the whole diagonal)
 * ordering  (n: the ordering algorithm's permutation before the supernodal renumbering; `perm` is the
 *           factor's, the two composed, src/solver.jl:1082-1085) */
int64_t sdsa_len(const sdsa_result* r, const char* name);
int sdsa_get(const sdsa_result* r, const char* name, int64_t* out);

/* Scalars by name: n nnz ns nnz_stored nnz_L flops factor_len sdepth alg_used
 * (1 amd, 2 nd, 3 natural, 4 user) npairs pair_rounds schur (the Schur root supernode, 1-based; 0 none)
 * schur_n (order of the Schur complement) */
double sdsa_stat(const sdsa_result* r, const char* name);

void sdsa_free(sdsa_result* r);

/* Matching and scaling of the n x n CSR matrix (rowptr, colval, nzval; index_base 0 or 1) from its
 * values: MC64 (Duff & Koster 2001) as the reference's compute_matching runs it at analysis
 * (src/matching/mc64.jl:302-398). `job` is the reference's matching_alg: 1 maximum cardinality,
 * 2 and 3 bottleneck (largest smallest matched |a_ij|), 4 maximum sum, 5 maximum product with the
 * scalings, 6 the automatic choice (= 5).
 * structure SDSA_STRUCTURE_G matches the stored rows; the symmetric structures match the full matrix
 * rebuilt from the triangle `view` selects, and return the symmetric scaling d = sqrt(r c)
 * (rscale = cscale = d, |d_i a_ij d_j| <= 1).
 * Outputs, n entries each: perm (1-based column matched to each row, the reference's
 * "perm_matching"; unmatched rows of a structurally singular matrix take the unmatched columns in
 * increasing order), matched (1 or 0), rscale and cscale ("scale_row", "scale_col"; ones for jobs 1-4).
 * Returns 0, or -1 with the message in sdsa_last_error(). */
int sdsa_matching(int64_t n, const int64_t* rowptr, const int64_t* colval, const double* nzval, int structure,
                  int view, int index_base, int job, int64_t* perm, int8_t* matched, double* rscale,
                  double* cscale);

/* The 2x2 pivot pairs of structure "S" from the cycles of a symmetric matching (the reference's
 * matching_pairs, src/matching/mc64.jl:380-441): perm, matched and d (= rscale) from sdsa_matching of
 * the same matrix. pivot_pairs SDSA_PAIRS_NONE gives none, SDSA_PAIRS_ALL keeps every pair of the
 * cycles, SDSA_PAIRS_DEFAULT only pairs with a 2x2 candidate (scaled |a_ii| <= pivot_pair_tolerance *
 * max_{j != i} scaled |a_ij|). Writes *npairs (partner, candidate) 1-based pairs, sorted by candidate,
 * into pairs (room for n entries: at most n / 2 pairs); pass them as sdsa_options.user_pairs.
 * Returns 0, or -1 with the message in sdsa_last_error(). */
int sdsa_matching_pairs(int64_t n, const int64_t* rowptr, const int64_t* colval, const double* nzval, int view,
                        int index_base, const int64_t* perm, const int8_t* matched, const double* d, int pivot_pairs,
                        double pivot_pair_tolerance, int64_t* pairs, int64_t* npairs);
const char* sdsa_last_error(void);

#ifdef __cplusplus
}
#endif
#endif

# cython: language_level=3, boundscheck=False, wraparound=False, cdivision=True, initializedcheck=False
"""Compiled front loop of blas_port.CholeskyPort -- TEST INFRASTRUCTURE ONLY.

The reference's CPU Cholesky (ref_factorize!, src/reference/cholesky.jl:44-111): per front in
postorder, assemble A and the children's contribution blocks, then LAPACK potrf and BLAS trsm and
syrk on the dense column-major front; the solve (src/reference/cholesky.jl:127-170) as supernodal
sweeps with BLAS trsm and gemm. The BLAS and LAPACK calls are scipy's (OpenBLAS, multithreaded).
All index arrays are 0-based.
"""
from libc.stdlib cimport calloc, free, malloc
from scipy.linalg.cython_blas cimport dgemm, dsyrk, dtrsm
from scipy.linalg.cython_lapack cimport dpotrf


def factorize(const long long[::1] post, const long long[::1] parent, const long long[::1] fr,
              const long long[::1] wd, const long long[::1] base, const long long[::1] aptr,
              const long long[::1] ai, const long long[::1] aj, const long long[::1] asrc,
              const long long[::1] cptr, const long long[::1] clist, const long long[::1] rptr,
              const long long[::1] rind, const double[::1] nz, double[::1] factor):
    """Returns -1 on success, else the 0-based front-local column of the first failed pivot times the
    number of fronts plus the front (decoded by the caller)."""
    cdef Py_ssize_t ns = post.shape[0]
    cdef double** cbs = <double**> calloc(ns, sizeof(double*))
    cdef long long* cbm = <long long*> calloc(ns, sizeof(long long))
    cdef Py_ssize_t t, s, c, k, ii, jj, i, j
    cdef long long f, w, m, mc, r0
    cdef int fi, wi, mi, info
    cdef double one = 1.0, mone = -1.0
    cdef double* F
    cdef double* cb
    cdef long long result = -1
    with nogil:
        for t in range(ns):
            s = post[t]
            f = fr[s]
            w = wd[s]
            m = f - w
            F = <double*> calloc(f * f, sizeof(double))
            for k in range(aptr[s], aptr[s + 1]):
                F[ai[k] + aj[k] * f] += nz[asrc[k]]
            for k in range(cptr[s], cptr[s + 1]):
                c = clist[k]
                cb = cbs[c]
                if cb == NULL:
                    continue
                mc = cbm[c]
                r0 = rptr[c]
                for jj in range(mc):
                    j = rind[r0 + jj]
                    for ii in range(jj, mc):
                        F[rind[r0 + ii] + j * f] += cb[ii + jj * mc]
                free(cb)
                cbs[c] = NULL
            fi = <int> f
            wi = <int> w
            mi = <int> m
            dpotrf(b"L", &wi, F, &fi, &info)
            if info != 0:
                result = (info - 1) * ns + s
                free(F)
                break
            if m > 0:
                dtrsm(b"R", b"L", b"T", b"N", &mi, &wi, &one, F, &fi, F + w, &fi)
                if parent[s] >= 0:
                    dsyrk(b"L", b"N", &mi, &wi, &mone, F + w, &fi, &one, F + w + w * f, &fi)
                    cb = <double*> malloc(m * m * sizeof(double))
                    for jj in range(m):
                        for ii in range(jj, m):
                            cb[ii + jj * m] = F[w + ii + (w + jj) * f]
                    cbs[s] = cb
                    cbm[s] = m
            for j in range(w):
                for i in range(j, f):
                    factor[base[s] + j * f + i] = F[i + j * f]
            free(F)
    for s in range(ns):
        if cbs[s] != NULL:
            free(cbs[s])
    free(cbs)
    free(cbm)
    return result


def solve(const long long[::1] post, const long long[::1] fr, const long long[::1] wd,
          const long long[::1] base, const long long[::1] c0, const long long[::1] rowptr,
          const long long[::1] rowval, const double[::1] factor, double[::1, :] Y):
    """In place: Y <- L^-T L^-1 Y (Y n x nrhs, column-major, rows in the factor's order)."""
    cdef Py_ssize_t ns = post.shape[0], t, s, i, r
    cdef int n = <int> Y.shape[0], nrhs = <int> Y.shape[1]
    cdef long long f, w, m
    cdef int fi, wi, mi
    cdef double one = 1.0, mone = -1.0, zero = 0.0
    cdef double* Yp = &Y[0, 0]
    cdef const double* P
    cdef double* T
    cdef long long maxm = 0
    for s in range(ns):
        if fr[s] - wd[s] > maxm:
            maxm = fr[s] - wd[s]
    T = <double*> malloc((maxm * nrhs + 1) * sizeof(double))
    with nogil:
        for t in range(ns):                      # forward: L y = b
            s = post[t]
            f = fr[s]
            w = wd[s]
            m = f - w
            fi = <int> f
            wi = <int> w
            mi = <int> m
            P = &factor[base[s]]
            dtrsm(b"L", b"L", b"N", b"N", &wi, &nrhs, &one, <double*> P, &fi, Yp + c0[s], &n)
            if m > 0:
                dgemm(b"N", b"N", &mi, &nrhs, &wi, &one, <double*> P + w, &fi, Yp + c0[s], &n, &zero, T, &mi)
                for r in range(nrhs):
                    for i in range(m):
                        Yp[rowval[rowptr[s] + w + i] + r * n] -= T[i + r * m]
        for t in range(ns - 1, -1, -1):          # backward: L^T x = y
            s = post[t]
            f = fr[s]
            w = wd[s]
            m = f - w
            fi = <int> f
            wi = <int> w
            mi = <int> m
            P = &factor[base[s]]
            if m > 0:
                for r in range(nrhs):
                    for i in range(m):
                        T[i + r * m] = Yp[rowval[rowptr[s] + w + i] + r * n]
                dgemm(b"T", b"N", &wi, &nrhs, &mi, &mone, <double*> P + w, &fi, T, &mi, &one, Yp + c0[s], &n)
            dtrsm(b"L", b"L", b"T", b"N", &wi, &nrhs, &one, <double*> P, &fi, Yp + c0[s], &n)
    free(T)

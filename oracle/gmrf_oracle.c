/*
 * CPU restatement of the element GMRF sampler's two sparse kernels.  TEST
 * INFRASTRUCTURE ONLY: built by oracle/Makefile into oracle/_ref/, loaded by
 * oracle/gmrf_oracle.py, used by the tests and by bench.py's reference arm (to
 * synthesise that arm's material without the product library).
 *
 * The reference samples X = L^{-T} Z from a Cholesky factor of the precision
 * (GMRF.py:304-354).  The factor itself comes from SciPy's SuperLU (a library);
 * these two routines act on it:
 *
 *   oracle_solve_lt    x <- L^{-T} x for a unit lower-triangular L given in CSC,
 *                      one right-hand side at a time (plain backward substitution
 *                      over the rows of L^T, which are the columns of L);
 *   oracle_marginals   diag(Q^{-1}) for Q = L D L^T by the Takahashi recurrences
 *                      (Takahashi, Fagan & Chen 1973; Rue & Held 2005, sec. 2.3.1)
 *                          S_ij = -sum_{k > j, k in col j} L_kj S_ki       (i > j, i in col j)
 *                          S_jj = 1/D_j - sum_{k > j, k in col j} L_kj S_kj
 *                      for j = n-1 .. 0, S kept only on the pattern of L (which
 *                      the recurrence never leaves, the pattern being fill-closed);
 *                      column j's rows are marked in a dense map, and each pair
 *                      k < i of them is met by walking column k.
 * Returns 0, or -1 on a malformed factor.
 */
#include <stdint.h>
#include <stdlib.h>

int oracle_solve_lt(int64_t n, const int64_t* colptr, const int64_t* rowind, const double* lval,
                    int64_t nrhs, int64_t ld, double* x) {
    if (n <= 0 || nrhs <= 0 || ld < nrhs) return -1;
    for (int64_t s = 0; s < nrhs; ++s) {
        for (int64_t i = n - 1; i >= 0; --i) {
            double v = x[i * ld + s];
            for (int64_t p = colptr[i]; p < colptr[i + 1]; ++p)
                if (rowind[p] > i) v -= lval[p] * x[rowind[p] * ld + s];
            x[i * ld + s] = v;
        }
    }
    return 0;
}

int oracle_marginals(int64_t n, const int64_t* colptr, const int64_t* rowind, const double* lval,
                     const double* d, double* out) {
    if (n <= 0) return -1;
    const int64_t nnz = colptr[n];
    double* sv = (double*)calloc((size_t)(nnz > 0 ? nnz : 1), sizeof(double));
    double* sd = (double*)calloc((size_t)n, sizeof(double));
    double* acc = (double*)calloc((size_t)n, sizeof(double));   /* S_ij being formed */
    double* lj = (double*)calloc((size_t)n, sizeof(double));    /* L_ij of column j */
    char* in_col = (char*)calloc((size_t)n, 1);                 /* row i is in column j */
    if (!sv || !sd || !acc || !lj || !in_col) {
        free(sv), free(sd), free(acc), free(lj), free(in_col);
        return -1;
    }
    int rc = 0;
    for (int64_t j = n - 1; j >= 0 && rc == 0; --j) {
        if (d[j] == 0.0) {
            rc = -1;
            break;
        }
        for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p) {
            const int64_t i = rowind[p];
            if (i <= j) continue;
            in_col[i] = 1;
            lj[i] = lval[p];
            acc[i] = -lval[p] * sd[i];      /* the k = i term */
        }
        /* the k != i terms: every pair k < i of rows of column j meets in column k */
        for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p) {
            const int64_t k = rowind[p];
            if (k <= j) continue;
            int64_t found = 0, want = 0;
            for (int64_t q = p + 1; q < colptr[j + 1]; ++q) want += rowind[q] > k;
            for (int64_t q = colptr[k]; q < colptr[k + 1] && found < want; ++q) {
                const int64_t i = rowind[q];
                if (i <= k || !in_col[i]) continue;
                ++found;
                acc[i] -= lj[k] * sv[q];    /* L_kj S_ik */
                acc[k] -= lj[i] * sv[q];    /* L_ij S_ik */
            }
            if (found != want) rc = -1;     /* the pattern is not fill-closed */
        }
        double s = 1.0 / d[j];
        for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p) {
            const int64_t i = rowind[p];
            if (i <= j) continue;
            sv[p] = acc[i];
            s -= lval[p] * acc[i];
            in_col[i] = 0;
        }
        sd[j] = s;
    }
    for (int64_t j = 0; j < n && rc == 0; ++j) out[j] = sd[j];
    free(sv), free(sd), free(acc), free(lj), free(in_col);
    return rc;
}

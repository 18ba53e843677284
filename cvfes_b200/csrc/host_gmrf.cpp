// Host-side selected inversion for the GMRF sampler: the diagonal of Q^{-1}
// from a sparse factor Q = L D Lᵀ (L unit lower triangular, CSC, rows sorted).
//
// The reference rescales each field by the empirical standard deviation across
// samples (GMRF.py:326-328); the exact marginal variances diag(Q^{-1}) used here
// come from the Takahashi recurrences
//     Z_ij = -sum_{k in R_j} L_kj Z_ik          (i in R_j)
//     Z_jj = 1/D_j - sum_{k in R_j} L_kj Z_kj
// with R_j the below-diagonal structure of column j, evaluated for j = n-1..0 on
// the (fill-closed) pattern of L.
#include <cstdint>
#include <vector>

#include "cvfes_b200.h"
#include "errors.h"

extern "C" int cvfes_gmrf_selected_inverse_diag(int64_t n, const int64_t* colptr,
                                                const int64_t* rowind, const double* lval,
                                                const double* d, double* out_diag) {
    if (n <= 0 || !colptr || !rowind || !lval || !d || !out_diag)
        return cvfes::fail(CVFES_ERR_ARG, "cvfes_gmrf_selected_inverse_diag: bad argument");
    // Z stored on L's pattern: zval[p] = Z[rowind[p], column of p]; zdiag[j] = Z_jj.
    std::vector<double> zval(colptr[n], 0.0), zdiag(n, 0.0);
    for (int64_t j = 0; j < n; ++j) {
        for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p) {
            if (rowind[p] < j)
                return cvfes::fail(CVFES_ERR_ARG, "selected inverse: factor is not lower");
            if (p > colptr[j] && rowind[p] <= rowind[p - 1])
                return cvfes::fail(CVFES_ERR_ARG, "selected inverse: rows not sorted");
        }
        if (d[j] == 0.0) return cvfes::fail(CVFES_ERR_ARG, "selected inverse: zero pivot");
    }
    std::vector<double> acc(n, 0.0);
    std::vector<int64_t> rows;
    std::vector<double> lk;
    for (int64_t j = n - 1; j >= 0; --j) {
        rows.clear();
        lk.clear();
        for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p)
            if (rowind[p] > j) {
                rows.push_back(rowind[p]);
                lk.push_back(lval[p]);
            }
        const size_t r = rows.size();
        for (size_t a = 0; a < r; ++a) acc[rows[a]] = 0.0;
        for (size_t a = 0; a < r; ++a) {
            const int64_t k = rows[a];
            const double lkj = lk[a];
            acc[k] -= lkj * zdiag[k];
            // merge column k's stored rows (> k) with rows[a+1..]
            int64_t p = colptr[k];
            const int64_t pe = colptr[k + 1];
            for (size_t b = a + 1; b < r; ++b) {
                const int64_t i = rows[b];
                while (p < pe && rowind[p] < i) ++p;
                if (p < pe && rowind[p] == i) {
                    const double zik = zval[p];
                    acc[i] -= lkj * zik;       // term k of Z_ij
                    acc[k] -= lk[b] * zik;     // term i of Z_kj
                } else {
                    return cvfes::fail(CVFES_ERR_ARG,
                                       "selected inverse: pattern is not fill-closed");
                }
            }
        }
        double zjj = 1.0 / d[j];
        for (size_t a = 0; a < r; ++a) zjj -= lk[a] * acc[rows[a]];
        int64_t p = colptr[j];
        for (size_t a = 0; a < r; ++a) {
            while (rowind[p] != rows[a]) ++p;
            zval[p] = acc[rows[a]];
        }
        zdiag[j] = zjj;
    }
    for (int64_t j = 0; j < n; ++j) out_diag[j] = zdiag[j];
    return CVFES_OK;
}

// Solve Lᵀ X = B in place for a unit lower-triangular L in CSC (the same arrays
// are Lᵀ in CSR), B row-major [n][nrhs] with the samples innermost.  Backward
// substitution; the sample columns are split over OpenMP threads.
extern "C" int cvfes_gmrf_solve_lt(int64_t n, const int64_t* colptr, const int64_t* rowind,
                                   const double* lval, int64_t nrhs, double* b) {
    if (n <= 0 || nrhs <= 0 || !colptr || !rowind || !lval || !b)
        return cvfes::fail(CVFES_ERR_ARG, "cvfes_gmrf_solve_lt: bad argument");
    const int64_t chunk = 16;
    const int64_t nchunks = (nrhs + chunk - 1) / chunk;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t c = 0; c < nchunks; ++c) {
        const int64_t s0 = c * chunk, s1 = (s0 + chunk < nrhs) ? s0 + chunk : nrhs;
        const int64_t w = s1 - s0;
        double acc[chunk];
        for (int64_t i = n - 1; i >= 0; --i) {
            double* bi = b + i * nrhs + s0;
            for (int64_t s = 0; s < w; ++s) acc[s] = bi[s];
            for (int64_t p = colptr[i]; p < colptr[i + 1]; ++p) {
                const int64_t r = rowind[p];
                if (r <= i) continue;
                const double l = lval[p];
                const double* xr = b + r * nrhs + s0;
                for (int64_t s = 0; s < w; ++s) acc[s] -= l * xr[s];
            }
            for (int64_t s = 0; s < w; ++s) bi[s] = acc[s];
        }
    }
    return CVFES_OK;
}

/*
 * Threaded host kernels for timing the oracle's Chebyshev loop on the host cores
 * at the benchmark's full size. TEST INFRASTRUCTURE ONLY: loaded by
 * oracle/cpu.py for bench.py's CPU legs; the product never links or calls it.
 *
 * Blocks are row-major n-by-k arrays (NumPy C order) with leading dimensions.
 * The arithmetic is that of the reference's CPU backend:
 *   - fe_oracle_csr_step: one step of ChebyshevSolver::chebyshev_filter
 *     (src/ChebyshevSolver.cpp:249-256: copy_from(prev), apply_block(2c, -1),
 *     add_scaled_columns(2d)) with the row loop of CpuCsrMatrix::apply_block
 *     (src/core/CsrMatrix.cpp:227-244): y = beta*prev, then y += (alpha*a)*x per
 *     nonzero in CSR order, then y += gamma*cur.
 *   - fe_oracle_residual_norms: the two column_norms of extract_projected_ritz_pairs
 *     (src/core/RitzExtraction.cpp:125-139) on R = AX - X*diag(lambda).
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

void fe_oracle_csr_step(int64_t n, const int32_t* rowptr, const int32_t* colind,
                        const double* val, const double* cur, int64_t ldc, const double* prev,
                        int64_t ldp, double* out, int64_t ldo, int64_t k, double alpha,
                        double gamma, double beta, int threads) {
#pragma omp parallel num_threads(threads)
  {
    double* y = (double*)malloc((size_t)(k > 0 ? k : 1) * sizeof(double));
#pragma omp for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      if (beta != 0.0) {
        const double* p = prev + i * ldp;
        for (int64_t j = 0; j < k; ++j) y[j] = beta * p[j];
      } else {
        memset(y, 0, (size_t)k * sizeof(double));
      }
      for (int32_t q = rowptr[i]; q < rowptr[i + 1]; ++q) {
        const double a = alpha * val[q];
        const double* x = cur + (int64_t)colind[q] * ldc;
        for (int64_t j = 0; j < k; ++j) y[j] += a * x[j];
      }
      if (gamma != 0.0) {
        const double* c = cur + i * ldc;
        for (int64_t j = 0; j < k; ++j) y[j] += gamma * c[j];
      }
      memcpy(out + i * ldo, y, (size_t)k * sizeof(double));
    }
    free(y);
  }
}

void fe_oracle_residual_norms(int64_t n, int64_t k, const double* AX, int64_t lda,
                              const double* X, int64_t ldx, const double* lambda,
                              double* rnorm, double* xnorm, int threads) {
  const int t = threads > 0 ? threads : 1;
  double* part = (double*)calloc((size_t)t * 2 * (size_t)k, sizeof(double));
#pragma omp parallel num_threads(t)
  {
    const int id = omp_get_thread_num();
    double* r2 = part + (size_t)id * 2 * (size_t)k;
    double* x2 = r2 + k;
#pragma omp for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      const double* a = AX + i * lda;
      const double* x = X + i * ldx;
      for (int64_t j = 0; j < k; ++j) {
        const double r = a[j] - lambda[j] * x[j];
        r2[j] += r * r;
        x2[j] += x[j] * x[j];
      }
    }
  }
  for (int64_t j = 0; j < k; ++j) {
    double r = 0.0, x = 0.0;
    for (int id = 0; id < t; ++id) {
      r += part[(size_t)id * 2 * (size_t)k + (size_t)j];
      x += part[(size_t)id * 2 * (size_t)k + (size_t)k + (size_t)j];
    }
    rnorm[j] = sqrt(r);
    xnorm[j] = sqrt(x);
  }
  free(part);
}

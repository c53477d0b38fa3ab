/*
 * A plain C consumer of the fasteig_b200 C ABI (include/fasteig_b200.h): it reads a
 * CSR matrix and expected eigenvalues from a binary file, runs fe_csr_create ->
 * fe_solve -> fe_csr_destroy for each solver named on the command line, and checks
 * the lowest eigenvalues with the rule of the reference's test harness,
 * |dl| <= 1e-10 + 1e-10 |l| (tests/scripts/run_case.py:246-260), and the returned
 * relative residuals against tol. Exit status 0 when every check passes.
 *
 * Input file layout (little endian): int64 n, int64 nnz, int64 nexp,
 * int32 rowptr[n + 1], int32 colind[nnz], double values[nnz], double expected[nexp].
 * Usage: consumer <input> <solver> [<solver> ...]
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fasteig_b200.h"

static void* read_exact(FILE* f, size_t bytes) {
  void* p = malloc(bytes ? bytes : 1);
  if (!p || fread(p, 1, bytes, f) != bytes) {
    fprintf(stderr, "short read\n");
    exit(3);
  }
  return p;
}

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s <input> <solver>...\n", argv[0]);
    return 2;
  }
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 2;
  int64_t hdr[3];
  if (fread(hdr, sizeof(int64_t), 3, f) != 3) return 3;
  const int64_t n = hdr[0], nnz = hdr[1], nexp = hdr[2];
  int32_t* rowptr = (int32_t*)read_exact(f, (size_t)(n + 1) * sizeof(int32_t));
  int32_t* colind = (int32_t*)read_exact(f, (size_t)nnz * sizeof(int32_t));
  double* values = (double*)read_exact(f, (size_t)nnz * sizeof(double));
  double* expected = (double*)read_exact(f, (size_t)nexp * sizeof(double));
  fclose(f);

  printf("library %s\n", fe_version());
  fe_csr_t A = NULL;
  if (fe_csr_create(n, n, nnz, rowptr, colind, values, &A) != FE_OK) {
    fprintf(stderr, "fe_csr_create: %s\n", fe_last_error());
    return 1;
  }
  int64_t rows = 0, cols = 0, stored = 0;
  if (fe_csr_info(A, &rows, &cols, &stored) != FE_OK || rows != n || cols != n || stored != nnz) {
    fprintf(stderr, "fe_csr_info mismatch\n");
    return 1;
  }
  /* An unknown option is an error with a message, not a crash. */
  double ev_bad[1], res_bad[1];
  if (fe_solve(A, NULL, "solver=chebyshev\nnev=1\nno_such_key=1", ev_bad, res_bad, NULL, NULL) !=
          FE_ERR_INVALID ||
      strstr(fe_last_error(), "unknown option") == NULL) {
    fprintf(stderr, "unknown option not rejected: %s\n", fe_last_error());
    return 1;
  }
  int failures = 0;
  for (int s = 2; s < argc; ++s) {
    const int nev = (int)nexp;
    char opts[256];
    snprintf(opts, sizeof opts, "solver=%s\nnev=%d\nwhich=SR\ntol=1e-8\nmaxiter=3000\nseed=1",
             argv[s], nev);
    double* ev = (double*)calloc((size_t)nev, sizeof(double));
    double* res = (double*)calloc((size_t)nev, sizeof(double));
    double* vec = (double*)calloc((size_t)nev * (size_t)n, sizeof(double));
    double stats[12] = {0};
    const int rc = fe_solve(A, NULL, opts, ev, res, vec, stats);
    if (rc != FE_OK) {
      fprintf(stderr, "%s: fe_solve failed (%d): %s\n", argv[s], rc, fe_last_error());
      ++failures;
      continue;
    }
    for (int j = 0; j < nev; ++j) {
      const double tolj = 1e-10 + 1e-10 * fabs(expected[j]);
      if (!(fabs(ev[j] - expected[j]) <= tolj) || !(res[j] <= 1e-8)) {
        fprintf(stderr, "%s: pair %d: %.15g vs %.15g, residual %.3e\n", argv[s], j, ev[j],
                expected[j], res[j]);
        ++failures;
      }
    }
    /* Eigenvectors come back column-major n x nev with unit norm. */
    for (int j = 0; j < nev; ++j) {
      double s2 = 0.0;
      for (int64_t i = 0; i < n; ++i) s2 += vec[(size_t)j * (size_t)n + (size_t)i] * vec[(size_t)j * (size_t)n + (size_t)i];
      if (fabs(sqrt(s2) - 1.0) > 1e-8) {
        fprintf(stderr, "%s: vector %d norm %.12g\n", argv[s], j, sqrt(s2));
        ++failures;
      }
    }
    printf("%s: %d pairs, %g cycles, %.3f s, lowest %.12f\n", argv[s], nev, stats[0], stats[2],
           ev[0]);
    free(ev);
    free(res);
    free(vec);
  }
  if (fe_csr_destroy(A) != FE_OK) ++failures;
  free(rowptr);
  free(colind);
  free(values);
  free(expected);
  return failures ? 1 : 0;
}

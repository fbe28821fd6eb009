/*
 * ref_shims.c -- TEST INFRASTRUCTURE ONLY (CPU oracle).
 *
 * The reference (akohta/bem3_emf_qd2) links Intel MKL for two solver calls:
 *   - PARDISO, wrapped by b_mkl_solver_pardiso_d/_s (d3qd2_src/d3qd2_mkl_solver.c:18-148,150-),
 *     called from solve_tmatrix_csr (d3qd2_src/d3qd2_solve_bieq.c:434-435);
 *   - LAPACKE_zgesv (d3qd2_src/d3qd2_solve_bieq.c:753).
 * MKL is not installed here, so the oracle build replaces d3qd2_mkl_solver.c with this
 * file: a plain dense complex LU with partial pivoting.  It reads the same CSR temp files
 * the reference writes (values, row pointers and column indices as 0-based size_t, RHS),
 * densifies them and solves.  Results agree with PARDISO to round-off (~1e-12), not bitwise.
 * Intended for small meshes only (the dense system is n^2 complex values).
 */
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mkl_types.h"

/* Solve A x = b in place (row-major n x n, nrhs right-hand sides stored row-major
 * with leading dimension ldb).  Returns 0, or k+1 if pivot k is exactly zero. */
static int dense_zlu_solve(size_t n, double complex *A, size_t lda, double complex *B, size_t nrhs,
                           size_t ldb, long long *perm_out)
{
  size_t *perm = (size_t *)malloc(n * sizeof(size_t));
  if (!perm) return -1;
  for (size_t i = 0; i < n; i++) perm[i] = i;
  for (size_t k = 0; k < n; k++) {
    size_t p = k;
    double best = cabs(A[k * lda + k]);
    for (size_t i = k + 1; i < n; i++) {
      double v = cabs(A[i * lda + k]);
      if (v > best) { best = v; p = i; }
    }
    if (best == 0.0) { free(perm); return (int)(k + 1); }
    if (p != k) {
      for (size_t j = 0; j < n; j++) { double complex t = A[k * lda + j]; A[k * lda + j] = A[p * lda + j]; A[p * lda + j] = t; }
      for (size_t j = 0; j < nrhs; j++) { double complex t = B[k * ldb + j]; B[k * ldb + j] = B[p * ldb + j]; B[p * ldb + j] = t; }
      size_t t = perm[k]; perm[k] = perm[p]; perm[p] = t;
    }
    double complex inv = 1.0 / A[k * lda + k];
#pragma omp parallel for schedule(static)
    for (size_t i = k + 1; i < n; i++) {
      double complex f = A[i * lda + k] * inv;
      if (f == 0.0) continue;
      A[i * lda + k] = f;
      double complex *ri = A + i * lda, *rk = A + k * lda;
      for (size_t j = k + 1; j < n; j++) ri[j] -= f * rk[j];
      for (size_t j = 0; j < nrhs; j++) B[i * ldb + j] -= f * B[k * ldb + j];
    }
  }
  for (size_t jj = n; jj-- > 0;) {
    for (size_t r = 0; r < nrhs; r++) {
      double complex s = B[jj * ldb + r];
      for (size_t j = jj + 1; j < n; j++) s -= A[jj * lda + j] * B[j * ldb + r];
      B[jj * ldb + r] = s / A[jj * lda + jj];
    }
  }
  if (perm_out) for (size_t i = 0; i < n; i++) perm_out[i] = (long long)perm[i] + 1;
  free(perm);
  return 0;
}

static void read_or_die(void *buf, size_t sz, size_t cnt, const char *fn)
{
  FILE *fp = fopen(fn, "rb");
  if (!fp) { printf("ref_shims: cannot open %s\n", fn); exit(1); }
  if (fread(buf, sz, cnt, fp) != cnt) { printf("ref_shims: short read on %s\n", fn); exit(1); }
  fclose(fp);
}

/* Replacement for b_mkl_solver_pardiso_d (d3qd2_src/d3qd2_mkl_solver.c:18). */
int b_mkl_solver_pardiso_d(size_t n, size_t nnz, char *fn_a, char *fn_xa, char *fn_asub, char *fn_b,
                           double complex *x)
{
  double complex *val = (double complex *)malloc(nnz * sizeof(double complex));
  size_t *ptr = (size_t *)malloc((n + 1) * sizeof(size_t));
  size_t *idx = (size_t *)malloc(nnz * sizeof(size_t));
  double complex *A = (double complex *)calloc(n * n, sizeof(double complex));
  if (!val || !ptr || !idx || !A) { printf("ref_shims: out of memory (n=%zu)\n", n); exit(1); }
  read_or_die(val, sizeof(double complex), nnz, fn_a);
  read_or_die(ptr, sizeof(size_t), n + 1, fn_xa);
  read_or_die(idx, sizeof(size_t), nnz, fn_asub);
  read_or_die(x, sizeof(double complex), n, fn_b);
  for (size_t i = 0; i < n; i++)
    for (size_t q = ptr[i]; q < ptr[i + 1]; q++) A[i * n + idx[q]] = val[q];
  int err = dense_zlu_solve(n, A, n, x, 1, 1, NULL);
  free(val); free(ptr); free(idx); free(A);
  return err;
}

/* Single-precision PARDISO variant is selected only when PARDISO_PREC==1; the oracle
 * always solves in double precision. */
int b_mkl_solver_pardiso_s(size_t n, size_t nnz, char *fn_a, char *fn_xa, char *fn_asub, char *fn_b,
                           double complex *x)
{
  return b_mkl_solver_pardiso_d(n, nnz, fn_a, fn_xa, fn_asub, fn_b, x);
}

/* Replacement for LAPACKE_zgesv in the row-major form used at d3qd2_solve_bieq.c:753. */
MKL_INT LAPACKE_zgesv(int layout, MKL_INT n, MKL_INT nrhs, MKL_Complex16 *a, MKL_INT lda, MKL_INT *ipiv,
                      MKL_Complex16 *b, MKL_INT ldb)
{
  if (layout != 101) { printf("ref_shims: LAPACKE_zgesv supports row-major only\n"); return -1; }
  return (MKL_INT)dense_zlu_solve((size_t)n, (double complex *)a, (size_t)lda, (double complex *)b,
                                  (size_t)nrhs, (size_t)ldb, (long long *)ipiv);
}

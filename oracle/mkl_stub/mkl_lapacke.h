/* Stand-in declaration of the one LAPACKE routine the reference calls
 * (d3qd2_src/d3qd2_solve_bieq.c:753); oracle/ref_shims.c implements it. */
#ifndef ORACLE_MKL_LAPACKE_STUB_H
#define ORACLE_MKL_LAPACKE_STUB_H
#include "mkl_types.h"
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
MKL_INT LAPACKE_zgesv(int layout, MKL_INT n, MKL_INT nrhs, MKL_Complex16 *a, MKL_INT lda,
                      MKL_INT *ipiv, MKL_Complex16 *b, MKL_INT ldb);
#endif

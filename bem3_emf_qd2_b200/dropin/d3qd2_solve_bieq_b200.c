/*
 * d3qd2_solve_bieq_b200.c -- link-time replacement of bem3_emf_qd2's d3qd2_solve_bieq.o.
 *
 * Provides `void solve_bieq(DQD2 *md)` with the signature and effect of the reference
 * (d3qd2_src/bem3_emf_qd2.h:31, d3qd2_src/d3qd2_solve_bieq.c:36-84): on return the boundary values
 * sb[d].U, dU, E, H, dE, dH of every domain are filled in place.  The work runs on the current
 * CUDA device through libbem3qd2 (bem3_solve_bieq_arrays); no temporary files are written and
 * no MKL is needed, so d3qd2_mkl_solver.o is dropped from the link as well.
 *
 * Build against the reference's headers (d3qd2_src, com_src, qgf2_src on the include path, an
 * MKL header stub where MKL is absent); see this directory's Makefile.  The DQD2 flattening is in
 * d3qd2_flat_b200.c.
 * Errors: like the reference, a failure prints a message and exits with status 1.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "d3qd2_flat_b200.h"

/* the field drop-in's device copy of a DQD2 (d3qd2_field_b200.c), when that drop-in is linked too */
void b200_field_invalidate(DQD2 *qd) __attribute__((weak));

void solve_bieq(DQD2 *md)
{
  time_t start, end;
  b200_flat f;
  bem3_bv *bv;
  double **buf;
  int d, rc, k;

  printf("\nsolve modified electromagnetic potential boundary value (%s)\n", bem3_version());
  time(&start);
  b200_flatten(md, &f);
  bv = b200_xcalloc((size_t)(md->MN + 1), sizeof(bem3_bv));
  buf = b200_xcalloc((size_t)(md->MN + 1) * 6, sizeof(double *));
  for (d = 0; d <= md->MN; d++) {
    const size_t ne = (size_t)md->bd.sb[d].Ne;
    for (k = 0; k < 6; k++) buf[6 * d + k] = b200_xcalloc((ne + 1) * 4 * (k < 2 ? 4 : 3) * 2, sizeof(double));
    bv[d].U = buf[6 * d + 0]; bv[d].dU = buf[6 * d + 1];
    bv[d].E = buf[6 * d + 2]; bv[d].dE = buf[6 * d + 3];
    bv[d].H = buf[6 * d + 4]; bv[d].dH = buf[6 * d + 5];
  }
  printf("  coefficient matrices, boundary values and fields on the GPU "); fflush(stdout);
  rc = bem3_solve_bieq_arrays(&f.P, bv);
  if (rc != 0) {
    printf("\nd3qd2_solve_bieq_b200.c, solve_bieq(), bem3_solve_bieq_arrays() failed. rc=%d. Exit...\n", rc);
    exit(1);
  }
  for (d = 0; d <= md->MN; d++) {
    SUBD *sb = &(md->bd.sb[d]);
    b200_scatter4(sb->U, bv[d].U, sb->Ne);
    b200_scatter4(sb->dU, bv[d].dU, sb->Ne);
    b200_scatter3(sb->E, bv[d].E, sb->Ne);
    b200_scatter3(sb->dE, bv[d].dE, sb->Ne);
    b200_scatter3(sb->H, bv[d].H, sb->Ne);
    b200_scatter3(sb->dH, bv[d].dH, sb->Ne);
  }
  if (b200_field_invalidate) b200_field_invalidate(md);  /* its boundary values have changed */
  time(&end);
  printf("finished. Elapsed time : %5g (sec)\n", difftime(end, start));
  for (k = 0; k < (md->MN + 1) * 6; k++) free(buf[k]);
  free(buf);
  free(bv);
  b200_release(&f);
  printf("Total elapsed time : %g (sec)\n", difftime(end, start));
}

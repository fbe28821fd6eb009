/*
 * d3qd2_flat_b200.h -- DQD2 <-> bem3_problem / bem3_bv layouts for the GPU drop-ins (d3qd2_flat_b200.c).
 */
#ifndef D3QD2_FLAT_B200_H_
#define D3QD2_FLAT_B200_H_

#include "bem3_emf_qd2.h"
#include "bem3_qd2_b200.h"

/* DQD2 (pointer-of-pointer arrays, 1-based ids) -> flat arrays of bem3_problem (P points into them). */
typedef struct {
  bem3_problem P;
  double *cr, *cw, *ren, *wen, *Ui, *dUi, *dEiz, *dEie, *rn, *kn;
  int *nv, *eni, *ed, *Ne_d;
  const int **sid;
  bem3_wave *waves;
} b200_flat;

void *b200_xcalloc(size_t n, size_t sz);  /* calloc that exits with a message on failure */
void b200_flatten(DQD2 *md, b200_flat *f);
void b200_release(b200_flat *f);
/* boundary values [(ne+1)][4][4] / [(ne+1)][4][3] complex: flat (interleaved re, im) <-> DQD2 */
void b200_scatter4(double complex ***dst, const double *src, int ne);
void b200_scatter3(double complex ***dst, const double *src, int ne);
void b200_gather4(double *dst, double complex ***src, int ne);
void b200_gather3(double *dst, double complex ***src, int ne);

#endif

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
 * MKL header stub where MKL is absent); see this directory's Makefile.
 * Errors: like the reference, a failure prints a message and exits with status 1.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "bem3_emf_qd2.h"
#include "bem3_qd2_b200.h"

static void *xcalloc(size_t n, size_t sz)
{
  void *p = calloc(n ? n : 1, sz);
  if (!p) {
    printf("d3qd2_solve_bieq_b200.c, solve_bieq(), memory allocation failed. Exit...\n");
    exit(1);
  }
  return p;
}

/* DQD2 (pointer-of-pointer arrays, 1-based ids) -> flat arrays of bem3_problem. */
typedef struct {
  bem3_problem P;
  double *cr, *cw, *ren, *wen, *Ui, *dUi, *dEiz, *dEie, *rn, *kn;
  int *nv, *eni, *ed, *Ne_d;
  const int **sid;
  bem3_wave *waves;
} flat_problem;

static void flatten(DQD2 *md, flat_problem *f)
{
  BOUD *bd = &(md->bd);
  const int Ne = bd->Ne, Nn = bd->Nn, MN = md->MN;
  int e, i, j, l, d;

  memset(f, 0, sizeof *f);
  f->cr = xcalloc((size_t)(Ne + 1) * 12, sizeof(double));
  f->cw = xcalloc((size_t)(Ne + 1) * 9, sizeof(double));
  f->ren = xcalloc((size_t)(Ne + 1) * 12, sizeof(double));
  f->wen = xcalloc((size_t)(Ne + 1) * 12, sizeof(double));
  f->Ui = xcalloc((size_t)(Ne + 1) * 32, sizeof(double));
  f->dUi = xcalloc((size_t)(Ne + 1) * 32, sizeof(double));
  f->dEiz = xcalloc((size_t)(Ne + 1) * 24, sizeof(double));
  f->dEie = xcalloc((size_t)(Ne + 1) * 24, sizeof(double));
  f->rn = xcalloc((size_t)(Nn + 1) * 3, sizeof(double));
  f->kn = xcalloc((size_t)(MN + 1) * 2, sizeof(double));
  f->nv = xcalloc((size_t)(Ne + 1), sizeof(int));
  f->eni = xcalloc((size_t)(Ne + 1) * 4, sizeof(int));
  f->ed = xcalloc((size_t)(Ne + 1) * 4, sizeof(int));
  f->Ne_d = xcalloc((size_t)(MN + 1), sizeof(int));
  f->sid = xcalloc((size_t)(MN + 1), sizeof(int *));
  f->waves = xcalloc((size_t)(md->pw.n_ipw > 0 ? md->pw.n_ipw : 1), sizeof(bem3_wave));

  for (e = 1; e <= Ne; e++) {
    f->nv[e] = (check_element_type(e, bd) == ELT3) ? 3 : 4;
    for (i = 0; i < 3; i++) {
      for (j = 0; j < 4; j++) f->cr[e * 12 + i * 4 + j] = bd->cr[e][i][j];
      for (j = 0; j < 3; j++) f->cw[e * 9 + i * 3 + j] = bd->cw[e][i][j];
    }
    for (l = 0; l < 4; l++) {
      for (i = 0; i < 3; i++) {
        f->ren[e * 12 + l * 3 + i] = bd->ren[e][l][i];
        f->wen[e * 12 + l * 3 + i] = bd->wen[e][l][i];
      }
      for (i = 0; i < 4; i++) {
        f->Ui[((e * 4 + l) * 4 + i) * 2 + 0] = creal(bd->Ui[e][l][i]);
        f->Ui[((e * 4 + l) * 4 + i) * 2 + 1] = cimag(bd->Ui[e][l][i]);
        f->dUi[((e * 4 + l) * 4 + i) * 2 + 0] = creal(bd->dUi[e][l][i]);
        f->dUi[((e * 4 + l) * 4 + i) * 2 + 1] = cimag(bd->dUi[e][l][i]);
      }
      f->eni[e * 4 + l] = bd->eni[e][l];
      f->ed[e * 4 + l] = bd->ed[e][l];
    }
    /* tangential derivatives of the incident field at the open-region nodes, as q1_solve_eh_bv
       (d3qd2_solve_bieq.c:1003-1004) takes them */
    if (bd->md[e] == 0) {
      for (l = 0; l < f->nv[e]; l++) {
        double vtz[3], vte[3];
        double complex ee[3], hh[3], dz[3], de[3], dh[3];
        tz_te_bd_node(vtz, vte, e, l, bd);
        calc_mipw_EH_dEHdv(ee, hh, dz, dh, bd->ren[e][l], vtz, &(md->pw));
        calc_mipw_EH_dEHdv(ee, hh, de, dh, bd->ren[e][l], vte, &(md->pw));
        for (i = 0; i < 3; i++) {
          f->dEiz[((e * 4 + l) * 3 + i) * 2 + 0] = creal(dz[i]);
          f->dEiz[((e * 4 + l) * 3 + i) * 2 + 1] = cimag(dz[i]);
          f->dEie[((e * 4 + l) * 3 + i) * 2 + 0] = creal(de[i]);
          f->dEie[((e * 4 + l) * 3 + i) * 2 + 1] = cimag(de[i]);
        }
      }
    }
  }
  for (i = 0; i <= Nn; i++)
    for (j = 0; j < 3; j++) f->rn[i * 3 + j] = bd->rn[i][j];
  for (d = 0; d <= MN; d++) {
    f->kn[2 * d + 0] = creal(md->kn[d]);
    f->kn[2 * d + 1] = cimag(md->kn[d]);
    f->Ne_d[d] = bd->sb[d].Ne;
    f->sid[d] = bd->sb[d].sid + 1;
  }
  for (i = 0; i < md->pw.n_ipw; i++) {
    const Ipw *w = &(md->pw.bd.ipw[i]);
    bem3_wave *W = &(f->waves[i]);
    W->E0 = w->data.E0; W->ki = w->data.ki;
    W->cos_t = w->data.cos_t; W->sin_t = w->data.sin_t; W->cos_p = w->data.cos_p; W->sin_p = w->data.sin_p;
    W->f[0] = w->fx; W->f[1] = w->fy; W->f[2] = w->fz;
    W->e[0] = creal(w->data.ex); W->e[1] = cimag(w->data.ex);
    W->e[2] = creal(w->data.ey); W->e[3] = cimag(w->data.ey);
    W->e[4] = creal(w->data.ez); W->e[5] = cimag(w->data.ez);
    W->h[0] = creal(w->data.hx); W->h[1] = cimag(w->data.hx);
    W->h[2] = creal(w->data.hy); W->h[3] = cimag(w->data.hy);
    W->h[4] = creal(w->data.hz); W->h[5] = cimag(w->data.hz);
  }

  f->P.MN = MN; f->P.Ne = Ne; f->P.NN = bd->NN; f->P.ps = bd->ps;
  f->P.mesh.Ne = Ne; f->P.mesh.cr = f->cr; f->P.mesh.cw = f->cw; f->P.mesh.ren = f->ren; f->P.mesh.wen = f->wen;
  f->P.mesh.nv = f->nv;
  f->P.md = bd->md; f->P.sd = bd->sd; f->P.eni = f->eni; f->P.Ne_d = f->Ne_d;
  f->P.sid = (const int *const *)f->sid; f->P.kn = f->kn;
  f->P.qd.k = bd->qd.k;
  for (i = 0; i < 3; i++) f->P.qd.vk[i] = bd->qd.vk[i];
  for (i = 0; i < 2; i++) { f->P.qd.vd1[i] = bd->qd.vd1[i]; f->P.qd.vd2[i] = bd->qd.vd2[i]; }
  f->P.lambda0 = md->pw.lambda_0;
  f->P.Ui = f->Ui; f->P.dUi = f->dUi; f->P.dEiz = f->dEiz; f->P.dEie = f->dEie;
  f->P.Nn = Nn; f->P.rn = f->rn; f->P.ed = f->ed;
  f->P.nwaves = md->pw.n_ipw; f->P.waves = f->waves;
}

static void release(flat_problem *f)
{
  free(f->cr); free(f->cw); free(f->ren); free(f->wen); free(f->Ui); free(f->dUi); free(f->dEiz); free(f->dEie);
  free(f->rn); free(f->kn); free(f->nv); free(f->eni); free(f->ed); free(f->Ne_d); free(f->sid); free(f->waves);
}

static void scatter4(double complex ***dst, const double *src, int ne)
{
  int t, l, i;
  for (t = 1; t <= ne; t++)
    for (l = 0; l < 4; l++)
      for (i = 0; i < 4; i++) dst[t][l][i] = src[((t * 4 + l) * 4 + i) * 2] + I * src[((t * 4 + l) * 4 + i) * 2 + 1];
}

static void scatter3(double complex ***dst, const double *src, int ne)
{
  int t, l, i;
  for (t = 1; t <= ne; t++)
    for (l = 0; l < 4; l++)
      for (i = 0; i < 3; i++) dst[t][l][i] = src[((t * 4 + l) * 3 + i) * 2] + I * src[((t * 4 + l) * 3 + i) * 2 + 1];
}

void solve_bieq(DQD2 *md)
{
  time_t start, end;
  flat_problem f;
  bem3_bv *bv;
  double **buf;
  int d, rc, k;

  printf("\nsolve modified electromagnetic potential boundary value (%s)\n", bem3_version());
  time(&start);
  flatten(md, &f);
  bv = xcalloc((size_t)(md->MN + 1), sizeof(bem3_bv));
  buf = xcalloc((size_t)(md->MN + 1) * 6, sizeof(double *));
  for (d = 0; d <= md->MN; d++) {
    const size_t ne = (size_t)md->bd.sb[d].Ne;
    for (k = 0; k < 6; k++) buf[6 * d + k] = xcalloc((ne + 1) * 4 * (k < 2 ? 4 : 3) * 2, sizeof(double));
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
    scatter4(sb->U, bv[d].U, sb->Ne);
    scatter4(sb->dU, bv[d].dU, sb->Ne);
    scatter3(sb->E, bv[d].E, sb->Ne);
    scatter3(sb->dE, bv[d].dE, sb->Ne);
    scatter3(sb->H, bv[d].H, sb->Ne);
    scatter3(sb->dH, bv[d].dH, sb->Ne);
  }
  time(&end);
  printf("finished. Elapsed time : %5g (sec)\n", difftime(end, start));
  for (k = 0; k < (md->MN + 1) * 6; k++) free(buf[k]);
  free(buf);
  free(bv);
  release(&f);
  printf("Total elapsed time : %g (sec)\n", difftime(end, start));
}

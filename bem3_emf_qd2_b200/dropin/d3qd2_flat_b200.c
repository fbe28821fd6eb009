/*
 * d3qd2_flat_b200.c -- the reference's DQD2 (d3qd2_src/d3qd2_elem.h:49-60: pointer-of-pointer arrays,
 * 1-based element and node ids) flattened into libbem3qd2's bem3_problem, and boundary values moved
 * between the two layouts.  Shared by the drop-in replacements of d3qd2_solve_bieq.o
 * (d3qd2_solve_bieq_b200.c) and of d3qd2_field.o / d3qd2_force.o (d3qd2_field_b200.c).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "d3qd2_flat_b200.h"

void *b200_xcalloc(size_t n, size_t sz)
{
  void *p = calloc(n ? n : 1, sz);
  if (!p) {
    printf("bem3_emf_qd2 GPU drop-in: memory allocation failed. Exit...\n");
    exit(1);
  }
  return p;
}

void b200_flatten(DQD2 *md, b200_flat *f)
{
  BOUD *bd = &(md->bd);
  const int Ne = bd->Ne, Nn = bd->Nn, MN = md->MN;
  int e, i, j, l, d;

  memset(f, 0, sizeof *f);
  f->cr = b200_xcalloc((size_t)(Ne + 1) * 12, sizeof(double));
  f->cw = b200_xcalloc((size_t)(Ne + 1) * 9, sizeof(double));
  f->ren = b200_xcalloc((size_t)(Ne + 1) * 12, sizeof(double));
  f->wen = b200_xcalloc((size_t)(Ne + 1) * 12, sizeof(double));
  f->Ui = b200_xcalloc((size_t)(Ne + 1) * 32, sizeof(double));
  f->dUi = b200_xcalloc((size_t)(Ne + 1) * 32, sizeof(double));
  f->dEiz = b200_xcalloc((size_t)(Ne + 1) * 24, sizeof(double));
  f->dEie = b200_xcalloc((size_t)(Ne + 1) * 24, sizeof(double));
  f->rn = b200_xcalloc((size_t)(Nn + 1) * 3, sizeof(double));
  f->kn = b200_xcalloc((size_t)(MN + 1) * 2, sizeof(double));
  f->nv = b200_xcalloc((size_t)(Ne + 1), sizeof(int));
  f->eni = b200_xcalloc((size_t)(Ne + 1) * 4, sizeof(int));
  f->ed = b200_xcalloc((size_t)(Ne + 1) * 4, sizeof(int));
  f->Ne_d = b200_xcalloc((size_t)(MN + 1), sizeof(int));
  f->sid = b200_xcalloc((size_t)(MN + 1), sizeof(int *));
  f->waves = b200_xcalloc((size_t)(md->pw.n_ipw > 0 ? md->pw.n_ipw : 1), sizeof(bem3_wave));

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

void b200_release(b200_flat *f)
{
  free(f->cr); free(f->cw); free(f->ren); free(f->wen); free(f->Ui); free(f->dUi); free(f->dEiz); free(f->dEie);
  free(f->rn); free(f->kn); free(f->nv); free(f->eni); free(f->ed); free(f->Ne_d); free(f->sid); free(f->waves);
}

void b200_scatter4(double complex ***dst, const double *src, int ne)
{
  int t, l, i;
  for (t = 1; t <= ne; t++)
    for (l = 0; l < 4; l++)
      for (i = 0; i < 4; i++) dst[t][l][i] = src[((t * 4 + l) * 4 + i) * 2] + I * src[((t * 4 + l) * 4 + i) * 2 + 1];
}

void b200_scatter3(double complex ***dst, const double *src, int ne)
{
  int t, l, i;
  for (t = 1; t <= ne; t++)
    for (l = 0; l < 4; l++)
      for (i = 0; i < 3; i++) dst[t][l][i] = src[((t * 4 + l) * 3 + i) * 2] + I * src[((t * 4 + l) * 3 + i) * 2 + 1];
}

void b200_gather4(double *dst, double complex ***src, int ne)
{
  int t, l, i;
  for (t = 1; t <= ne; t++)
    for (l = 0; l < 4; l++)
      for (i = 0; i < 4; i++) {
        dst[((t * 4 + l) * 4 + i) * 2] = creal(src[t][l][i]);
        dst[((t * 4 + l) * 4 + i) * 2 + 1] = cimag(src[t][l][i]);
      }
}

void b200_gather3(double *dst, double complex ***src, int ne)
{
  int t, l, i;
  for (t = 1; t <= ne; t++)
    for (l = 0; l < 4; l++)
      for (i = 0; i < 3; i++) {
        dst[((t * 4 + l) * 3 + i) * 2] = creal(src[t][l][i]);
        dst[((t * 4 + l) * 3 + i) * 2 + 1] = cimag(src[t][l][i]);
      }
}

/*
 * ref_probe.c -- TEST INFRASTRUCTURE ONLY (CPU oracle).
 *
 * A thin ctypes-friendly layer over the reference (akohta/bem3_emf_qd2) compiled from its own
 * sources by oracle/Makefile.  It holds one problem (DQD2) in a static and exposes:
 *   - problem loading through the reference's own readers (read_dqd2 + initialize_dqd2,
 *     d3qd2_src/d3qd2_setup.c:3,105) or dat_read (d3qd2_setup.c:300);
 *   - geometry export (cr, cw, ren, wen, sid, ...) so the GPU path can be fed the identical inputs;
 *   - one element pair exactly as create_cmatrix_domain evaluates it (d3qd2_solve_bieq.c:193-211);
 *   - a row-range restatement of the create_cmatrix_domain loop (d3qd2_solve_bieq.c:190-238)
 *     writing the same matrices to memory instead of temp files;
 *   - the quasi-periodic Green's function entry points (qgf2_src/d3_qpgf_d2.h:112-126) and
 *     Faddeeva_w (qgf2_src/Faddeeva.h);
 *   - the full solve (solve_bieq, d3qd2_solve_bieq.c:36) with ref_shims.c's dense solvers,
 *     boundary-value export, EH_t (d3qd2_field.c:271) and force_FN (d3qd2_force.c:10).
 * It is never linked into the product library.
 */
#include <omp.h>

#include "bem3_emf_qd2.h"

static DQD2 g_qd;
static int g_state = 0; /* 0: empty, 1: loaded by read_dqd2+initialize_dqd2, 2: loaded by dat_read */

int rp_load(const char *ipw, const char *ped, const char *med, const char *msh)
{
  char *argv[6];
  argv[0] = (char *)"oracle";
  argv[1] = (char *)ipw;
  argv[2] = (char *)ped;
  argv[3] = (char *)med;
  argv[4] = (char *)msh;
  argv[5] = (char *)"unused.dat";
  memset(&g_qd, 0, sizeof(g_qd));
  read_dqd2(6, argv, &g_qd);
  initialize_dqd2(&g_qd);
  g_state = 1;
  return 0;
}

int rp_load_dat(const char *dat)
{
  memset(&g_qd, 0, sizeof(g_qd));
  dat_read((char *)dat, &g_qd);
  g_state = 2;
  return 0;
}

void rp_write_dat(const char *dat) { dat_write((char *)dat, &g_qd); }

/* out: MN, Ne, Nn, NN, ps, then sb[d].Ne for d=0..MN (caller provides >= 5+MN+1 ints). */
int rp_info(int *out)
{
  int d;
  out[0] = g_qd.MN;
  out[1] = g_qd.bd.Ne;
  out[2] = g_qd.bd.Nn;
  out[3] = g_qd.bd.NN;
  out[4] = g_qd.bd.ps;
  for (d = 0; d <= g_qd.MN; d++) out[5 + d] = g_qd.bd.sb[d].Ne;
  return g_state;
}

/* Element data for ids 0..Ne (index 0 is the unused slot of the 1-based reference arrays). */
void rp_get_elems(double *cr, double *cw, double *ren, double *wen, int *ed, int *eni, int *md, int *sd)
{
  int i, j, l;
  for (i = 0; i <= g_qd.bd.Ne; i++) {
    for (j = 0; j < 3; j++) {
      for (l = 0; l < 4; l++) cr[(i * 3 + j) * 4 + l] = g_qd.bd.cr[i][j][l];
      for (l = 0; l < 3; l++) cw[(i * 3 + j) * 3 + l] = g_qd.bd.cw[i][j][l];
    }
    for (j = 0; j < 4; j++)
      for (l = 0; l < 3; l++) {
        ren[(i * 4 + j) * 3 + l] = g_qd.bd.ren[i][j][l];
        wen[(i * 4 + j) * 3 + l] = g_qd.bd.wen[i][j][l];
      }
    for (j = 0; j < 4; j++) {
      ed[i * 4 + j] = g_qd.bd.ed[i][j];
      eni[i * 4 + j] = g_qd.bd.eni[i][j];
    }
    md[i] = g_qd.bd.md[i];
    sd[i] = g_qd.bd.sd[i];
  }
}

void rp_get_nodes(double *rn)
{
  int i, l;
  for (i = 0; i <= g_qd.bd.Nn; i++)
    for (l = 0; l < 3; l++) rn[i * 3 + l] = g_qd.bd.rn[i][l];
}

void rp_get_sid(int d, int *sid)
{
  int i;
  for (i = 0; i <= g_qd.bd.sb[d].Ne; i++) sid[i] = g_qd.bd.sb[d].sid[i];
}

/* k, vk[3], vd1[2], vd2[2] */
void rp_get_qpd(double *out)
{
  out[0] = g_qd.bd.qd.k;
  out[1] = g_qd.bd.qd.vk[0]; out[2] = g_qd.bd.qd.vk[1]; out[3] = g_qd.bd.qd.vk[2];
  out[4] = g_qd.bd.qd.vd1[0]; out[5] = g_qd.bd.qd.vd1[1];
  out[6] = g_qd.bd.qd.vd2[0]; out[7] = g_qd.bd.qd.vd2[1];
}

/* complex wave number and refractive index per domain (MN+1 each, interleaved re/im) */
void rp_get_media(double *kn, double *n)
{
  int d;
  for (d = 0; d <= g_qd.MN; d++) {
    kn[2 * d] = creal(g_qd.kn[d]); kn[2 * d + 1] = cimag(g_qd.kn[d]);
    n[2 * d] = creal(g_qd.n[d]);   n[2 * d + 1] = cimag(g_qd.n[d]);
  }
}

/* lambda_0, n_0, n_ipw */
void rp_get_pw(double *out)
{
  out[0] = g_qd.pw.lambda_0;
  out[1] = g_qd.pw.n_0;
  out[2] = (double)g_qd.pw.n_ipw;
}

void rp_get_quad(double *xli, double *wli, double *xhi, double *whi)
{
  int i;
  for (i = 0; i < GLN; i++) { xli[i] = g_qd.bd.xli[i]; wli[i] = g_qd.bd.wli[i]; }
  for (i = 0; i < GHN; i++) { xhi[i] = g_qd.bd.xhi[i]; whi[i] = g_qd.bd.whi[i]; }
}

/* Incident field at element nodes: Ui, dUi [(Ne+1)][4][4] complex */
void rp_get_incident(double complex *Ui, double complex *dUi)
{
  int i, j, l;
  for (i = 0; i <= g_qd.bd.Ne; i++)
    for (j = 0; j < 4; j++)
      for (l = 0; l < 4; l++) {
        Ui[(i * 4 + j) * 4 + l] = g_qd.bd.Ui[i][j][l];
        dUi[(i * 4 + j) * 4 + l] = g_qd.bd.dUi[i][j][l];
      }
}

/* One (collocation node (t,tn), source s) evaluation of domain did, exactly as
 * create_cmatrix_domain makes it (d3qd2_solve_bieq.c:193-211).  t and s are 1-based
 * positions in sb[did].sid.  out = CC[9], dCz[9], dCe[9] (complex). */
void rp_pair(int did, int t, int tn, int s, double complex *out)
{
  double vtz[3], vte[3];
  int td = g_qd.bd.sb[did].sid[t];
  int sd = g_qd.bd.sb[did].sid[s];
  double complex kc = g_qd.kn[did];
  tz_te_bd_node(vtz, vte, td, tn, &(g_qd.bd));
  if (did == 0 && g_qd.bd.ps == 1)
    q0_dcoef_bd_node_t2_cc(out, out + 9, out + 18, td, tn, vtz, vte, sd, kc, PREC_DEF_BE, &(g_qd.bd));
  else
    dcoef_bd_node_t2(out, out + 9, out + 18, td, tn, vtz, vte, sd, kc, PREC_DEF_BE, &(g_qd.bd));
}

/* A batch of pairs (did, t, tn, s) in parallel, for the timed CPU baseline and fixtures. */
void rp_pairs(int n, const int *quads, double complex *out, int nthreads)
{
  int i;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic)
  for (i = 0; i < n; i++) rp_pair(quads[4 * i], quads[4 * i + 1], quads[4 * i + 2], quads[4 * i + 3], out + 27 * (size_t)i);
}

/* Rows t0..t1 (1-based, inclusive) of create_cmatrix_domain (d3qd2_solve_bieq.c:190-238),
 * written to memory in the reference's layout restricted to those rows:
 *   G,H   [(t-t0)*4 + tn][N]     dG,dH [((t-t0)*4 + tn)*2 + {0:tz,1:te}][N]     dF [(t-t0)*4+tn][3]
 * with N = 4*Ne_d.  Rows tn=3 of triangles are zero-filled except for the diagonal of H. */
void rp_assemble_rows(int did, int t0, int t1, double complex *G, double complex *H, double complex *dG,
                      double complex *dH, double *dF, int nthreads)
{
  size_t Ne = (size_t)g_qd.bd.sb[did].Ne, N = 4 * Ne;
  double complex kc = g_qd.kn[did];
  int t;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic)
  for (t = t0; t <= t1; t++) {
    double complex CC[9], dCz[9], dCe[9];
    double vtz[3], vte[3], F, dFz, dFe;
    size_t s, tn, tl, i, row;
    int td = g_qd.bd.sb[did].sid[t], sd;
    tl = (ELT3 == check_element_type(td, &(g_qd.bd))) ? 3 : 4;
    for (tn = 0; tn < tl; tn++) {
      row = (size_t)(t - t0) * 4 + tn;
      tz_te_bd_node(vtz, vte, td, (int)tn, &(g_qd.bd));
      F = 0.0; dFz = 0.0; dFe = 0.0;
      for (s = 1; s <= Ne; s++) {
        sd = g_qd.bd.sb[did].sid[s];
        if (did == 0 && g_qd.bd.ps == 1)
          q0_dcoef_bd_node_t2_cc(CC, dCz, dCe, td, (int)tn, vtz, vte, sd, kc, PREC_DEF_BE, &(g_qd.bd));
        else
          dcoef_bd_node_t2(CC, dCz, dCe, td, (int)tn, vtz, vte, sd, kc, PREC_DEF_BE, &(g_qd.bd));
        for (i = 0; i < 4; i++) {
          G[row * N + (s - 1) * 4 + i] = CC[i];
          H[row * N + (s - 1) * 4 + i] = CC[i + 4];
          dG[(row * 2 + 0) * N + (s - 1) * 4 + i] = dCz[i];
          dH[(row * 2 + 0) * N + (s - 1) * 4 + i] = dCz[i + 4];
          dG[(row * 2 + 1) * N + (s - 1) * 4 + i] = dCe[i];
          dH[(row * 2 + 1) * N + (s - 1) * 4 + i] = dCe[i + 4];
        }
        F += creal(CC[8]);
        dFz += creal(dCz[8]);
        dFe += creal(dCe[8]);
      }
      if (did == 0) {
        H[row * N + (size_t)(t - 1) * 4 + tn] += 1.0 + F;
        dF[row * 3 + 0] = 1.0 + F;
      } else {
        H[row * N + (size_t)(t - 1) * 4 + tn] += F;
        dF[row * 3 + 0] = F;
      }
      dF[row * 3 + 1] = dFz;
      dF[row * 3 + 2] = dFe;
    }
  }
}

/* rp_assemble_rows for the n elements ts[] (1-based positions in domain did's list, any order),
 * parallel over every (element, node, source) of them: rows r = 4 i + tn for element ts[i], same
 * layout and values as rp_assemble_rows element by element.  F and its derivatives are summed per
 * row in source order after the parallel part. */
void rp_assemble_rows_list(int did, int n, const int *ts, double complex *G, double complex *H, double complex *dG,
                           double complex *dH, double *dF, int nthreads)
{
  size_t Ne = (size_t)g_qd.bd.sb[did].Ne, N = 4 * Ne;
  double complex kc = g_qd.kn[did];
  long long total = (long long)n * 4 * (long long)Ne, q;
  double *Fs = (double *)calloc((size_t)total * 3, sizeof(double));
  if (!Fs) return;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
  for (q = 0; q < total; q++) {
    int i = (int)(q / (4 * (long long)Ne)), tn = (int)((q / (long long)Ne) % 4);
    size_t s = (size_t)(q % (long long)Ne) + 1, row = (size_t)i * 4 + tn, k;
    int td = g_qd.bd.sb[did].sid[ts[i]], sd = g_qd.bd.sb[did].sid[s];
    double complex CC[9], dCz[9], dCe[9];
    double vtz[3], vte[3];
    if (tn == 3 && ELT3 == check_element_type(td, &(g_qd.bd))) continue;
    tz_te_bd_node(vtz, vte, td, tn, &(g_qd.bd));
    if (did == 0 && g_qd.bd.ps == 1)
      q0_dcoef_bd_node_t2_cc(CC, dCz, dCe, td, tn, vtz, vte, sd, kc, PREC_DEF_BE, &(g_qd.bd));
    else
      dcoef_bd_node_t2(CC, dCz, dCe, td, tn, vtz, vte, sd, kc, PREC_DEF_BE, &(g_qd.bd));
    for (k = 0; k < 4; k++) {
      G[row * N + (s - 1) * 4 + k] = CC[k];
      H[row * N + (s - 1) * 4 + k] = CC[k + 4];
      dG[(row * 2 + 0) * N + (s - 1) * 4 + k] = dCz[k];
      dH[(row * 2 + 0) * N + (s - 1) * 4 + k] = dCz[k + 4];
      dG[(row * 2 + 1) * N + (s - 1) * 4 + k] = dCe[k];
      dH[(row * 2 + 1) * N + (s - 1) * 4 + k] = dCe[k + 4];
    }
    Fs[3 * q] = creal(CC[8]); Fs[3 * q + 1] = creal(dCz[8]); Fs[3 * q + 2] = creal(dCe[8]);
  }
  /* row sums in source order, as create_cmatrix_domain adds them (d3qd2_solve_bieq.c:222-236) */
  for (int i = 0; i < n; i++) {
    int td = g_qd.bd.sb[did].sid[ts[i]], tn;
    int tl = (ELT3 == check_element_type(td, &(g_qd.bd))) ? 3 : 4;
    for (tn = 0; tn < tl; tn++) {
      size_t row = (size_t)i * 4 + tn, s;
      double F = 0.0, dFz = 0.0, dFe = 0.0;
      for (s = 0; s < Ne; s++) {
        long long q2 = ((long long)i * 4 + tn) * (long long)Ne + (long long)s;
        F += Fs[3 * q2]; dFz += Fs[3 * q2 + 1]; dFe += Fs[3 * q2 + 2];
      }
      H[row * N + (size_t)(ts[i] - 1) * 4 + tn] += (did == 0) ? 1.0 + F : F;
      dF[row * 3 + 0] = (did == 0) ? 1.0 + F : F;
      dF[row * 3 + 1] = dFz;
      dF[row * 3 + 2] = dFe;
    }
  }
  free(Fs);
}

/* rp_assemble_rows with the collocation nodes of elements t0..t1 moved by `ulps` units in the last
 * place along z (nextafter steps; the nodes are restored before return): the reference's own
 * sensitivity to the last bit of a node's height, for rows whose sources lie in the plane of the
 * node to within one ulp. */
void rp_assemble_rows_zshift(int did, int t0, int t1, int ulps, double complex *G, double complex *H,
                             double complex *dG, double complex *dH, double *dF, int nthreads)
{
  int t, tn, k;
  double keep[4096][4];
  if (t1 - t0 + 1 > 4096) return;
  for (t = t0; t <= t1; t++) {
    int td = abs(g_qd.bd.sb[did].sid[t]);
    for (tn = 0; tn < 4; tn++) {
      double *z = &(g_qd.bd.ren[td][tn][2]);
      keep[t - t0][tn] = *z;
      for (k = 0; k < abs(ulps); k++) *z = nextafter(*z, ulps > 0 ? INFINITY : -INFINITY);
    }
  }
  {
    int ts[4096];
    for (t = t0; t <= t1; t++) ts[t - t0] = t;
    rp_assemble_rows_list(did, t1 - t0 + 1, ts, G, H, dG, dH, dF, nthreads);
  }
  for (t = t0; t <= t1; t++) {
    int td = abs(g_qd.bd.sb[did].sid[t]);
    for (tn = 0; tn < 4; tn++) g_qd.bd.ren[td][tn][2] = keep[t - t0][tn];
  }
}

static void set_qpd(QPD2 *q, const double *p)
{
  q->k = p[0];
  q->vk[0] = p[1]; q->vk[1] = p[2]; q->vk[2] = p[3];
  q->vd1[0] = p[4]; q->vd1[1] = p[5];
  q->vd2[0] = p[6]; q->vd2[1] = p[7];
}

/* QPGF entry points over a batch of points.  p = k, vk[3], vd1[2], vd2[2].
 * out per point: qG, dqG[3] (complex); ret per point: the reference's return code. */
void rp_qpgf_v1(int n, const double *r, const double *p, double eps, double complex *out, int *ret)
{
  QPD2 q;
  int i;
  set_qpd(&q, p);
#pragma omp parallel for schedule(dynamic, 64)
  for (i = 0; i < n; i++) ret[i] = d3hm_qpgf_d2_v1(out + 4 * (size_t)i, out + 4 * (size_t)i + 1, (double *)r + 3 * (size_t)i, eps, &q);
}

void rp_qpgf_qG(int n, const double *r, const double *p, double eps, double complex *out, int *ret)
{
  QPD2 q;
  int i;
  set_qpd(&q, p);
#pragma omp parallel for schedule(dynamic, 64)
  for (i = 0; i < n; i++) ret[i] = d3hm_qpgf_d2_qG(out + i, (double *)r + 3 * (size_t)i, eps, &q);
}

void rp_qpgf_dqG(int n, const double *r, const double *p, double eps, double complex *out, int *ret)
{
  QPD2 q;
  int i;
  set_qpd(&q, p);
#pragma omp parallel for schedule(dynamic, 64)
  for (i = 0; i < n; i++) ret[i] = d3hm_qpgf_d2_dqG(out + 3 * (size_t)i, (double *)r + 3 * (size_t)i, eps, &q);
}

/* d3hm_qpgf_d2_v2 (d3_qpgf_d2.c:178-230): out per point qG, dqG[3], d2qG[6] (xx, yy, zz, xy,
 * yz, zx). */
void rp_qpgf_v2(int n, const double *r, const double *p, double eps, double complex *out, int *ret)
{
  QPD2 q;
  int i;
  set_qpd(&q, p);
#pragma omp parallel for schedule(dynamic, 64)
  for (i = 0; i < n; i++)
    ret[i] = d3hm_qpgf_d2_v2(out + 10 * (size_t)i, out + 10 * (size_t)i + 1, out + 10 * (size_t)i + 4,
                             (double *)r + 3 * (size_t)i, eps, &q);
}

void rp_faddeeva(int n, const double complex *z, double relerr, double complex *w)
{
  int i;
  for (i = 0; i < n; i++) w[i] = Faddeeva_w(z[i], relerr);
}

/* Full reference solve on the loaded problem; temp files go to the current directory. */
void rp_solve_bieq(void) { solve_bieq(&g_qd); }

/* Boundary values of domain d for sb[d] positions 0..Ne_d: U,dU [..][4][4], E,dE,H,dH [..][4][3]. */
void rp_get_bv(int d, double complex *U, double complex *dU, double complex *E, double complex *dE,
               double complex *H, double complex *dH)
{
  int i, j, l;
  SUBD *sb = &(g_qd.bd.sb[d]);
  for (i = 0; i <= sb->Ne; i++)
    for (j = 0; j < 4; j++) {
      for (l = 0; l < 4; l++) {
        U[(i * 4 + j) * 4 + l] = sb->U[i][j][l];
        dU[(i * 4 + j) * 4 + l] = sb->dU[i][j][l];
      }
      for (l = 0; l < 3; l++) {
        E[(i * 4 + j) * 3 + l] = sb->E[i][j][l];
        dE[(i * 4 + j) * 3 + l] = sb->dE[i][j][l];
        H[(i * 4 + j) * 3 + l] = sb->H[i][j][l];
        dH[(i * 4 + j) * 3 + l] = sb->dH[i][j][l];
      }
    }
}

void rp_set_bv(int d, const double complex *U, const double complex *dU, const double complex *E,
               const double complex *dE, const double complex *H, const double complex *dH)
{
  int i, j, l;
  SUBD *sb = &(g_qd.bd.sb[d]);
  for (i = 0; i <= sb->Ne; i++)
    for (j = 0; j < 4; j++) {
      for (l = 0; l < 4; l++) {
        sb->U[i][j][l] = U[(i * 4 + j) * 4 + l];
        sb->dU[i][j][l] = dU[(i * 4 + j) * 4 + l];
      }
      for (l = 0; l < 3; l++) {
        sb->E[i][j][l] = E[(i * 4 + j) * 3 + l];
        sb->dE[i][j][l] = dE[(i * 4 + j) * 3 + l];
        sb->H[i][j][l] = H[(i * 4 + j) * 3 + l];
        sb->dH[i][j][l] = dH[(i * 4 + j) * 3 + l];
      }
    }
}

/* EH_t / EH_s at n points (d3qd2_field.c:203,271); returns domain ids in did. */
/* total: 0 EH_s, 1 EH_t, 2 EH_i (d3qd2_field.c:203-300) */
void rp_EH(int n, const double *r, int type, int total, double complex *E, double complex *H, int *did)
{
  int i;
#pragma omp parallel for schedule(dynamic)
  for (i = 0; i < n; i++) {
    double complex *e = E + 3 * (size_t)i, *h = H + 3 * (size_t)i;
    double *p = (double *)r + 3 * (size_t)i;
    if (total == 2) did[i] = EH_i(e, h, p, type, &g_qd);
    else if (total) did[i] = EH_t(e, h, p, type, &g_qd);
    else did[i] = EH_s(e, h, p, type, &g_qd);
  }
}

/* Modified electromagnetic potentials U[4] (vector potential, scalar potential) at points;
 * total: 0 mEMP_s, 1 mEMP_t, 2 mEMP_i (d3qd2_field.c:10-87). */
void rp_mEMP(int n, const double *r, int type, int total, double complex *U, int *did)
{
  int i;
#pragma omp parallel for schedule(dynamic)
  for (i = 0; i < n; i++) {
    double complex *u = U + 4 * (size_t)i;
    double *p = (double *)r + 3 * (size_t)i;
    if (total == 2) did[i] = mEMP_i(u, p, type, &g_qd);
    else if (total) did[i] = mEMP_t(u, p, type, &g_qd);
    else did[i] = mEMP_s(u, p, type, &g_qd);
  }
}

/* Fields from the derivatives of the potentials; total: 0 EH_mEMP_s, 1 EH_mEMP_t, 2 EH_mEMP_i
 * (d3qd2_field.c:89-201). */
void rp_EH_mEMP(int n, const double *r, int type, int total, double complex *E, double complex *H, int *did)
{
  int i;
#pragma omp parallel for schedule(dynamic)
  for (i = 0; i < n; i++) {
    double complex *e = E + 3 * (size_t)i, *h = H + 3 * (size_t)i;
    double *p = (double *)r + 3 * (size_t)i;
    if (total == 2) did[i] = EH_mEMP_i(e, h, p, type, &g_qd);
    else if (total) did[i] = EH_mEMP_t(e, h, p, type, &g_qd);
    else did[i] = EH_mEMP_s(e, h, p, type, &g_qd);
  }
}

int rp_force(double *F, double *N, const double *rc, int type) { return force_FN(F, N, (double *)rc, type, &g_qd); }

int rp_domain_id(const double *r) { return q0_domain_id((double *)r, &g_qd); }

/* Coefficients and their gradients of source element sd at point rt for domain did, as
 * EH_mEMP_s (d3qd2_field.c:124-125) computes them: CC[9], dC[3][9]. */
void rp_dcoef_rt_grad(int did, const double *rt, int sd, int type, double complex *CC, double complex *dC)
{
  double complex d[3][9];
  int p, i;
  if (did == 0 && g_qd.bd.ps == 1) q0_dcoef_rt_grad(CC, d, (double *)rt, sd, g_qd.kn[did], type, &(g_qd.bd));
  else dcoef_rt_grad(CC, d, (double *)rt, sd, g_qd.kn[did], type, &(g_qd.bd));
  for (p = 0; p < 3; p++)
    for (i = 0; i < 9; i++) dC[9 * p + i] = d[p][i];
}

/* Field coefficients of source element sd (signed id) at point rt for domain did, as EH_s
 * (d3qd2_field.c:229-231) computes them: q0_coef_rt in the periodic open region, coef_rt else. */
void rp_coef_rt(int did, const double *rt, int sd, int type, double complex *CC)
{
  if (did == 0 && g_qd.bd.ps == 1) q0_coef_rt(CC, (double *)rt, sd, g_qd.kn[did], type, &(g_qd.bd));
  else coef_rt(CC, (double *)rt, sd, g_qd.kn[did], type, &(g_qd.bd));
}

/*
 * d3qd2_field_b200.c -- link-time replacement of bem3_emf_qd2's d3qd2_field.o and d3qd2_force.o.
 *
 * Every function of the reference's field and force files, with the reference's signatures
 * (d3qd2_src/bem3_emf_qd2.h:36-76), evaluated on the current CUDA device by libbem3qd2:
 *   mEMP_s / mEMP_t / mEMP_i           (d3qd2_field.c:10-87)   -> bem3_ctx_potential
 *   EH_mEMP_s / EH_mEMP_t / EH_mEMP_i  (d3qd2_field.c:89-201)  -> bem3_ctx_field_memp
 *   EH_s / EH_t / EH_i                 (d3qd2_field.c:203-297) -> bem3_ctx_field
 *   EH_s_bd / EH_t_bd / EH_i_bd        (d3qd2_field.c:299-410) -> bem3_ctx_field_bd, bem3_ctx_field (incident)
 *   force_FN                           (d3qd2_force.c:10-54)   -> bem3_ctx_force
 * Return values are the reference's: the point's domain id (the EH_mEMP_* flags for points too close
 * to the boundary included), 0 / -1 for force_FN.
 *
 * The first call with a DQD2 copies its geometry, media, incident waves and boundary values to the
 * device (a bem3_ctx kept for later calls with the same DQD2).  The copy is keyed by the DQD2's
 * address, its boundary-value arrays and a sample of their values, so that a DQD2 read again from
 * another result file gets a fresh copy; the drop-in solve_bieq drops the copy of the DQD2 it solves.
 * A caller that edits boundary values in place otherwise calls b200_field_invalidate(qd).
 *
 * Threads: the reference's examples call the point functions from OpenMP threads
 * (example2.c:30,56,82).  Calls for one DQD2 queue up; whichever caller finds the device idle takes
 * every queued point of the same kind and evaluates them in one library call, then wakes the others.
 * So concurrent callers share launches instead of serialising one point per launch.
 *
 * Not provided (the reference has them): integration type 4 (double-exponential), and the boundary
 * fields EH_s_bd / EH_t_bd of interior domains (did > 0).  Such a call prints a message and exits
 * with status 1, the reference's error convention.
 */
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "d3qd2_flat_b200.h"

#define B200_MAX_CTX 16
#define B200_MAX_BATCH 512

typedef struct b200_req {
  int kind;                 /* 0 EH (bem3_ctx_field), 1 potentials (bem3_ctx_potential), 2 EH_mEMP */
  int type, total;
  double r[3];
  double out[12];           /* E, H (6 + 6 doubles) or U (8 doubles) */
  int did, rc, done;        /* done: written under the entry's mutex only */
  int grouped;              /* run_batch's own marker */
  struct b200_req *next;
} b200_req;

typedef struct {
  DQD2 *qd;
  const void *key_ptr[4];
  int Ne, MN;
  double key_sum;
  bem3_ctx ctx;
  pthread_mutex_t mu;
  pthread_cond_t cv;
  b200_req *head, *tail;    /* queued requests */
  int busy;                 /* a caller is evaluating a batch */
  int used;
} b200_entry;

static b200_entry g_ent[B200_MAX_CTX];
static pthread_mutex_t g_mu = PTHREAD_MUTEX_INITIALIZER;

static void die(const char *fn, const char *msg, int rc)
{
  printf("d3qd2_field_b200.c, %s(), %s (rc=%d). Exit...\n", fn, msg, rc);
  exit(1);
}

/* a sample of the boundary values: tells a DQD2 read from another result file apart */
static double bv_sample(DQD2 *qd)
{
  double s = 0.0;
  int d, t, step;
  for (d = 0; d <= qd->MN; d++) {
    const SUBD *sb = &(qd->bd.sb[d]);
    step = sb->Ne / 16 > 0 ? sb->Ne / 16 : 1;
    for (t = 1; t <= sb->Ne; t += step) {
      s += cabs(sb->E[t][0][0]) + 2.0 * cabs(sb->H[t][1][1]) + 3.0 * cabs(sb->dE[t][0][2]) + 5.0 * cabs(sb->U[t][0][3]);
    }
  }
  return s;
}

static void key_of(DQD2 *qd, const void **kp, int *Ne, int *MN, double *sum)
{
  kp[0] = qd->bd.sb;
  kp[1] = qd->bd.sb[0].E;
  kp[2] = qd->bd.sb[0].dH;
  kp[3] = qd->bd.cr;
  *Ne = qd->bd.Ne;
  *MN = qd->MN;
  *sum = bv_sample(qd);
}

static bem3_ctx make_ctx(DQD2 *qd)
{
  b200_flat f;
  bem3_ctx c = NULL;
  bem3_bv *bv;
  double **buf;
  int d, k, rc;

  b200_flatten(qd, &f);
  rc = bem3_ctx_create(&f.P, &c);
  if (rc) die("make_ctx", "bem3_ctx_create() failed", rc);
  bv = b200_xcalloc((size_t)(qd->MN + 1), sizeof(bem3_bv));
  buf = b200_xcalloc((size_t)(qd->MN + 1) * 6, sizeof(double *));
  for (d = 0; d <= qd->MN; d++) {
    SUBD *sb = &(qd->bd.sb[d]);
    const size_t ne = (size_t)sb->Ne;
    for (k = 0; k < 6; k++) buf[6 * d + k] = b200_xcalloc((ne + 1) * 4 * (k < 2 ? 4 : 3) * 2, sizeof(double));
    b200_gather4(buf[6 * d + 0], sb->U, sb->Ne);
    b200_gather4(buf[6 * d + 1], sb->dU, sb->Ne);
    b200_gather3(buf[6 * d + 2], sb->E, sb->Ne);
    b200_gather3(buf[6 * d + 3], sb->dE, sb->Ne);
    b200_gather3(buf[6 * d + 4], sb->H, sb->Ne);
    b200_gather3(buf[6 * d + 5], sb->dH, sb->Ne);
    bv[d].U = buf[6 * d + 0]; bv[d].dU = buf[6 * d + 1];
    bv[d].E = buf[6 * d + 2]; bv[d].dE = buf[6 * d + 3];
    bv[d].H = buf[6 * d + 4]; bv[d].dH = buf[6 * d + 5];
  }
  rc = bem3_ctx_set_bv(c, bv);
  if (rc) die("make_ctx", "bem3_ctx_set_bv() failed", rc);
  for (k = 0; k < (qd->MN + 1) * 6; k++) free(buf[k]);
  free(buf);
  free(bv);
  b200_release(&f);
  return c;
}

/* The device copy of qd (created on first use). */
static b200_entry *entry_of(DQD2 *qd)
{
  const void *kp[4];
  int Ne, MN, i, slot = -1;
  double sum;
  b200_entry *e;

  key_of(qd, kp, &Ne, &MN, &sum);
  pthread_mutex_lock(&g_mu);
  for (i = 0; i < B200_MAX_CTX; i++) {
    e = &g_ent[i];
    if (!e->used || e->qd != qd) continue;
    if (e->Ne == Ne && e->MN == MN && e->key_sum == sum && !memcmp(e->key_ptr, kp, sizeof kp)) {
      pthread_mutex_unlock(&g_mu);
      return e;
    }
    slot = i;  /* same DQD2, other contents: replace its copy */
    break;
  }
  if (slot < 0) {
    for (i = 0; i < B200_MAX_CTX && slot < 0; i++)
      if (!g_ent[i].used) slot = i;
  }
  if (slot < 0) die("entry_of", "more than 16 DQD2 problems in use", 0);
  e = &g_ent[slot];
  if (e->used) {
    pthread_mutex_lock(&e->mu);
    while (e->busy || e->head) pthread_cond_wait(&e->cv, &e->mu);
    bem3_ctx_destroy(e->ctx);
    e->ctx = NULL;
    pthread_mutex_unlock(&e->mu);
  } else {
    pthread_mutex_init(&e->mu, NULL);
    pthread_cond_init(&e->cv, NULL);
    e->head = e->tail = NULL;
    e->busy = 0;
  }
  e->ctx = make_ctx(qd);
  e->qd = qd;
  memcpy(e->key_ptr, kp, sizeof kp);
  e->Ne = Ne;
  e->MN = MN;
  e->key_sum = sum;
  e->used = 1;
  pthread_mutex_unlock(&g_mu);
  return e;
}

void b200_field_invalidate(DQD2 *qd)
{
  int i;
  pthread_mutex_lock(&g_mu);
  for (i = 0; i < B200_MAX_CTX; i++) {
    b200_entry *e = &g_ent[i];
    if (!e->used || e->qd != qd) continue;
    pthread_mutex_lock(&e->mu);
    while (e->busy || e->head) pthread_cond_wait(&e->cv, &e->mu);
    bem3_ctx_destroy(e->ctx);
    e->ctx = NULL;
    e->used = 0;
    e->qd = NULL;
    pthread_mutex_unlock(&e->mu);
  }
  pthread_mutex_unlock(&g_mu);
}

/* Evaluates one batch (requests of any kinds) with one library call per (kind, type, total). */
static void run_batch(bem3_ctx c, b200_req **rq, int n)
{
  static __thread double *r = NULL, *E = NULL, *H = NULL;
  static __thread int *did = NULL, cap = 0;
  int i, j, m, kind, type, total, rc;
  b200_req *sel[B200_MAX_BATCH];

  if (cap < n) {
    free(r); free(E); free(H); free(did);
    cap = n;
    r = b200_xcalloc((size_t)cap * 3, sizeof(double));
    E = b200_xcalloc((size_t)cap * 8, sizeof(double));
    H = b200_xcalloc((size_t)cap * 6, sizeof(double));
    did = b200_xcalloc((size_t)cap, sizeof(int));
  }
  for (i = 0; i < n; i++) rq[i]->grouped = 0;
  for (i = 0; i < n; i++) {
    if (rq[i]->grouped) continue;
    kind = rq[i]->kind; type = rq[i]->type; total = rq[i]->total;
    m = 0;
    for (j = i; j < n; j++) {
      if (rq[j]->grouped || rq[j]->kind != kind || rq[j]->type != type || rq[j]->total != total) continue;
      sel[m] = rq[j];
      memcpy(r + 3 * m, rq[j]->r, 3 * sizeof(double));
      rq[j]->grouped = 1;
      m++;
    }
    if (kind == 0) rc = bem3_ctx_field(c, m, r, type, total, E, H, did);
    else if (kind == 1) rc = bem3_ctx_potential(c, m, r, type, total, E, did);
    else rc = bem3_ctx_field_memp(c, m, r, type, total, E, H, did);
    for (j = 0; j < m; j++) {
      sel[j]->rc = rc;
      sel[j]->did = did[j];
      if (kind == 1) {
        memcpy(sel[j]->out, E + 8 * j, 8 * sizeof(double));
      } else {
        memcpy(sel[j]->out, E + 6 * j, 6 * sizeof(double));
        memcpy(sel[j]->out + 6, H + 6 * j, 6 * sizeof(double));
      }
    }
  }
}

/* Queues one point and returns once it is evaluated (by this caller or another). */
static void submit(b200_entry *e, b200_req *q)
{
  b200_req *batch[B200_MAX_BATCH];
  int n;

  q->done = 0;
  q->next = NULL;
  pthread_mutex_lock(&e->mu);
  if (e->tail) e->tail->next = q; else e->head = q;
  e->tail = q;
  while (!q->done) {
    if (e->busy) {
      pthread_cond_wait(&e->cv, &e->mu);
      continue;
    }
    /* the device is idle: evaluate what is queued (this request among it) */
    e->busy = 1;
    n = 0;
    while (e->head && n < B200_MAX_BATCH) {
      batch[n++] = e->head;
      e->head = e->head->next;
    }
    if (!e->head) e->tail = NULL;
    pthread_mutex_unlock(&e->mu);
    run_batch(e->ctx, batch, n);
    pthread_mutex_lock(&e->mu);
    for (int i = 0; i < n; i++) batch[i]->done = 1;
    e->busy = 0;
    pthread_cond_broadcast(&e->cv);
  }
  pthread_mutex_unlock(&e->mu);
}

static int point_call(const char *fn, int kind, double complex *A, double complex *B, double *rt, int type, int total,
                      DQD2 *qd)
{
  b200_req q;
  int l;
  if (type < 0 || type > 3) die(fn, "integration type 4 (double-exponential) is not provided by the GPU drop-in", type);
  memset(&q, 0, sizeof q);
  q.kind = kind; q.type = type; q.total = total;
  q.r[0] = rt[0]; q.r[1] = rt[1]; q.r[2] = rt[2];
  submit(entry_of(qd), &q);
  if (q.rc < 0) die(fn, "libbem3qd2 failed", q.rc);
  if (kind == 1) {
    for (l = 0; l < 4; l++) A[l] = q.out[2 * l] + I * q.out[2 * l + 1];
  } else {
    for (l = 0; l < 3; l++) {
      A[l] = q.out[2 * l] + I * q.out[2 * l + 1];
      B[l] = q.out[6 + 2 * l] + I * q.out[6 + 2 * l + 1];
    }
  }
  return q.did;
}

int mEMP_s(double complex *U, double *rt, int type, DQD2 *qd) { return point_call("mEMP_s", 1, U, NULL, rt, type, 0, qd); }
int mEMP_t(double complex *U, double *rt, int type, DQD2 *qd) { return point_call("mEMP_t", 1, U, NULL, rt, type, 1, qd); }
int mEMP_i(double complex *U, double *rt, int type, DQD2 *qd) { return point_call("mEMP_i", 1, U, NULL, rt, type, 2, qd); }

int EH_mEMP_s(double complex *E, double complex *H, double *rt, int type, DQD2 *qd)
{
  return point_call("EH_mEMP_s", 2, E, H, rt, type, 0, qd);
}
int EH_mEMP_t(double complex *E, double complex *H, double *rt, int type, DQD2 *qd)
{
  return point_call("EH_mEMP_t", 2, E, H, rt, type, 1, qd);
}
int EH_mEMP_i(double complex *E, double complex *H, double *rt, int type, DQD2 *qd)
{
  return point_call("EH_mEMP_i", 2, E, H, rt, type, 2, qd);
}

int EH_s(double complex *E, double complex *H, double *rt, int type, DQD2 *qd) { return point_call("EH_s", 0, E, H, rt, type, 0, qd); }
int EH_t(double complex *E, double complex *H, double *rt, int type, DQD2 *qd) { return point_call("EH_t", 0, E, H, rt, type, 1, qd); }
int EH_i(double complex *E, double complex *H, double *rt, int type, DQD2 *qd) { return point_call("EH_i", 0, E, H, rt, type, 2, qd); }

static void bd_call(const char *fn, double complex *E, double complex *H, int did, int t, double zeta_t, double eta_t,
                    int type, int total, DQD2 *qd)
{
  b200_entry *e;
  double ze[2] = {zeta_t, eta_t}, Eo[6], Ho[6];
  int rc, l;
  if (type < 0 || type > 3) die(fn, "integration type 4 (double-exponential) is not provided by the GPU drop-in", type);
  if (did != 0 || qd->bd.ps != 1) die(fn, "boundary fields of interior domains are not provided by the GPU drop-in", did);
  e = entry_of(qd);
  pthread_mutex_lock(&e->mu);
  while (e->busy) pthread_cond_wait(&e->cv, &e->mu);
  e->busy = 1;
  pthread_mutex_unlock(&e->mu);
  rc = bem3_ctx_field_bd(e->ctx, did, 1, &t, ze, type, total, Eo, Ho);
  pthread_mutex_lock(&e->mu);
  e->busy = 0;
  pthread_cond_broadcast(&e->cv);
  pthread_mutex_unlock(&e->mu);
  if (rc < 0) die(fn, "bem3_ctx_field_bd() failed", rc);
  for (l = 0; l < 3; l++) {
    E[l] = Eo[2 * l] + I * Eo[2 * l + 1];
    H[l] = Ho[2 * l] + I * Ho[2 * l + 1];
  }
}

void EH_s_bd(double complex *E, double complex *H, int did, int t, double zeta_t, double eta_t, int type, DQD2 *qd)
{
  bd_call("EH_s_bd", E, H, did, t, zeta_t, eta_t, type, 0, qd);
}
void EH_t_bd(double complex *E, double complex *H, int did, int t, double zeta_t, double eta_t, int type, DQD2 *qd)
{
  bd_call("EH_t_bd", E, H, did, t, zeta_t, eta_t, type, 1, qd);
}
/* the incident field at the point r(zeta_t, eta_t) of the element in the open region, zero elsewhere
   (d3qd2_field.c:388-410) */
void EH_i_bd(double complex *E, double complex *H, int did, int t, double zeta_t, double eta_t, int type, DQD2 *qd)
{
  double rt[3];
  int l;
  (void)type;
  if (did != 0) {
    for (l = 0; l < 3; l++) { E[l] = 0.0; H[l] = 0.0; }
    return;
  }
  r_bd(rt, qd->bd.sb[did].sid[t], zeta_t, eta_t, &(qd->bd));
  point_call("EH_i_bd", 0, E, H, rt, 0, 2, qd);
}

int force_FN(double *F, double *N, double *rc, int type, DQD2 *qd)
{
  b200_entry *e;
  int r;
  if (qd->bd.sb[0].Ne <= 0) return -1;
  e = entry_of(qd);
  pthread_mutex_lock(&e->mu);
  while (e->busy) pthread_cond_wait(&e->cv, &e->mu);
  e->busy = 1;
  pthread_mutex_unlock(&e->mu);
  r = bem3_ctx_force(e->ctx, rc, type == 0 ? 0 : 1, F, N);
  pthread_mutex_lock(&e->mu);
  e->busy = 0;
  pthread_cond_broadcast(&e->cv);
  pthread_mutex_unlock(&e->mu);
  if (r < 0) die("force_FN", "bem3_ctx_force() failed", r);
  return 0;
}

/*
 * qpgf_oracle.c -- TEST INFRASTRUCTURE ONLY: a plain-C99 restatement of the reference's
 * quasi-periodic Green's function and regular element rules, used as a checker (and as the
 * "port" CPU baseline when the compiled reference is not available).  It is pinned against the
 * reference itself by tests/test_oracle_and_math.py (golden vectors from tests/golden/).
 *
 * Restated functions (akohta/bem3_emf_qd2):
 *   qgf2_src/d3_qpgf_d2.c:124-176   d3hm_qpgf_d2_v1 (method selection)      -> or_qpgf_v1
 *   qgf2_src/d3_qpgf_d2.c:409-438   lattice reduction + Bloch phase           -> or_qpgf_v1
 *   qgf2_src/d3_qpgf_d2.c:1671-1712 d3hm_qpgf_d2v1_ew_sd (split parameter)    -> or_ew
 *   qgf2_src/d3_qpgf_d2.c:1714-1838 ew_qG1_v1 (real-space sum)               -> or_ew_real
 *   qgf2_src/d3_qpgf_d2.c:1840-2009 ew_qG2_v1 (spectral sum)                 -> or_ew_spec
 *   qgf2_src/d3_qpgf_d2.c:745-885   d3hm_qpgf_d2v1_fd_sd (Fourier sum)       -> or_fd
 *   qgf2_src/d3_qpgf_d2.c:471-482   stop tests                                -> same / small
 *   qgf2_src/Faddeeva.cc:679-       Faddeeva_w: restated from the published methods
 *                                   (Maclaurin series, trapezoid rule with pole correction,
 *                                   Laplace continued fraction) with a different step (h=0.45)
 *                                   and thresholds than the device code, as an independent check.
 *   d3qd2_src/q0_bil_dcoef_v2_cc.c:129-204, q0_lit_dcoef_v2_cc.c:156-237  -> or_pair_periodic
 *   d3qd2_src/bil_dcoef_v2.c:141-232, lit_dcoef_v2.c:185-270             -> or_pair_interior
 * The element rules follow the reference's loop order (shape function outermost) literally.
 */
#include <complex.h>
#include <math.h>
#include <string.h>

typedef double complex cx;

/* ---------------------------------------------------------------- Faddeeva w(z) */
static cx w_upper(double x, double y)
{
  cx z = x + I * y;
  double r2 = x * x + y * y;
  if (r2 >= 81.0) { /* continued fraction, depth 24 */
    cx t = z;
    for (int n = 24; n >= 1; n--) t = z - 0.5 * n / t;
    return I / (sqrt(M_PI) * t);
  }
  if (r2 < 0.09) { /* Maclaurin series sum (iz)^n / Gamma(n/2+1) */
    cx s = 0, p = 1;
    for (int n = 0; n < 30; n++) {
      s += p / tgamma(0.5 * n + 1.0);
      p *= I * z;
    }
    return s;
  }
  const double h = 0.45;
  const int M = 18;
  double u = fabs(x) / h, fr = u - floor(u);
  int full = fmin(fr, 1.0 - fr) >= fabs(fr - 0.5);
  cx s = 0;
  for (int n = -M; n <= M; n++) {
    double t = full ? n * h : (n + 0.5) * h;
    if (!full && n == M) break;
    s += exp(-t * t) / (z - t);
  }
  cx w = I * h / M_PI * s;
  cx E = cexp(-2.0 * M_PI * I * z / h);
  w += 2.0 * cexp(-z * z) / (full ? 1.0 - E : 1.0 + E);
  return w;
}

cx or_faddeeva(cx z)
{
  double x = creal(z), y = cimag(z);
  if (y >= 0) return w_upper(x, y);
  return 2.0 * cexp(-z * z) - w_upper(-x, -y);
}

void or_faddeeva_batch(int n, const double *z, double *w)
{
  for (int i = 0; i < n; i++) {
    cx v = or_faddeeva(z[2 * i] + I * z[2 * i + 1]);
    w[2 * i] = creal(v);
    w[2 * i + 1] = cimag(v);
  }
}

/* ---------------------------------------------------------------- QPGF */
typedef struct { double k, vk[3], d1[2], d2[2]; } Q;

static int same(cx a, cx b, double e)
{
  return 2 * fabs(creal(a) - creal(b)) <= e * (fabs(creal(a)) + fabs(creal(b))) &&
         2 * fabs(cimag(a) - cimag(b)) <= e * (fabs(cimag(a)) + fabs(cimag(b)));
}
static int small(cx v, cx s, double e) { return fabs(creal(v)) <= fabs(creal(s)) * 0.1 * e && fabs(cimag(v)) <= fabs(cimag(s)) * 0.1 * e; }

static void recip(const Q *q, double g1[2], double g2[2], double *idd)
{
  double det = q->d1[0] * q->d2[1] - q->d2[0] * q->d1[1];
  *idd = 1.0 / det;
  g1[0] = 2 * M_PI * *idd * q->d2[1];  g1[1] = -2 * M_PI * *idd * q->d2[0];
  g2[0] = -2 * M_PI * *idd * q->d1[1]; g2[1] = 2 * M_PI * *idd * q->d1[0];
}

/* real-space Ewald sum; adds terms; returns term count or -1 */
static int or_ew_real(const Q *q, const double *r, double ve, double eps, cx *G, cx dG[3])
{
  int cc = 0;
  *G = 0; dG[0] = dG[1] = dG[2] = 0;
  double ad22 = q->d2[0] * q->d2[0] + q->d2[1] * q->d2[1];
  for (int pass = 0; pass < 3; pass++) {
    int l1 = pass == 0 ? 0 : (pass == 1 ? 1 : -1), st = pass == 2 ? -1 : 1;
    for (; abs(l1) < 100; l1 += st) {
      cx oG = *G;
      int lc = -(int)round(((r[0] + l1 * q->d1[0]) * q->d2[0] + (r[1] + l1 * q->d1[1]) * q->d2[1]) / ad22);
      for (int side = 0; side < 3; side++) {
        int l2 = side == 0 ? lc : (side == 1 ? lc + 1 : lc - 1), s2 = side == 2 ? -1 : 1;
        for (; abs(l2 - lc) < 100; l2 += s2) {
          double R0 = l1 * q->d1[0] + l2 * q->d2[0], R1 = l1 * q->d1[1] + l2 * q->d2[1];
          double px = r[0] + R0, py = r[1] + R1;
          double rl = sqrt(px * px + py * py + r[2] * r[2]);
          double ke = q->k * ve, a = rl / (2 * ve);
          cx ce = cexp(I * (q->vk[0] * R0 + q->vk[1] * R1));
          double ef = exp(ke * ke - a * a);
          cx w = or_faddeeva(ke + I * a);
          cx F = ce / rl * ef * creal(w);
          cx cf = ce / (rl * rl) * ef * (creal(w) / rl - q->k * cimag(w) + 1.0 / (ve * sqrt(M_PI)));
          *G += F; dG[0] += px * cf; dG[1] += py * cf; dG[2] += cf;
          cc++;
          if (side == 0) break;
          if (small(F, *G, eps)) break;
        }
        if (side > 0 && abs(l2 - lc) >= 100) return -1;
      }
      if (pass == 0) break;
      if (same(*G, oG, eps)) break;
    }
    if (pass > 0 && abs(l1) >= 100) return -1;
  }
  *G /= 4 * M_PI; dG[0] /= -4 * M_PI; dG[1] /= -4 * M_PI; dG[2] *= -r[2] / (4 * M_PI);
  return cc;
}

/* spectral Ewald sum; returns term count or negative */
static int or_ew_spec(const Q *q, const double *r, double ve, double eps, cx *G, cx dG[3])
{
  double g1[2], g2[2], idd;
  recip(q, g1, g2, &idd);
  int nc = (int)round((q->vk[0] * q->d1[0] + q->vk[1] * q->d1[1]) / (2 * M_PI)), cc = 0;
  *G = 0; dG[0] = dG[1] = dG[2] = 0;
  for (int pass = 0; pass < 3; pass++) {
    int n1 = nc + (pass == 0 ? 0 : (pass == 1 ? 1 : -1)), st = pass == 2 ? -1 : 1;
    for (; abs(n1 - nc) < 100; n1 += st) {
      cx od = dG[2];
      int nc2 = (int)round(-((-q->vk[0] + n1 * g1[0]) * g2[0] + (-q->vk[1] + n1 * g1[1]) * g2[1]) /
                           (g2[0] * g2[0] + g2[1] * g2[1]));
      int prop = 0;
      for (int side = 0; side < 3; side++) {
        int n2 = side == 0 ? nc2 : (side == 1 ? nc2 + 1 : nc2 - 1), s2 = side == 2 ? -1 : 1;
        for (; abs(n2 - nc2) < 100; n2 += s2) {
          double a0 = -q->vk[0] + n1 * g1[0] + n2 * g2[0], a1 = -q->vk[1] + n1 * g1[1] + n2 * g2[1];
          double b2 = q->k * q->k - a0 * a0 - a1 * a1;
          cx ce = cexp(I * (a0 * r[0] + a1 * r[1])), F, dz;
          int evan;
          if (b2 > 0) {
            double b = sqrt(b2), az = r[2] / (2 * ve);
            double ef = exp(b2 * ve * ve - az * az);
            cx ff = cexp(I * b * r[2]), w = or_faddeeva(b * ve + I * az);
            F = 2.0 * ce / b * (I * ef * cimag(w) + ff);
            dz = 2.0 * ce * (ef * creal(w) - ff);
            evan = 0;
          } else if (b2 < 0) {
            double b = sqrt(-b2), az = r[2] / (2 * ve), eb = exp(b * r[2]);
            double f1 = eb * erfc(b * ve + az), f2 = erfc(b * ve - az) / eb;
            F = ce / (I * b) * (f1 + f2);
            dz = ce * (f1 - f2);
            evan = 1;
          } else return -3;
          *G += F; dG[0] += F * a0; dG[1] += F * a1; dG[2] += dz;
          cc++;
          if (side == 0) break;
          if (evan) { if (small(dz, dG[2], eps)) break; } else prop++;
        }
        if (side > 0 && abs(n2 - nc2) >= 100) return -2;
      }
      if (pass == 0) break;
      if (prop == 0 && same(dG[2], od, eps)) break;
    }
    if (pass > 0 && abs(n1 - nc) >= 100) return -2;
  }
  double a = fabs(idd);
  *G *= 0.25 * I * a; dG[0] *= -0.25 * a; dG[1] *= -0.25 * a; dG[2] *= 0.25 * a;
  return cc;
}

static int or_fd(const Q *q, const double *r, double eps, cx *G, cx dG[3])
{
  if (r[2] == 0.0) return -4;
  double g1[2], g2[2], idd;
  recip(q, g1, g2, &idd);
  int nc = (int)round((q->vk[0] * q->d1[0] + q->vk[1] * q->d1[1]) / (2 * M_PI)), cc = 0;
  *G = 0; dG[0] = dG[1] = dG[2] = 0;
  for (int pass = 0; pass < 3; pass++) {
    int n1 = nc + (pass == 0 ? 0 : (pass == 1 ? 1 : -1)), st = pass == 2 ? -1 : 1;
    for (; abs(n1 - nc) < 100; n1 += st) {
      cx od = dG[2];
      int nc2 = (int)round((q->vk[0] * g2[0] + q->vk[1] * g2[1] - n1 * (g1[0] * g2[0] + g1[1] * g2[1])) /
                           (g2[0] * g2[0] + g2[1] * g2[1]));
      for (int side = 0; side < 3; side++) {
        int n2 = side == 0 ? nc2 : (side == 1 ? nc2 + 1 : nc2 - 1), s2 = side == 2 ? -1 : 1;
        for (; abs(n2 - nc2) < 100; n2 += s2) {
          double a0 = -q->vk[0] + n1 * g1[0] + n2 * g2[0], a1 = -q->vk[1] + n1 * g1[1] + n2 * g2[1];
          double b2 = q->k * q->k - a0 * a0 - a1 * a1;
          cx dz, F;
          int evan;
          if (b2 > 0) {
            double b = sqrt(b2);
            dz = cexp(I * (a0 * r[0] + a1 * r[1] + b * fabs(r[2])));
            F = dz / b; evan = 0;
          } else if (b2 < 0) {
            double b = sqrt(-b2);
            dz = cexp(I * (a0 * r[0] + a1 * r[1])) * exp(-b * fabs(r[2]));
            F = -I * dz / b; evan = 1;
          } else return -2;
          *G += F; dG[0] += F * a0; dG[1] += F * a1; dG[2] += dz;
          cc++;
          if (side == 0) break;
          if (evan && small(dz, dG[2], eps)) break;
        }
        if (side > 0 && abs(n2 - nc2) >= 100) return -1;
      }
      if (pass == 0) break;
      if (same(dG[2], od, eps)) break;
    }
    if (pass > 0 && abs(n1 - nc) >= 100) return -1;
  }
  double a = fabs(idd);
  *G *= 0.5 * I * a; dG[0] *= -0.5 * a; dG[1] *= -0.5 * a; dG[2] *= -0.5 * a * r[2] / fabs(r[2]);
  return cc;
}

int or_qpgf_v1(const double *p, const double *rin, cx *G, cx dG[3])
{
  Q q = {p[0], {p[1], p[2], p[3]}, {p[4], p[5]}, {p[6], p[7]}};
  const double eps = 1e-15;
  double det = q.d1[0] * q.d2[1] - q.d2[0] * q.d1[1], idd = 1.0 / det;
  int l1 = (int)floor((rin[0] * q.d2[1] - rin[1] * q.d2[0]) * idd + 0.5);
  int l2 = (int)floor(-(rin[0] * q.d1[1] - rin[1] * q.d1[0]) * idd + 0.5);
  double r[3] = {rin[0] - l1 * q.d1[0] - l2 * q.d2[0], rin[1] - l1 * q.d1[1] - l2 * q.d2[1], rin[2]};
  /* selection */
  double k2 = q.k * q.k, cpd = 2 * M_PI * idd;
  double ad12 = q.d1[0] * q.d1[0] + q.d1[1] * q.d1[1], ad22 = q.d2[0] * q.d2[0] + q.d2[1] * q.d2[1];
  int n1 = (int)round((q.vk[0] * q.d1[0] + q.vk[1] * q.d1[1]) / (2 * M_PI));
  int n2 = (int)round((q.vk[0] * q.d2[0] + q.vk[1] * q.d2[1]) / (2 * M_PI));
  double ax = -q.vk[0] + n1 * cpd * q.d2[1] - n2 * cpd * q.d1[1], ay = -q.vk[1] - n1 * cpd * q.d2[0] + n2 * cpd * q.d1[0];
  double bN = sqrt(k2 - ax * ax - ay * ay);
  int m1p = n1, m1m = n1, m2p = n2, m2m = n2;
  if (ad22 < ad12) { m1p += 15; m1m -= 15; } else { m2p += 15; m2m -= 15; }
  double px = -q.vk[0] + m1p * cpd * q.d2[1] - m2p * cpd * q.d1[1], py = -q.vk[1] - m1p * cpd * q.d2[0] + m2p * cpd * q.d1[0];
  double mx = -q.vk[0] + m1m * cpd * q.d2[1] - m2m * cpd * q.d1[1], my = -q.vk[1] - m1m * cpd * q.d2[0] + m2m * cpd * q.d1[0];
  double bp = k2 - px * px - py * py, bm = k2 - mx * mx - my * my;
  int fd = 0, err;
  if (!(bp > 0 || bm > 0)) {
    bp = sqrt(-bp); bm = sqrt(-bm);
    fd = bN / bp * exp(-bp * fabs(r[2])) < eps && bN / bm * exp(-bm * fabs(r[2])) < eps;
  }
  if (fd) {
    err = or_fd(&q, r, eps, G, dG);
    if (err < 0) return err - 10;
  } else {
    double adp = sqrt(pow(q.d1[0] + q.d2[0], 2) + pow(q.d1[1] + q.d2[1], 2));
    double adm = sqrt(pow(q.d1[0] - q.d2[0], 2) + pow(q.d1[1] - q.d2[1], 2));
    double ve = sqrt(fabs(det) / (4 * M_PI) * adp / adm), r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    if (k2 * ve * ve - r2 / (4 * ve * ve) > 3.0) ve = sqrt(3.0 + sqrt(k2 * r2 + 9.0)) / (sqrt(2.0) * q.k);
    cx G2, d2[3];
    int c1 = or_ew_real(&q, r, ve, eps, G, dG);
    if (c1 < 0) return c1 - 20;
    int c2 = or_ew_spec(&q, r, ve, eps, &G2, d2);
    if (c2 < 0) return c2 - 20;
    *G += G2; dG[0] += d2[0]; dG[1] += d2[1]; dG[2] += d2[2];
    err = c1 + c2;
  }
  if (l1 || l2) {
    cx cf = cexp(-I * (q.vk[0] * (l1 * q.d1[0] + l2 * q.d2[0]) + q.vk[1] * (l1 * q.d1[1] + l2 * q.d2[1])));
    *G *= cf; dG[0] *= cf; dG[1] *= cf; dG[2] *= cf;
  }
  return err;
}

void or_qpgf_batch(int n, const double *r, const double *p, double *out, int *ret)
{
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n; i++) {
    cx G, dG[3];
    ret[i] = or_qpgf_v1(p, r + 3 * i, &G, dG);
    out[8 * i] = creal(G); out[8 * i + 1] = cimag(G);
    for (int c = 0; c < 3; c++) { out[8 * i + 2 + 2 * c] = creal(dG[c]); out[8 * i + 3 + 2 * c] = cimag(dG[c]); }
  }
}

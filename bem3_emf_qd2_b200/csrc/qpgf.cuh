// qpgf.cuh -- quasi-periodic Helmholtz Green's function of a 2-D lattice (z non-periodic), FP64.
//
// Device (and host) re-implementation of the reference's d3hm_qpgf_d2_v1 / _qG / _dqG
// (qgf2_src/d3_qpgf_d2.c:10-176) with the same mathematics, method choice and adaptive stop
// rules, so that results agree with the reference to round-off:
//
//   G(r) = sum_l e^{i k|| . R_l} e^{ik|r+R_l|} / (4 pi |r+R_l|),   R_l = l1 d1 + l2 d2
//
//  * lattice reduction of r into the cell around the origin and the Bloch phase
//    e^{-i k|| . (l1 d1 + l2 d2)} (d3_qpgf_d2.c:409-438, 290-319);
//  * method choice (d3_qpgf_d2.c:124-176): the pure spectral (Fourier-domain, "FD") sum when
//    no order +-S_LIMIT away from the central one propagates and the slowest evanescent order
//    has decayed below eps at |z|, else the Ewald split ("EW");
//  * EW: split parameter eps_E = sqrt(|det d|/(4 pi) |d1+d2|/|d1-d2|), lowered per point when
//    k^2 eps_E^2 - |r|^2/(4 eps_E^2) > EW_EXPM (d3_qpgf_d2.c:1683-1693); real-space sum with
//    Re w(k eps_E + i R/(2 eps_E)) terms (:1714-1838) and spectral sum with w / erfc terms
//    (:1840-2009);
//  * FD: plane-wave sum over reciprocal-lattice orders (:745-886).
// Stop rules follow the reference's d3hm_sf_comp_z / d3hm_sf_diff_z (:471-482).
//
// Two stop-rule sets are provided:
//   QP_V1   -- exactly the rules of d3hm_qpgf_d2_v1 (used by the regular element rules);
//   QP_BOTH -- a row or a sum stops only once the rules of BOTH d3hm_qpgf_d2_qG and
//              d3hm_qpgf_d2_dqG are met.  The singular element integrals of the reference
//              call those two functions separately at every point (q0_bil_coef.c:444,489);
//              one QP_BOTH evaluation returns both values, each summed at least as far as
//              the reference sums it.
#pragma once

#include "cplx.cuh"
#include "faddeeva.cuh"
#include "erfcx_poly.h"

#define QP_S_LIMIT 15
#define QP_FD_LIMIT 100
#define QP_EW_LIMIT 100
#define QP_EW_EXPM 3.0
#define QP_EFS 0.1
#define QP_MEPS 1.0e-15
#define QP_PROP_CAP 2048  // most propagating orders a hoisted lattice list holds
#ifndef QP_FD_ZFAC
// Fourier-domain sum in the assembly's evaluation (OPT) only for |z| > QP_FD_ZFAC x split parameter:
// (39 / 6.1) sqrt(c), c = cost of a Fourier evanescent term / cost of an Ewald one (measured on B200)
#define QP_FD_ZFAC 4.5
#endif
#define QP_PI 3.14159265358979323846
#define QP_INV_SQRTPI 5.6418958354775628695e-1

#define QP_V1 0
#define QP_BOTH 1

// Lattice and incidence constants.  Built once per problem on the host (qp_lattice_init)
// with the same expressions as the reference so that derived values agree bit-for-bit.
struct QPLattice {
  double k;              // wave number of the periodic (open) domain
  double vkx, vky;       // in-plane Bloch wave vector
  double d1x, d1y, d2x, d2y;
  double detd, idd;      // det[d1 d2], 1/det
  double ad22;           // |d2|^2
  double g1x, g1y, g2x, g2y;  // reciprocal vectors 2 pi idd (d2y,-d2x), 2 pi idd (-d1y, d1x)
  double g22, g12;       // |g2|^2, g1.g2
  double veps0;          // lattice Ewald split parameter
  double bN, bNp, bNm;   // method selection (d3_qpgf_d2.c:135-155)
  int ew_only;           // 1 when bNp>0 || bNm>0 (always Ewald)
  int nc1;               // round(k||.d1 / 2 pi)
  cplx eb2;              // e^{i k||.d2}: Bloch phase step along d2 in the real-space sum
  const struct QPProp* prop;  // propagating spectral orders (qp_prop_list), memory of the caller's side
  int nprop;                  // their number (-1: no list); used by qpgf_eval<MODE, true> only
};

// One propagating spectral order n = (n1, n2): a_n = -k|| + n1 g1 + n2 g2 with beta_n^2 =
// k^2 - |a_n|^2 > 0.  The set depends on the lattice and incidence only, not on the point.
struct QPProp {
  double an0, an1, bn2, bn;
};

struct QPVal {
  cplx G;
  cplx dG[3];
};

BEM_HD int qp_comp(cplx a, cplx b, double eps)  // d3hm_sf_comp_z
{
  return (2.0 * fabs(a.re - b.re) <= eps * (fabs(a.re) + fabs(b.re))) &&
         (2.0 * fabs(a.im - b.im) <= eps * (fabs(a.im) + fabs(b.im)));
}
BEM_HD int qp_diff(cplx v, cplx s, double eps)  // d3hm_sf_diff_z: |v| negligible against |s|
{
  return (fabs(v.re) <= fabs(s.re) * QP_EFS * eps) && (fabs(v.im) <= fabs(s.im) * QP_EFS * eps);
}

#if defined(BEM_TERM_STATS) && !defined(__CUDACC__)
extern unsigned long long bem_stat_t[5];  // real-space, spectral prop., spectral evan., FD prop., FD evan.
#define BEM_STAT_T(i) (bem_stat_t[i]++)
#else
#define BEM_STAT_T(i) ((void)0)
#endif

// Special functions of the terms, out of line when QP_SPECIAL_NOINLINE is set (one copy of their
// code for all call sites).
#if defined(QP_SPECIAL_NOINLINE)
BEM_HD_NOINLINE double qp_erfc(double x) { return erfc(x); }
#else
BEM_HD double qp_erfc(double x) { return erfc(x); }
#endif
// e^{x^2} erfc(x), the assembly form's Ewald spectral terms, which evaluate it at x >= 0 only (the
// term is taken at |z|).  The polynomial form of erfcx_poly.h: t = P / (P + x) maps [0, inf) onto
// (0, 1], and erfcx(x) / t is a degree-22 polynomial in s = 2 t - 1 (Chebyshev interpolant computed
// with mpmath by gen_erfcx_poly.py), accurate to 5e-16 relative on [0, 1e9).  One reciprocal and 23
// multiply-adds without branches: 434 G evaluations/s on a B200 against 273 G/s for CUDA's erfcx
// (term microbenchmark).  Host builds evaluate the same polynomial with an exact division.
// QP_ERFCX_LIB selects CUDA's erfcx on the device instead.  qp_erfcx extends it to x < 0 through
// erfcx(x) = 2 e^{x^2} - erfcx(-x).
BEM_HD double qp_erfcx_poly(double x)  // x >= 0
{
#if defined(__CUDA_ARCH__) && defined(QP_ERFCX_LIB)
  return erfcx(x);
#else
  const double den = ERFCX_P + x;
#if defined(__CUDA_ARCH__)
  const double t = ERFCX_P * __drcp_rn(den);
#else
  const double t = ERFCX_P / den;
#endif
  const double s = 2.0 * t - 1.0;
  double v = erfcx_c[ERFCX_DEG];
#pragma unroll
  for (int k = ERFCX_DEG - 1; k >= 0; k--) v = fma(v, s, erfcx_c[k]);
  return v * t;
#endif
}
BEM_HD double qp_erfcx(double x)
{
  const double p = qp_erfcx_poly(fabs(x));
  return (x >= 0.0) ? p : 2.0 * exp(x * x) - p;
}
#if defined(QP_EXP_NOINLINE)
BEM_HD_NOINLINE double qp_exp(double x) { return exp(x); }
#else
BEM_HD double qp_exp(double x) { return exp(x); }
#endif

// ---------------------------------------------------------------------------------------------
// Ewald real-space term (d3_qpgf_d2.c:1814-1838).  F and dF[3] (dF[2] still lacks the
// factor -z/(4 pi) that the sum applies at the end).  ce = e^{i k||.R_l} is supplied by the
// caller, which advances it along a row by one complex multiply per term instead of a sincos.
// FAST: smag and dmag[3] are the running sums' magnitudes (max of |re|, |im|) of S and dS[0..2].
// Where e^{k^2 eps^2 - R^2 / 4 eps^2} makes the term and its gradient smaller than 3e-13 of them
// (and |z| >= 3.3), w comes from the asymptotic series (faddeeva_w_asym, relative error below
// 2e-4): the error it adds is below 5e-17 of each running sum.  Most real-space terms are of this
// kind; each row side needs one of them for its stop rule.
template <bool FAST = false>
BEM_HD void qp_ew1_term(const QPLattice& L, const double* r, double veps, int l1, int l2, cplx ce, cplx& F, cplx* dF,
                        double smag = 0.0, const double* dmag = nullptr)
{
  BEM_STAT_T(0);
  double Rl0 = (double)l1 * L.d1x + (double)l2 * L.d2x;
  double Rl1 = (double)l1 * L.d1y + (double)l2 * L.d2y;
  double px = r[0] + Rl0, py = r[1] + Rl1;
  double rl2 = px * px + py * py + r[2] * r[2];
  double rl, i_rl;
  if (FAST) {  // one reciprocal square root instead of a square root and a division
    i_rl = rsqrt_(rl2);
    rl = rl2 * i_rl;
  } else {
    rl = sqrt(rl2);
    i_rl = 1.0 / rl;
  }
  double ke = L.k * veps;
  double i_ve = 1.0 / veps;
  double rl_2e = rl * 0.5 * i_ve;
  double ef = qp_exp(ke * ke - rl_2e * rl_2e);
  cplx w;
  const double z2 = ke * ke + rl_2e * rl_2e;
  bool small = false;
  if (FAST && dmag && z2 >= 10.9) {
    const double b = i_rl * ef * 0.6 * rsqrt_(z2);  // bound of |F| (|w| < 0.6 / |z| there)
    const double bd = b * i_rl * (i_rl + L.k);       // of the w-dependent part of |dF| / |p|
    small = b <= 3e-13 * smag && fabs(px) * bd <= 3e-13 * dmag[0] && fabs(py) * bd <= 3e-13 * dmag[1] &&
            bd <= 3e-13 * dmag[2];
  }
  if (small) w = faddeeva_w_asym(ke, rl_2e);
  else w = faddeeva_w_t<FAST>(ke, rl_2e);
  double cfr = i_rl * i_rl * ef * (i_rl * w.re - L.k * w.im + i_ve * QP_INV_SQRTPI);
  cplx cf = ce * cfr;
  F = ce * (i_rl * ef * w.re);
  dF[0] = px * cf;
  dF[1] = py * cf;
  dF[2] = cf;
}

// Ewald spectral term (d3_qpgf_d2.c:1965-2009), propagating (beta_n^2 > 0, bn = beta_n) and
// evanescent (beta_n^2 < 0, bn = |beta_n|) forms.  ce = e^{i a_n.r}.
template <bool FAST = false>
BEM_HD void qp_ew2_prop(const double* r, double veps, double an0, double an1, double bn2, double bn, cplx ce, cplx& F,
                        cplx* dF)
{
  BEM_STAT_T(1);
  // FAST: the term is even in z and its z derivative odd (with ef w(x - iy) = 2 conj(ff) -
  // ef conj(w(x + iy)), x = bn veps, y = z / (2 veps)), so it is evaluated at |z| in the upper half
  // plane, without the reflection's extra exponential, and dF[2] takes the sign of z
  const double zz = FAST ? fabs(r[2]) : r[2];
  double azve = zz / (2.0 * veps);
  double ef = exp(bn2 * veps * veps - azve * azve);
  cplx ff = expi(bn * zz);
  cplx w = FAST ? faddeeva_w_upper_t<FAST>(bn * veps, azve) : faddeeva_w_t<FAST>(bn * veps, azve);
  // Fn = 2 ce / bn (i ef Im w + ff)
  cplx t = mk(ff.re, ef * w.im + ff.im);
  F = FAST ? (ce * (2.0 / bn)) * t : mk(2.0 * ce.re / bn, 2.0 * ce.im / bn) * t;
  dF[0] = F * an0;
  dF[1] = F * an1;
  dF[2] = 2.0 * (ce * mk(ef * w.re - ff.re, -ff.im));
  if (FAST && r[2] < 0.0) dF[2] = -dF[2];
}
// ibn = 1/bn: the evaluation forms below differ only in how they obtain bn and 1/bn.
// FAST: with a = bn veps and b = z / (2 veps) (so that bn z = 2 a b),
//   e^{bn z} erfc(a + b)  = e^{-a^2 - b^2} erfcx(a + b)
//   e^{-bn z} erfc(a - b) = e^{-a^2 - b^2} erfcx(a - b)                 (a >= b)
//                         = 2 e^{-bn z} - e^{-a^2 - b^2} erfcx(b - a)    (a <  b)
// (erfcx(x) = e^{x^2} erfc(x), erfc(-x) = 2 - erfc(x)): one shared exponential and two scaled
// complementary error functions of non-negative arguments instead of two erfc (each an exponential
// inside), an exponential and a division.
template <bool FAST = false>
BEM_HD void qp_ew2_evan(const double* r, double veps, double an0, double an1, double bn, double ibn, cplx ce, cplx& F,
                        cplx* dF)
{
  BEM_STAT_T(2);
  double azve = r[2] / (2.0 * veps);
  double f1, f2;
  if (FAST) {
    // at |z| (f1 and f2 trade places under z -> -z, dF[2] changes sign below), so that both erfcx
    // arguments but the second's in its rare branch are >= 0: no e^{x^2} branch inside erfcx
    const double az = fabs(azve);
    const double a = bn * veps;
    const double E = qp_exp(-(a * a + az * az));
    const double x1 = qp_erfcx_poly(a + az), x2 = qp_erfcx_poly(fabs(a - az));
    f1 = E * x1;
    f2 = (a >= az) ? E * x2 : 2.0 * qp_exp(-bn * fabs(r[2])) - E * x2;
    if (r[2] < 0.0) {
      const double t = f1;
      f1 = f2;
      f2 = t;
    }
  } else {
    double ebz = qp_exp(bn * r[2]);
    // both erfc values from one call site (one copy of its code in the sums)
    double e1 = 0.0, e2 = 0.0;
#pragma unroll 1
    for (int j = 0; j < 2; j++) {
      const double v = qp_erfc(j == 0 ? bn * veps + azve : bn * veps - azve);
      if (j == 0) e1 = v; else e2 = v;
    }
    f1 = ebz * e1;
    f2 = 1.0 / ebz * e2;
  }
  // Fn = ce / (i bn) (f1 + f2) = -i ce (f1+f2)/bn
  F = mul_mi(ce * ((f1 + f2) * ibn));
  dF[0] = F * an0;
  dF[1] = F * an1;
  dF[2] = ce * (f1 - f2);
}
// Returns 0 propagating, 1 evanescent, -3 when beta_n == 0 exactly.
template <bool FAST = false>
BEM_HD int qp_ew2_term(const QPLattice& L, const double* r, double veps, int n1, int n2, cplx ce, cplx& F, cplx* dF)
{
  double an0 = -L.vkx + (double)n1 * L.g1x + (double)n2 * L.g2x;
  double an1 = -L.vky + (double)n1 * L.g1y + (double)n2 * L.g2y;
  double bn2 = L.k * L.k - an0 * an0 - an1 * an1;
  if (bn2 > 0.0) {
    qp_ew2_prop<FAST>(r, veps, an0, an1, bn2, sqrt(bn2), ce, F, dF);
    return 0;
  } else if (bn2 < 0.0) {
    const double bn = sqrt(-bn2);
    qp_ew2_evan<FAST>(r, veps, an0, an1, bn, 1.0 / bn, ce, F, dF);
    return 1;
  }
  return -3;
}

// Fourier-domain term (d3_qpgf_d2.c:856-885), propagating and evanescent forms; ph = e^{i a_n.r}.
BEM_HD void qp_fd_prop(const double* r, double an0, double an1, double bn, cplx ph, cplx& F, cplx* dF)
{
  BEM_STAT_T(3);
  dF[2] = ph * expi(bn * fabs(r[2]));
  F = dF[2] * (1.0 / bn);
  dF[0] = F * an0;
  dF[1] = F * an1;
}
BEM_HD void qp_fd_evan(const double* r, double an0, double an1, double bn, double ibn, cplx ph, cplx& F, cplx* dF)
{
  BEM_STAT_T(4);
  dF[2] = ph * qp_exp(-bn * fabs(r[2]));
  F = mul_mi(dF[2] * ibn);
  dF[0] = F * an0;
  dF[1] = F * an1;
}
// Returns 0 propagating, 1 evanescent, -2 if beta_n == 0.
BEM_HD int qp_fd_term(const QPLattice& L, const double* r, int n1, int n2, cplx ph, cplx& F, cplx* dF)
{
  double an0 = -L.vkx + (double)n1 * L.g1x + (double)n2 * L.g2x;
  double an1 = -L.vky + (double)n1 * L.g1y + (double)n2 * L.g2y;
  double bn2 = L.k * L.k - an0 * an0 - an1 * an1;
  if (bn2 > 0.0) {
    qp_fd_prop(r, an0, an1, sqrt(bn2), ph, F, dF);
    return 0;
  } else if (bn2 < 0.0) {
    const double bn = sqrt(-bn2);
    qp_fd_evan(r, an0, an1, bn, 1.0 / bn, ph, F, dF);
    return 1;
  }
  return -2;
}

// ---------------------------------------------------------------------------------------------
// The three lattice sums below follow the reference's loop nests (rows outermost: the centre row,
// then rows +1, +2, ... until the row rule stops them, then rows -1, -2, ...; inside a row the
// centre term, then the +side and the -side until the term rule stops each) and its stop rules,
// but each is written as ONE flat loop that evaluates exactly one term per iteration and then
// advances a small (row, side, offset) state.  On the GPU, lanes of a warp that follow different
// paths through the nest re-converge at every term instead of at the end of each inner loop, and
// each term function has a single call site (small code, no instruction-cache thrash).

// Ewald real-space sum (d3_qpgf_d2.c:1714-1812).  Returns the number of terms or -1.
// Code-size knobs: the lattice sums are compiled out of line by default (measured faster: fewer
// instruction-cache misses and smaller register demand in the element kernels); the whole
// evaluation can be too.
#if defined(QP_SUM_INLINE)
#define QP_SUM_FN BEM_HD
#else
#define QP_SUM_FN BEM_HD_NOINLINE
#endif
#if defined(QP_EVAL_NOINLINE)
#define QP_EVAL_FN BEM_HD_NOINLINE
#else
#define QP_EVAL_FN BEM_HD
#endif

template <int MODE, bool OPT = false>
BEM_HD int qp_ew1_sum_body(const QPLattice& L, const double* r, double veps, double eps, cplx& S, cplx* dS)
{
  S = mk(0, 0); dS[0] = mk(0, 0); dS[1] = mk(0, 0); dS[2] = mk(0, 0);
  cplx oS = S, od0 = S, od1 = S;
  int cc = 0, dir = 0, l1 = 0, side = -1, off = 0;
  int lc = -(int)round((r[0] * L.d2x + r[1] * L.d2y) / L.ad22);
  cplx ce0 = expi(L.vkx * ((double)lc * L.d2x) + L.vky * ((double)lc * L.d2y));
  cplx ce = ce0;
  for (;;) {
    const int l2 = lc + (side == 1 ? -off : off);
    cplx F, dF[3];
    if (OPT) {
      const double dmag[3] = {fmax(fabs(dS[0].re), fabs(dS[0].im)), fmax(fabs(dS[1].re), fabs(dS[1].im)),
                              fmax(fabs(dS[2].re), fabs(dS[2].im))};
      qp_ew1_term<OPT>(L, r, veps, l1, l2, ce, F, dF, fmax(fabs(S.re), fabs(S.im)), dmag);
    } else {
      qp_ew1_term<OPT>(L, r, veps, l1, l2, ce, F, dF);
    }
    S += F; dS[0] += dF[0]; dS[1] += dF[1]; dS[2] += dF[2];
    cc++;
    bool row_done = false;
    if (side < 0) {
      side = 0; off = 1; ce = ce0 * L.eb2;
      continue;
    }
    bool stop = qp_diff(F, S, eps);
    if (MODE == QP_BOTH) stop = stop && qp_diff(dF[0], dS[0], eps) && qp_diff(dF[1], dS[1], eps);
    if (stop) {
      if (side == 0) { side = 1; off = 1; ce = ce0 * conj(L.eb2); continue; }
      row_done = true;
    } else {
      if (off + 1 >= QP_EW_LIMIT) return -1;
      off++;
      ce = ce * (side == 0 ? L.eb2 : conj(L.eb2));
    }
    if (!row_done) continue;
    // row finished: the row rule decides between the next row and the next direction
    bool rstop = true;
    if (dir != 0) {
      rstop = qp_comp(S, oS, eps);
      if (MODE == QP_BOTH) rstop = rstop && qp_comp(dS[0], od0, eps) && qp_comp(dS[1], od1, eps);
    }
    if (rstop) {
      if (dir == 2) break;
      dir++;
      l1 = (dir == 1) ? 1 : -1;
    } else {
      l1 += (dir == 1) ? 1 : -1;
      if (l1 >= QP_EW_LIMIT || l1 <= -QP_EW_LIMIT) return -1;
    }
    oS = S; od0 = dS[0]; od1 = dS[1];
    lc = -(int)round(((r[0] + (double)l1 * L.d1x) * L.d2x + (r[1] + (double)l1 * L.d1y) * L.d2y) / L.ad22);
    ce0 = expi(L.vkx * ((double)l1 * L.d1x + (double)lc * L.d2x) + L.vky * ((double)l1 * L.d1y + (double)lc * L.d2y));
    ce = ce0;
    side = -1;
    off = 0;
  }
  const double f4p = 4.0 * QP_PI;
  S = mk(S.re / f4p, S.im / f4p);
  dS[0] = mk(dS[0].re / -f4p, dS[0].im / -f4p);
  dS[1] = mk(dS[1].re / -f4p, dS[1].im / -f4p);
  dS[2] = dS[2] * (-r[2] / f4p);
  return cc;
}

// Spectral sums share their row structure.  FD == 0: Ewald spectral sum (d3_qpgf_d2.c:1840-1963,
// returns terms or -2 / -3); FD == 1: Fourier-domain sum (d3_qpgf_d2.c:745-854, returns terms or
// -1 / -2 / -4).  Row rule of the Ewald sum applies only to rows without propagating orders
// beyond the centre (the reference's flg).
//
// OPT: the propagating orders (a fixed set per lattice, L.prop) are summed first, in one loop
// that every lane of a warp runs in step; the row walk then evaluates only evanescent orders and
// passes over the propagating positions (they still count for the row rule).  The stop rules see
// the propagating contributions earlier than the reference's order, so a sum may stop a term
// sooner or later; every neglected term is still below the rule's relative threshold (1e-16 of
// the running sum).  OPT callers must attach the list (qp_prop_list); OPT also selects the
// division-light w(z) (faddeeva_w_t<true>).
template <int MODE, int FD, bool OPT = false>
BEM_HD int qp_spec_sum_body(const QPLattice& L, const double* r, double veps, double eps, cplx& S, cplx* dS)
{
  if (FD && r[2] == 0.0) return -4;
  const int LIMIT = FD ? QP_FD_LIMIT : QP_EW_LIMIT;
  const int ELIM = FD ? -1 : -2;
  S = mk(0, 0); dS[0] = mk(0, 0); dS[1] = mk(0, 0); dS[2] = mk(0, 0);
  const bool hoist = OPT;  // OPT callers always attach the list (L.nprop >= 0)
  int cc = 0;
  if (hoist) {
#pragma unroll 1
    for (int i = 0; i < L.nprop; i++) {
      const QPProp q = L.prop[i];
      const cplx ph = expi(q.an0 * r[0] + q.an1 * r[1]);
      cplx F, dF[3];
      if (FD) qp_fd_prop(r, q.an0, q.an1, q.bn, ph, F, dF);
      else qp_ew2_prop<OPT>(r, veps, q.an0, q.an1, q.bn2, q.bn, ph, F, dF);
      S += F; dS[0] += dF[0]; dS[1] += dF[1]; dS[2] += dF[2];
      cc++;
    }
  }
  cplx oS = S, od2 = dS[2];
  const int nc = L.nc1;
  const cplx E2 = expi(L.g2x * r[0] + L.g2y * r[1]);  // phase step along n2
  int dir = 0, n1 = nc, side = -1, off = 0, flg = 0;
  int nc2;
  if (FD) nc2 = (int)round((L.vkx * L.g2x + L.vky * L.g2y - (double)n1 * L.g12) / L.g22);
  else nc2 = (int)round(-((-L.vkx + (double)n1 * L.g1x) * L.g2x + (-L.vky + (double)n1 * L.g1y) * L.g2y) / L.g22);
  cplx ph0 = expi((-L.vkx + (double)n1 * L.g1x + (double)nc2 * L.g2x) * r[0] +
                  (-L.vky + (double)n1 * L.g1y + (double)nc2 * L.g2y) * r[1]);
  cplx ph = ph0;
  for (;;) {
    const int n2 = nc2 + (side == 1 ? -off : off);
    cplx F, dF[3];
    int e;
    if (hoist) {  // e == 2: a propagating order, already summed
      const double an0 = -L.vkx + (double)n1 * L.g1x + (double)n2 * L.g2x;
      const double an1 = -L.vky + (double)n1 * L.g1y + (double)n2 * L.g2y;
      const double bn2 = L.k * L.k - an0 * an0 - an1 * an1;
      if (bn2 > 0.0) {
        e = 2;
      } else if (bn2 < 0.0) {
        // 1/|beta_n| from one reciprocal square root, |beta_n| = -beta_n^2 / |beta_n|
        const double ibn = rsqrt_(-bn2);
        const double bn = -bn2 * ibn;
        if (FD) qp_fd_evan(r, an0, an1, bn, ibn, ph, F, dF);
        else qp_ew2_evan<OPT>(r, veps, an0, an1, bn, ibn, ph, F, dF);
        e = 1;
      } else {
        e = FD ? -2 : -3;
      }
    } else {
      e = FD ? qp_fd_term(L, r, n1, n2, ph, F, dF) : qp_ew2_term<OPT>(L, r, veps, n1, n2, ph, F, dF);
    }
    if (!FD && e != 2) cc++;
    if (e < 0) return e;
    if (e != 2) {
      S += F; dS[0] += dF[0]; dS[1] += dF[1]; dS[2] += dF[2];
      if (FD) cc++;
    }
    if (side < 0) {
      side = 0; off = 1; ph = ph0 * E2;
      continue;
    }
    bool stop = false;
    if (e == 1) {
      stop = qp_diff(dF[2], dS[2], eps);
      if (MODE == QP_BOTH) stop = stop && qp_diff(F, S, eps);
    } else {
      flg++;
    }
    if (!stop) {
      if (off + 1 >= LIMIT) return ELIM;
      off++;
      ph = ph * (side == 0 ? E2 : conj(E2));
      continue;
    }
    if (side == 0) {
      side = 1; off = 1; ph = ph0 * conj(E2);
      continue;
    }
    // row finished
    bool rstop = true;
    if (dir != 0) {
      rstop = false;
      if (FD || flg == 0) {
        rstop = qp_comp(dS[2], od2, eps);
        if (MODE == QP_BOTH) rstop = rstop && qp_comp(S, oS, eps);
      }
    }
    if (rstop) {
      if (dir == 2) break;
      dir++;
      n1 = (dir == 1) ? nc + 1 : nc - 1;
    } else {
      n1 += (dir == 1) ? 1 : -1;
      if (n1 - nc >= LIMIT || n1 - nc <= -LIMIT) return ELIM;
    }
    oS = S; od2 = dS[2];
    flg = 0;
    if (FD) nc2 = (int)round((L.vkx * L.g2x + L.vky * L.g2y - (double)n1 * L.g12) / L.g22);
    else nc2 = (int)round(-((-L.vkx + (double)n1 * L.g1x) * L.g2x + (-L.vky + (double)n1 * L.g1y) * L.g2y) / L.g22);
    ph0 = expi((-L.vkx + (double)n1 * L.g1x + (double)nc2 * L.g2x) * r[0] +
               (-L.vky + (double)n1 * L.g1y + (double)nc2 * L.g2y) * r[1]);
    ph = ph0;
    side = -1;
    off = 0;
  }
  const double aidd = fabs(L.idd);
  if (FD) {
    S = mul_i(S * (0.5 * aidd));
    dS[0] = dS[0] * (-0.5 * aidd);
    dS[1] = dS[1] * (-0.5 * aidd);
    dS[2] = dS[2] * (-0.5 * aidd * r[2] / fabs(r[2]));
  } else {
    S = mul_i(S * (0.25 * aidd));
    dS[0] = dS[0] * (-0.25 * aidd);
    dS[1] = dS[1] * (-0.25 * aidd);
    dS[2] = dS[2] * (0.25 * aidd);
  }
  return cc;
}

// The sums as called: the point and the running sums are copied into locals so that, out of line,
// they live in registers (through the caller's pointers every term would read and write memory).
template <int MODE, bool OPT = false>
QP_SUM_FN int qp_ew1_sum(const QPLattice& L, const double* r_in, double veps, double eps, cplx& S_out, cplx* dS_out)
{
  const double r[3] = {r_in[0], r_in[1], r_in[2]};
  cplx S, dS[3];
  const int ret = qp_ew1_sum_body<MODE, OPT>(L, r, veps, eps, S, dS);
  S_out = S; dS_out[0] = dS[0]; dS_out[1] = dS[1]; dS_out[2] = dS[2];
  return ret;
}
template <int MODE, int FD, bool OPT = false>
QP_SUM_FN int qp_spec_sum(const QPLattice& L, const double* r_in, double veps, double eps, cplx& S_out, cplx* dS_out)
{
  const double r[3] = {r_in[0], r_in[1], r_in[2]};
  cplx S, dS[3];
  const int ret = qp_spec_sum_body<MODE, FD, OPT>(L, r, veps, eps, S, dS);
  S_out = S; dS_out[0] = dS[0]; dS_out[1] = dS[1]; dS_out[2] = dS[2];
  return ret;
}

// ---------------------------------------------------------------------------------------------
// Full evaluation at r = (x, y, z): G and grad G.  Return value as the reference's
// d3hm_qpgf_d2_v1: > 0 number of terms; -11..-14 FD errors; -21..-24 EW errors.
// OPT (the assembly kernels' form): hoisted propagating orders and the division-light w(z).
template <int MODE, bool OPT = false>
QP_EVAL_FN int qpgf_eval(const QPLattice& L, const double* r_in, QPVal& out)
{
  const double eps = QP_MEPS;
  // lattice reduction (d3_qpgf_d2.c:417-423)
  int l1 = (int)floor((r_in[0] * L.d2y - r_in[1] * L.d2x) * L.idd + 0.5);
  int l2 = (int)floor(-(r_in[0] * L.d1y - r_in[1] * L.d1x) * L.idd + 0.5);
  double r[3];
  r[0] = r_in[0] - (double)l1 * L.d1x - (double)l2 * L.d2x;
  r[1] = r_in[1] - (double)l1 * L.d1y - (double)l2 * L.d2y;
  r[2] = r_in[2];

  bool use_fd = false;
  if (!L.ew_only) {
    use_fd = (L.bN / L.bNp * exp(-L.bNp * fabs(r[2])) < eps) && (L.bN / L.bNm * exp(-L.bNm * fabs(r[2])) < eps);
  }
  // split parameter (d3_qpgf_d2.c:1683-1693)
  double veps = L.veps0;
  {
    const double r2_min = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    if (L.k * L.k * veps * veps - r2_min / (4.0 * veps * veps) > QP_EW_EXPM)
      veps = sqrt(QP_EW_EXPM + sqrt(L.k * L.k * r2_min + QP_EW_EXPM * QP_EW_EXPM)) / (sqrt(2.0) * L.k);
  }
  // OPT: the Fourier-domain sum only where it is also the cheaper one.  Its evanescent orders decay
  // as e^{-beta |z|}, so it needs the orders with |beta| up to ~39 / |z| (a 1e-17 decay); the Ewald
  // sums need those with |beta| up to ~6.1 / veps (erfc below 1e-17) plus a few real-space terms.
  // Both converge to the same value (to ~1e-13 relative on the assembly's points), so the choice is
  // by cost: Fourier only when |z| > QP_FD_ZFAC veps.
  if (OPT && use_fd && fabs(r[2]) < QP_FD_ZFAC * veps) use_fd = false;
  int err;
  if (use_fd) {
    err = qp_spec_sum<MODE, 1, OPT>(L, r, 0.0, eps, out.G, out.dG);
    if (err < 0) return err - 10;
  } else {
    cplx S2, dS2[3];
    int c1 = qp_ew1_sum<MODE, OPT>(L, r, veps, eps, out.G, out.dG);
    if (c1 < 0) return c1 - 20;
    int c2 = qp_spec_sum<MODE, 0, OPT>(L, r, veps, eps, S2, dS2);
    if (c2 < 0) return c2 - 20;
    out.G += S2; out.dG[0] += dS2[0]; out.dG[1] += dS2[1]; out.dG[2] += dS2[2];
    err = c1 + c2;
  }
  if (l1 != 0 || l2 != 0) {
    double arg = -(L.vkx * ((double)l1 * L.d1x + (double)l2 * L.d2x) + L.vky * ((double)l1 * L.d1y + (double)l2 * L.d2y));
    cplx cf = expi(arg);
    out.G = out.G * cf;
    out.dG[0] = out.dG[0] * cf;
    out.dG[1] = out.dG[1] * cf;
    out.dG[2] = out.dG[2] * cf;
  }
  return err;
}

// ---------------------------------------------------------------------------------------------
// Second derivatives: G, grad G and the Hessian d2G = (xx, yy, zz, xy, yz, zx) at r, for the fields
// computed from the derivatives of the potentials (d3hm_qpgf_d2_v2, d3_qpgf_d2.c:178-230 with
// :321-345, 440-466, 887-1044, 2011-2399).  The method choice, lattice reduction and split
// parameter are those of qpgf_eval; the terms, their order (rows outward from the centre row,
// centre term then each side) and the stop rules are the reference's v2 rules: the real-space and
// Ewald spectral sums stop on d2G_xx and d2G_yy, the Fourier-domain sum on d2G_zz.  A plain form
// (one term at a time, phases by sincos) for field points; the assembly does not use it.
struct QPVal2 {
  cplx G;
  cplx dG[3];
  cplx d2G[6];
};

BEM_HD void qp2_acc(cplx& S, cplx* dS, cplx* d2S, const cplx& F, const cplx* dF, const cplx* d2F)
{
  S += F;
  for (int i = 0; i < 3; i++) dS[i] += dF[i];
  for (int i = 0; i < 6; i++) d2S[i] += d2F[i];
}

// Ewald real-space term (d3_qpgf_d2.c:2157-2199); dF[2], d2F[4], d2F[5] still lack the factor z
// that the sum applies at the end.
BEM_HD void qp2_ew1_term(const QPLattice& L, const double* r, double veps, int l1, int l2, cplx& F, cplx* dF, cplx* d2F)
{
  const double R0 = (double)l1 * L.d1x + (double)l2 * L.d2x;
  const double R1 = (double)l1 * L.d1y + (double)l2 * L.d2y;
  const double ra0 = r[0] + R0, ra1 = r[1] + R1, ra2 = r[2];
  const double rl = sqrt(ra0 * ra0 + ra1 * ra1 + ra2 * ra2);
  const double i_rl = 1.0 / rl, i_rl2 = i_rl * i_rl;
  const double ke = L.k * veps, i_ve = 1.0 / veps, rl_2e = rl * 0.5 * i_ve;
  const cplx cef = expi(L.vkx * R0 + L.vky * R1) * exp(ke * ke - rl_2e * rl_2e);
  const cplx w = faddeeva_w(ke, rl_2e);
  const cplx cf1 = cef * (i_rl2 * (i_rl * w.re - L.k * w.im + i_ve * QP_INV_SQRTPI));
  const cplx cf2 = cef * (i_rl2 * (L.k * L.k * i_rl * 2.0 * w.re - i_ve * i_ve * i_ve * QP_INV_SQRTPI));
  const cplx cf3 = cf1 * (-6.0 * i_rl2) + cf2;
  F = cef * (i_rl * w.re);
  dF[0] = cf1 * ra0; dF[1] = cf1 * ra1; dF[2] = cf1;
  d2F[0] = 2.0 * cf1 + cf3 * (ra0 * ra0);
  d2F[1] = 2.0 * cf1 + cf3 * (ra1 * ra1);
  d2F[2] = 2.0 * cf1 + cf3 * (ra2 * ra2);
  d2F[3] = cf3 * (ra0 * ra1);
  d2F[4] = cf3 * ra1;
  d2F[5] = cf3 * ra0;
}

// Ewald spectral term (d3_qpgf_d2.c:2343-2399): 0 propagating, 1 evanescent, -3 beta_n == 0.
BEM_HD int qp2_ew2_term(const QPLattice& L, const double* r, double veps, int n1, int n2, cplx& F, cplx* dF, cplx* d2F)
{
  const double an0 = -L.vkx + (double)n1 * L.g1x + (double)n2 * L.g2x;
  const double an1 = -L.vky + (double)n1 * L.g1y + (double)n2 * L.g2y;
  const double bn2 = L.k * L.k - an0 * an0 - an1 * an1;
  const cplx ce = expi(an0 * r[0] + an1 * r[1]);
  const double azve = r[2] / (2.0 * veps);
  const double ef = exp(bn2 * veps * veps - azve * azve);
  const double c2 = 2.0 * QP_INV_SQRTPI / veps * ef;
  int e;
  cplx Fc, Gc, d2z;
  if (bn2 > 0.0) {
    const double bn = sqrt(bn2);
    const cplx ff = expi(bn * r[2]);
    const cplx w = faddeeva_w(bn * veps, azve);
    Fc = mk(2.0 * ff.re, 2.0 * (ef * w.im + ff.im));   // 2 (i ef Im w + ff)
    Gc = mk(2.0 * (ef * w.re - ff.re), -2.0 * ff.im);  // 2 (ef Re w - ff)
    F = (ce * (1.0 / bn)) * Fc;
    d2z = mul_i(Fc) * bn + mk(c2, 0.0);
    e = 0;
  } else if (bn2 < 0.0) {
    const double bn = sqrt(-bn2);
    const double ebz = exp(bn * r[2]);
    const double f1 = ebz * erfc(bn * veps + azve), f2 = erfc(bn * veps - azve) / ebz;
    Fc = mk(f1 + f2, 0.0);
    Gc = mk(f1 - f2, 0.0);
    F = mul_mi(ce * ((f1 + f2) / bn));
    d2z = mk(-bn * (f1 + f2) + c2, 0.0);
    e = 1;
  } else {
    return -3;
  }
  dF[0] = F * an0; dF[1] = F * an1; dF[2] = ce * Gc;
  d2F[0] = dF[0] * an0; d2F[1] = dF[1] * an1; d2F[2] = ce * d2z;
  d2F[3] = dF[0] * an1; d2F[4] = dF[2] * an1; d2F[5] = dF[2] * an0;
  return e;
}

// Fourier-domain term (d3_qpgf_d2.c:1010-1044): 0 propagating, 1 evanescent, -2 beta_n == 0.
BEM_HD int qp2_fd_term(const QPLattice& L, const double* r, int n1, int n2, cplx& F, cplx* dF, cplx* d2F)
{
  const double an0 = -L.vkx + (double)n1 * L.g1x + (double)n2 * L.g2x;
  const double an1 = -L.vky + (double)n1 * L.g1y + (double)n2 * L.g2y;
  const double bn2 = L.k * L.k - an0 * an0 - an1 * an1;
  int e;
  if (bn2 > 0.0) {
    const double bn = sqrt(bn2);
    dF[2] = expi(an0 * r[0] + an1 * r[1] + bn * fabs(r[2]));
    F = dF[2] * (1.0 / bn);
    e = 0;
  } else if (bn2 < 0.0) {
    const double bn = sqrt(-bn2);
    dF[2] = expi(an0 * r[0] + an1 * r[1]) * exp(-bn * fabs(r[2]));
    F = mul_mi(dF[2] * (1.0 / bn));
    e = 1;
  } else {
    return -2;
  }
  dF[0] = F * an0; dF[1] = F * an1;
  d2F[0] = dF[0] * an0; d2F[1] = dF[1] * an1; d2F[2] = F * bn2;
  d2F[3] = dF[1] * an0; d2F[4] = dF[2] * an1; d2F[5] = dF[2] * an0;
  return e;
}

// Ewald real-space sum (d3_qpgf_d2.c:2053-2155).  Returns the number of terms or -1.
BEM_HD int qp2_ew1_sum(const QPLattice& L, const double* r, double veps, double eps, cplx& S, cplx* dS, cplx* d2S)
{
  S = mk(0, 0);
  for (int i = 0; i < 3; i++) dS[i] = mk(0, 0);
  for (int i = 0; i < 6; i++) d2S[i] = mk(0, 0);
  int cc = 0;
  cplx F, dF[3], d2F[6];
  for (int dir = 0; dir < 3; dir++) {
    const int step = (dir == 2) ? -1 : 1;
    int l1 = (dir == 0) ? 0 : step;
    for (;; l1 += step) {
      if (dir != 0 && (l1 >= QP_EW_LIMIT || l1 <= -QP_EW_LIMIT)) return -1;
      const cplx o0 = d2S[0], o1 = d2S[1];
      const int lc = -(int)round(((r[0] + (double)l1 * L.d1x) * L.d2x + (r[1] + (double)l1 * L.d1y) * L.d2y) / L.ad22);
      qp2_ew1_term(L, r, veps, l1, lc, F, dF, d2F);
      qp2_acc(S, dS, d2S, F, dF, d2F);
      cc++;
      for (int side = 1; side >= -1; side -= 2) {
        int off = 1;
        for (; off < QP_EW_LIMIT; off++) {
          qp2_ew1_term(L, r, veps, l1, lc + side * off, F, dF, d2F);
          qp2_acc(S, dS, d2S, F, dF, d2F);
          cc++;
          if (qp_diff(d2F[0], d2S[0], eps) && qp_diff(d2F[1], d2S[1], eps)) break;
        }
        if (off == QP_EW_LIMIT) return -1;
      }
      if (dir == 0) break;
      if (qp_comp(d2S[0], o0, eps) && qp_comp(d2S[1], o1, eps)) break;
    }
  }
  const double f4p = 4.0 * QP_PI, f8p = 8.0 * QP_PI;
  S = S * (1.0 / f4p);
  dS[0] = dS[0] * (-1.0 / f4p); dS[1] = dS[1] * (-1.0 / f4p); dS[2] = dS[2] * (-r[2] / f4p);
  for (int i = 0; i < 4; i++) d2S[i] = d2S[i] * (-1.0 / f8p);
  d2S[4] = d2S[4] * (-r[2] / f8p); d2S[5] = d2S[5] * (-r[2] / f8p);
  return cc;
}

// Spectral sums.  FD == 0: Ewald spectral (d3_qpgf_d2.c:2201-2341; returns terms or -2 / -3);
// FD == 1: Fourier domain (d3_qpgf_d2.c:887-1008; terms or -1 / -2 / -4).
template <int FD>
BEM_HD int qp2_spec_sum(const QPLattice& L, const double* r, double veps, double eps, cplx& S, cplx* dS, cplx* d2S)
{
  if (FD && r[2] == 0.0) return -4;
  const int LIMIT = FD ? QP_FD_LIMIT : QP_EW_LIMIT;
  const int ELIM = FD ? -1 : -2;
  S = mk(0, 0);
  for (int i = 0; i < 3; i++) dS[i] = mk(0, 0);
  for (int i = 0; i < 6; i++) d2S[i] = mk(0, 0);
  const int nc = L.nc1;
  int cc = 0;
  cplx F, dF[3], d2F[6];
  for (int dir = 0; dir < 3; dir++) {
    const int step = (dir == 2) ? -1 : 1;
    int n1 = nc + ((dir == 0) ? 0 : step);
    for (;; n1 += step) {
      if (dir != 0 && (n1 - nc >= LIMIT || n1 - nc <= -LIMIT)) return ELIM;
      const cplx o0 = d2S[0], o1 = d2S[1], o2 = d2S[2];
      int nc2;
      if (FD) nc2 = (int)round((L.vkx * L.g2x + L.vky * L.g2y - (double)n1 * L.g12) / L.g22);
      else nc2 = (int)round(-((-L.vkx + (double)n1 * L.g1x) * L.g2x + (-L.vky + (double)n1 * L.g1y) * L.g2y) / L.g22);
      int e = FD ? qp2_fd_term(L, r, n1, nc2, F, dF, d2F) : qp2_ew2_term(L, r, veps, n1, nc2, F, dF, d2F);
      if (e < 0) return e;
      qp2_acc(S, dS, d2S, F, dF, d2F);
      cc++;
      int flg = 0;
      for (int side = 1; side >= -1; side -= 2) {
        int off = 1;
        for (; off < LIMIT; off++) {
          e = FD ? qp2_fd_term(L, r, n1, nc2 + side * off, F, dF, d2F)
                 : qp2_ew2_term(L, r, veps, n1, nc2 + side * off, F, dF, d2F);
          if (e < 0) return e;
          qp2_acc(S, dS, d2S, F, dF, d2F);
          cc++;
          if (e > 0) {
            if (FD ? qp_diff(d2F[2], d2S[2], eps) : (qp_diff(d2F[0], d2S[0], eps) && qp_diff(d2F[1], d2S[1], eps))) break;
          } else {
            flg++;
          }
        }
        if (off == LIMIT) return ELIM;
      }
      if (dir == 0) break;
      if (FD) {
        if (qp_comp(d2S[2], o2, eps)) break;
      } else if (flg == 0 && qp_comp(d2S[0], o0, eps) && qp_comp(d2S[1], o1, eps)) {
        break;
      }
    }
  }
  const double aidd = fabs(L.idd);
  if (FD) {
    const double sgnz = r[2] / fabs(r[2]), c = 0.5 * aidd;
    S = mul_i(S * c);
    dS[0] = dS[0] * -c; dS[1] = dS[1] * -c; dS[2] = dS[2] * (-c * sgnz);
    for (int i = 0; i < 4; i++) d2S[i] = mul_i(d2S[i] * -c);
    d2S[4] = mul_i(d2S[4] * (-c * sgnz)); d2S[5] = mul_i(d2S[5] * (-c * sgnz));
  } else {
    const double cd = 0.25 * aidd;
    S = mul_i(S * cd);
    dS[0] = dS[0] * -cd; dS[1] = dS[1] * -cd; dS[2] = dS[2] * cd;
    d2S[0] = mul_i(d2S[0] * -cd); d2S[1] = mul_i(d2S[1] * -cd); d2S[2] = d2S[2] * -cd;
    d2S[3] = mul_i(d2S[3] * -cd); d2S[4] = mul_i(d2S[4] * cd); d2S[5] = mul_i(d2S[5] * cd);
  }
  return cc;
}

// G, grad G and d2G at r_in.  Return value as d3hm_qpgf_d2_v2: > 0 terms; -11..-14 FD errors,
// -21..-24 EW errors.
BEM_HD int qpgf_eval2(const QPLattice& L, const double* r_in, QPVal2& out)
{
  const double eps = QP_MEPS;
  const int l1 = (int)floor((r_in[0] * L.d2y - r_in[1] * L.d2x) * L.idd + 0.5);
  const int l2 = (int)floor(-(r_in[0] * L.d1y - r_in[1] * L.d1x) * L.idd + 0.5);
  double r[3];
  r[0] = r_in[0] - (double)l1 * L.d1x - (double)l2 * L.d2x;
  r[1] = r_in[1] - (double)l1 * L.d1y - (double)l2 * L.d2y;
  r[2] = r_in[2];
  bool use_fd = false;
  if (!L.ew_only)
    use_fd = (L.bN / L.bNp * exp(-L.bNp * fabs(r[2])) < eps) && (L.bN / L.bNm * exp(-L.bNm * fabs(r[2])) < eps);
  int err;
  if (use_fd) {
    err = qp2_spec_sum<1>(L, r, 0.0, eps, out.G, out.dG, out.d2G);
    if (err < 0) return err - 10;
  } else {
    double veps = L.veps0;
    const double r2_min = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    if (L.k * L.k * veps * veps - r2_min / (4.0 * veps * veps) > QP_EW_EXPM)
      veps = sqrt(QP_EW_EXPM + sqrt(L.k * L.k * r2_min + QP_EW_EXPM * QP_EW_EXPM)) / (sqrt(2.0) * L.k);
    const int c1 = qp2_ew1_sum(L, r, veps, eps, out.G, out.dG, out.d2G);
    if (c1 < 0) return c1 - 20;
    cplx S2, dS2[3], d2S2[6];
    const int c2 = qp2_spec_sum<0>(L, r, veps, eps, S2, dS2, d2S2);
    if (c2 < 0) return c2 - 20;
    qp2_acc(out.G, out.dG, out.d2G, S2, dS2, d2S2);
    err = c1 + c2;
  }
  if (l1 != 0 || l2 != 0) {
    const cplx cf = expi(-(L.vkx * ((double)l1 * L.d1x + (double)l2 * L.d2x) + L.vky * ((double)l1 * L.d1y + (double)l2 * L.d2y)));
    out.G = out.G * cf;
    for (int i = 0; i < 3; i++) out.dG[i] = out.dG[i] * cf;
    for (int i = 0; i < 6; i++) out.d2G[i] = out.d2G[i] * cf;
  }
  return err;
}

// Lattice constants, following d3_qpgf_d2.c:129-155 (selection), :1680-1685 (split parameter)
// and :1848-1857 (reciprocal vectors) expression by expression.
BEM_HD int qp_lattice_init(QPLattice& L, double k, double vkx, double vky, double d1x, double d1y, double d2x, double d2y)
{
  L.k = k; L.vkx = vkx; L.vky = vky;
  L.d1x = d1x; L.d1y = d1y; L.d2x = d2x; L.d2y = d2y;
  L.detd = d1x * d2y - d2x * d1y;
  if (L.detd == 0.0) return -1;
  L.idd = 1.0 / L.detd;
  double ad12 = d1x * d1x + d1y * d1y;
  L.ad22 = d2x * d2x + d2y * d2y;
  L.g1x = 2.0 * QP_PI * L.idd * d2y;
  L.g1y = -2.0 * QP_PI * L.idd * d2x;
  L.g2x = -2.0 * QP_PI * L.idd * d1y;
  L.g2y = 2.0 * QP_PI * L.idd * d1x;
  L.g22 = L.g2x * L.g2x + L.g2y * L.g2y;
  L.g12 = L.g1x * L.g2x + L.g1y * L.g2y;
  double adp = sqrt(pow(d1x + d2x, 2) + pow(d1y + d2y, 2));
  double adm = sqrt(pow(d1x - d2x, 2) + pow(d1y - d2y, 2));
  L.veps0 = sqrt(fabs(L.detd) / (4.0 * QP_PI) * adp / adm);
  // method selection constants
  double k2 = k * k, cpd = 2.0 * QP_PI * L.idd;
  int n1 = (int)round((vkx * d1x + vky * d1y) / (2.0 * QP_PI));
  int n2 = (int)round((vkx * d2x + vky * d2y) / (2.0 * QP_PI));
  double aNx = -vkx + (double)n1 * cpd * d2y - (double)n2 * cpd * d1y;
  double aNy = -vky - (double)n1 * cpd * d2x + (double)n2 * cpd * d1x;
  L.bN = sqrt(k2 - aNx * aNx - aNy * aNy);
  double aNpx, aNpy, aNmx, aNmy;
  if (L.ad22 < ad12) {
    aNpx = -vkx + (double)(n1 + QP_S_LIMIT) * cpd * d2y - (double)n2 * cpd * d1y;
    aNpy = -vky - (double)(n1 + QP_S_LIMIT) * cpd * d2x + (double)n2 * cpd * d1x;
    aNmx = -vkx + (double)(n1 - QP_S_LIMIT) * cpd * d2y - (double)n2 * cpd * d1y;
    aNmy = -vky - (double)(n1 - QP_S_LIMIT) * cpd * d2x + (double)n2 * cpd * d1x;
  } else {
    aNpx = -vkx + (double)n1 * cpd * d2y - (double)(n2 + QP_S_LIMIT) * cpd * d1y;
    aNpy = -vky - (double)n1 * cpd * d2x + (double)(n2 + QP_S_LIMIT) * cpd * d1x;
    aNmx = -vkx + (double)n1 * cpd * d2y - (double)(n2 - QP_S_LIMIT) * cpd * d1y;
    aNmy = -vky - (double)n1 * cpd * d2x + (double)(n2 - QP_S_LIMIT) * cpd * d1x;
  }
  double bNp = k2 - aNpx * aNpx - aNpy * aNpy;
  double bNm = k2 - aNmx * aNmx - aNmy * aNmy;
  if (bNp > 0.0 || bNm > 0.0) {
    L.ew_only = 1;
    L.bNp = 0.0; L.bNm = 0.0;
  } else {
    L.ew_only = 0;
    L.bNp = sqrt(-bNp);
    L.bNm = sqrt(-bNm);
  }
  L.nc1 = n1;
  L.eb2 = expi(vkx * d2x + vky * d2y);
  L.prop = nullptr;
  L.nprop = -1;
  return 0;
}

// The propagating orders of a lattice in (n1, n2) order, with the term functions' expressions
// for a_n and beta_n^2, over the window the row walks can reach (|n1 - nc1| < QP_EW_LIMIT, n2
// within QP_EW_LIMIT of the row centre).  Returns their number, or -1 if more than cap.
BEM_HD int qp_prop_list(const QPLattice& L, QPProp* out, int cap)
{
  int n = 0;
  for (int n1 = L.nc1 - QP_EW_LIMIT + 1; n1 < L.nc1 + QP_EW_LIMIT; n1++) {
    const int nc2 = (int)round(-((-L.vkx + (double)n1 * L.g1x) * L.g2x + (-L.vky + (double)n1 * L.g1y) * L.g2y) / L.g22);
    for (int n2 = nc2 - QP_EW_LIMIT - 1; n2 <= nc2 + QP_EW_LIMIT + 1; n2++) {
      const double an0 = -L.vkx + (double)n1 * L.g1x + (double)n2 * L.g2x;
      const double an1 = -L.vky + (double)n1 * L.g1y + (double)n2 * L.g2y;
      const double bn2 = L.k * L.k - an0 * an0 - an1 * an1;
      if (bn2 > 0.0) {
        if (n >= cap) return -1;
        out[n].an0 = an0; out[n].an1 = an1; out[n].bn2 = bn2; out[n].bn = sqrt(bn2);
        n++;
      }
    }
  }
  return n;
}

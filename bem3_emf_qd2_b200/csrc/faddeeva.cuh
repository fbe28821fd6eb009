// faddeeva.cuh -- the Faddeeva function w(z) = exp(-z^2) erfc(-i z) in FP64, host+device.
//
// Replaces Faddeeva_w (qgf2_src/Faddeeva.cc:679-, S. G. Johnson's MIT package vendored by the
// reference) on the QPGF hot path (qgf2_src/d3_qpgf_d2.c:1831,1982 and their qG/dqG twins).
// This is an independent implementation from the published mathematics, not a port:
//
//  * |z| >= 8, Im z >= 0: the Laplace continued fraction
//        w(z) = (i/sqrt(pi)) / (z - (1/2)/(z - 1/(z - (3/2)/(z - ...))))
//    evaluated bottom-up at a fixed depth (20 levels, chosen by measurement against
//    mpmath at 40 digits: component-wise relative error < 1e-15 for |z| >= 8).
//  * |z| < 0.5: the Maclaurin series w(z) = sum_n (i z)^n / Gamma(n/2 + 1), 24 terms.
//  * otherwise, Im z >= 0: the trapezoidal rule with pole correction for the integral
//        w(z) = (i/pi) \int e^{-t^2} / (z - t) dt            (Im z > 0)
//    with step h = 0.42 (aliasing error ~ exp(-pi^2/h^2) ~ 5e-25).  With nodes t_n = n h:
//        w(z) = (i h / pi) sum_n e^{-t_n^2}/(z - t_n) + 2 e^{-z^2} / (1 - e^{-2 pi i z/h}),
//    and with the half-shifted nodes t_n = (n + 1/2) h the pole term's denominator becomes
//    1 + e^{-2 pi i z/h}.  The node set whose nodes lie farther from Re z is used, so the
//    node term and the pole term never nearly cancel.  Symmetric pairing gives
//        sum_n e^{-t_n^2}/(z - t_n) = sum_{t_n >= 0} c_n 2z/(z^2 - t_n^2)  (+ 1/z for t_0 = 0).
//    (Chiarella & Reichel 1968; the same construction underlies Zaghloul & Ali, ACM TOMS
//    Algorithm 916, 2011.)
//  * Im z < 0: reflection w(z) = 2 exp(-z^2) - w(-z).
// The weights e^{-t_n^2} below were computed with mpmath at 40 digits for h = 0.42.
//
// The assembly kernels' form (FAST) replaces the series and the trapezoidal rule (|z| < 8) by
// Weideman's rational approximation (SIAM J. Numer. Anal. 31 (1994) 1497-1518), a polynomial of
// degree 39 in Z = (L + iz)/(L - iz) times 1/(L - iz)^2 plus pi^{-1/2}/(L - iz): one complex
// reciprocal and 39 complex multiply-adds, no branch inside the disk (coefficients in
// faddeeva_weideman.h, generated by gen_faddeeva_weideman.py), and the continued fraction in its
// single-division (Wallis) form for |z| >= 8.
#pragma once

#include "cplx.cuh"

#if defined(__CUDACC__)
#define BEM_CONST __device__ __constant__
#else
#define BEM_CONST static const
#endif

#include "faddeeva_weideman.h"

#define FAD_NFULL 18
#define FAD_NHALF 17

BEM_CONST double fad_cfull[FAD_NFULL] = {
    1.0, 8.3828260322423347594e-1, 4.9381219803334612553e-1, 2.0441562097826399655e-1,
    5.9463059974303169775e-2, 1.2155178329914937215e-2, 1.7460485771277553444e-3,
    1.7625125424738445977e-4, 1.2502274127541389562e-5, 6.2319896697822480818e-7,
    2.1829577951254792091e-8, 5.3733466674381974499e-10, 9.294484093066937156e-12,
    1.1297611163578632306e-13, 9.6500344752061033519e-16, 5.7923128853948579235e-18,
    2.4431833970432752826e-20, 7.2417083525696746133e-23};
BEM_CONST double fad_tfull[FAD_NFULL] = {  // (n h)^2
    0.0, 1.764e-1, 7.056e-1, 1.5876, 2.8224, 4.41, 6.3504, 8.6436, 1.12896e+1, 1.42884e+1,
    1.764e+1, 2.13444e+1, 2.54016e+1, 2.98116e+1, 3.45744e+1, 3.969e+1, 4.51584e+1, 5.09796e+1};
BEM_CONST double fad_chalf[FAD_NHALF] = {
    9.5685826686190967266e-1, 6.7240126239700272678e-1, 3.3203994534466064202e-1,
    1.1522137512179343879e-1, 2.8096788427793083622e-2, 4.814611126123969182e-3,
    5.7975787411862236613e-4, 4.9058357456207695791e-5, 2.9171600516592813046e-6,
    1.2189570925149132158e-7, 3.5792949402287995251e-9, 7.3856285415805615869e-11,
    1.0709232382508076456e-12, 1.0912145063014343686e-14, 7.813449790825644105e-17,
    3.9314832299765398667e-19, 1.3901156607797321885e-21};
BEM_CONST double fad_thalf[FAD_NHALF] = {  // ((n + 1/2) h)^2
    4.41e-2, 3.969e-1, 1.1025, 2.1609, 3.5721, 5.3361, 7.4529, 9.9225, 1.27449e+1, 1.59201e+1,
    1.94481e+1, 2.33289e+1, 2.75625e+1, 3.21489e+1, 3.70881e+1, 4.23801e+1, 4.80249e+1};
BEM_CONST double fad_taylor[24] = {  // 1 / Gamma(n/2 + 1)
    1.0, 1.1283791670955125739, 1.0, 7.5225277806367504926e-1, 5.0e-1, 3.0090111122547001971e-1,
    1.6666666666666666667e-1, 8.597174606442000563e-2, 4.1666666666666666667e-2,
    1.9104832458760001251e-2, 8.3333333333333333333e-3, 3.4736059015927275002e-3,
    1.3888888888888888889e-3, 5.3440090793734269234e-4, 1.984126984126984127e-4,
    7.1253454391645692312e-5, 2.4801587301587301587e-5, 8.3827593401936108602e-6,
    2.7557319223985890653e-6, 8.8239572002038009055e-7, 2.7557319223985890653e-7,
    8.4037687620988580052e-8, 2.5052108385441718775e-8, 7.3076250105207460915e-9};

#define FAD_H 0.42
#define FAD_TWOPI_OVER_H 1.4959965017094253516e+1
#define FAD_H_OVER_PI 1.3369015219719208205e-1
#define FAD_INV_SQRTPI 5.6418958354775628695e-1

#if defined(BEM_TERM_STATS) && !defined(__CUDACC__)
// host-only instrumentation for the term-mix study (never defined in the CUDA library build)
extern unsigned long long bem_stat_w[3];
#define BEM_STAT_W(i) (bem_stat_w[i]++)
#else
#define BEM_STAT_W(i) ((void)0)
#endif

// w(z) for Im z >= 0 (upper half plane incl. the real axis).  Kept out of line and not unrolled:
// one small copy serves every call site, which keeps the lattice-sum kernels inside the
// instruction cache.
// Complex reciprocal with one real division.  The denominators met below are well scaled
// (|t| >= 8 in the continued fraction; |z^2 - t_n| bounded away from 0 and from overflow by the
// node choice), so Smith's scaling is not needed there; the result differs from crecip in the
// last bits only.
BEM_HD cplx crecip_fast(cplx b)
{
  const double d = 1.0 / (b.re * b.re + b.im * b.im);
  return mk(b.re * d, -b.im * d);
}

// FAST selects crecip_fast for the reciprocals of the continued fraction and of the node sum.
// Inline by default: out of line, every call from a lattice-sum loop made the loop save and restore
// its live sums in local memory (measured 12-14 % slower on the assembly kernel).
#if defined(FAD_W_NOINLINE)
#define FAD_W_FN BEM_HD_NOINLINE
#else
#define FAD_W_FN BEM_HD
#endif
template <bool FAST>
FAD_W_FN cplx faddeeva_w_upper_t(double x, double y)
{
  const double r2 = x * x + y * y;
  if (FAST && r2 < 64.0) {
    BEM_STAT_W(1);
    const cplx il = crecip_fast(mk(FAD_WL + y, -x));  // 1 / (L - i z); |L - i z| >= L
    const cplx Z = mk(FAD_WL - y, x) * il;           // (L + i z) / (L - i z)
    double pr = fad_wc[0], pi = 0.0;
#pragma unroll
    for (int n = 1; n < FAD_WN; n++) {
      const double t = pr * Z.re - pi * Z.im + fad_wc[n];
      pi = pr * Z.im + pi * Z.re;
      pr = t;
    }
    return (mk(2.0 * pr, 2.0 * pi) * il + mk(FAD_INV_SQRTPI, 0.0)) * il;
  }
  if (FAST && r2 >= 64.0 && r2 < 1.0e8) {
    BEM_STAT_W(0);
    // the same 20-level continued fraction by the forward (Wallis) recurrence of its numerators
    // and denominators: f = A_20 / B_20 with A_k = z A_{k-1} - (k/2) A_{k-2} (B likewise), one
    // division in all.  |A_k| ~ |z|^k stays far from overflow for |z| < 1e4.
    const cplx z = mk(x, y);
    cplx Am = mk(1.0, 0.0), A = z, Bm = mk(0.0, 0.0), B = mk(1.0, 0.0);
#pragma unroll 1
    for (int k = 1; k <= 20; k++) {
      const double a = -0.5 * k;
      const cplx An = z * A + a * Am, Bn = z * B + a * Bm;
      Am = A; A = An; Bm = B; B = Bn;
    }
    const cplx q = B * crecip_fast(A);  // 1 / f
    return mk(-FAD_INV_SQRTPI * q.im, FAD_INV_SQRTPI * q.re);
  }
  if (r2 >= 64.0) {
    BEM_STAT_W(0);
    // continued fraction, 20 levels, bottom-up
    cplx z = mk(x, y);
    cplx t = z;
#pragma unroll 1
    for (int n = 20; n >= 1; n--) t = z - (0.5 * n) * (FAST ? crecip_fast(t) : crecip(t));
    cplx q = FAST ? crecip_fast(t) : crecip(t);
    return mk(-FAD_INV_SQRTPI * q.im, FAD_INV_SQRTPI * q.re);  // i q / sqrt(pi)
  }
  if (r2 < 0.25) {
    BEM_STAT_W(1);
    // Maclaurin series in (i z), Horner form
    cplx iz = mk(-y, x);
    cplx s = mk(fad_taylor[23], 0.0);
#pragma unroll 1
    for (int n = 22; n >= 0; n--) s = s * iz + mk(fad_taylor[n], 0.0);
    return s;
  }
  BEM_STAT_W(2);
  // trapezoid + pole correction; pick the node set farther from x
  const double u = fabs(x) * (1.0 / FAD_H);
  const double frac = u - floor(u);
  const bool use_full = fmin(frac, 1.0 - frac) >= fabs(frac - 0.5);
  const cplx z = mk(x, y);
  const cplx z2 = z * z;
  cplx s = mk(0.0, 0.0);
  if (FAST) {
    // the node sum two terms at a time over a common denominator:
    //   c_a/(w - t_a) + c_b/(w - t_b) = ((c_a + c_b) w - (c_a t_b + c_b t_a)) / (w^2 - (t_a + t_b) w + t_a t_b)
    // (w = z^2), one division per pair
    const double* c = use_full ? fad_cfull : fad_chalf;
    const double* tt = use_full ? fad_tfull : fad_thalf;
    const int lo = use_full ? 1 : 0;
    const int hi = use_full ? FAD_NFULL - 1 : FAD_NHALF - 1;
    const cplx w2 = z2 * z2;
    int n = hi;
#pragma unroll 1
    for (; n - 1 >= lo; n -= 2) {
      const double ca = c[n], cb = c[n - 1], ta = tt[n], tb = tt[n - 1];
      const cplx D = mk(w2.re - (ta + tb) * z2.re + ta * tb, w2.im - (ta + tb) * z2.im);
      const cplx N = mk((ca + cb) * z2.re - (ca * tb + cb * ta), (ca + cb) * z2.im);
      s += N * crecip_fast(D);
    }
    if (n >= lo) s += c[n] * crecip_fast(mk(z2.re - tt[n], z2.im));
    s = use_full ? (2.0 * s) * z + crecip_fast(z) : (2.0 * s) * z;
  } else if (use_full) {
#pragma unroll 1
    for (int n = FAD_NFULL - 1; n >= 1; n--) {
      const cplx d = mk(z2.re - fad_tfull[n], z2.im);
      s += fad_cfull[n] * (FAST ? crecip_fast(d) : crecip(d));
    }
    s = (2.0 * s) * z + (FAST ? crecip_fast(z) : crecip(z));
  } else {
#pragma unroll 1
    for (int n = FAD_NHALF - 1; n >= 0; n--) {
      const cplx d = mk(z2.re - fad_thalf[n], z2.im);
      s += fad_chalf[n] * (FAST ? crecip_fast(d) : crecip(d));
    }
    s = (2.0 * s) * z;
  }
  // (i h / pi) * s
  cplx w = mk(-FAD_H_OVER_PI * s.im, FAD_H_OVER_PI * s.re);
  // pole term 2 e^{-z^2} / (1 -+ e^{-2 pi i z / h})
  cplx ez2 = cexp_(mk(-z2.re, -z2.im));
  cplx E = cexp_(mk(FAD_TWOPI_OVER_H * y, -FAD_TWOPI_OVER_H * x));
  cplx den = use_full ? mk(1.0 - E.re, -E.im) : mk(1.0 + E.re, E.im);
  w += cdiv(2.0 * ez2, den);
  return w;
}

BEM_HD cplx faddeeva_w_upper(double x, double y) { return faddeeva_w_upper_t<false>(x, y); }

// w(z) ~ (i / (sqrt(pi) z)) (1 + 1/(2 z^2) + 3/(4 z^4) + 15/(8 z^6) + 105/(16 z^8)), the first five
// terms of the asymptotic series: relative error below 2e-4 for |z| >= 3.3 with arg z in
// [pi/4, pi/2) (checked against scipy.special.wofz).  For terms whose size only has to be known to
// a few digits (the lattice sums use it where a term cannot reach 1e-16 of the running sum).
BEM_HD cplx faddeeva_w_asym(double x, double y)
{
  const cplx iz = crecip_fast(mk(x, y));
  const cplx u = iz * iz;
  cplx s = mk(6.5625, 0.0) * u + mk(1.875, 0.0);
  s = s * u + mk(0.75, 0.0);
  s = s * u + mk(0.5, 0.0);
  s = s * u + mk(1.0, 0.0);
  return mul_i(iz * s) * FAD_INV_SQRTPI;
}

// w(z) on the whole plane.
template <bool FAST>
BEM_HD cplx faddeeva_w_t(double x, double y)
{
  if (y >= 0.0) return faddeeva_w_upper_t<FAST>(x, y);
  cplx wm = faddeeva_w_upper_t<FAST>(-x, -y);
  cplx e = cexp_(mk(y * y - x * x, -2.0 * x * y));  // e^{-z^2}
  return mk(2.0 * e.re - wm.re, 2.0 * e.im - wm.im);
}
BEM_HD cplx faddeeva_w(double x, double y) { return faddeeva_w_t<false>(x, y); }

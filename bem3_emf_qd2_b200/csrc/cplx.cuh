// cplx.cuh -- minimal FP64 complex arithmetic usable from host and device code.
//
// The kernels keep every complex value in a pair of registers; this struct is the only
// complex type on the hot path (no cuComplex / thrust / std::complex), so the same
// arithmetic compiles for sm_100a and, in the host-side math checks, for the CPU.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define BEM_HD __host__ __device__ __forceinline__
#define BEM_HD_NOINLINE __host__ __device__ __noinline__
#else
#define BEM_HD static inline
#define BEM_HD_NOINLINE static
#endif

struct cplx {
  double re, im;
};

BEM_HD cplx mk(double re, double im) { cplx z; z.re = re; z.im = im; return z; }
BEM_HD cplx operator+(cplx a, cplx b) { return mk(a.re + b.re, a.im + b.im); }
BEM_HD cplx operator-(cplx a, cplx b) { return mk(a.re - b.re, a.im - b.im); }
BEM_HD cplx operator-(cplx a) { return mk(-a.re, -a.im); }
BEM_HD cplx operator*(cplx a, cplx b) { return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
BEM_HD cplx operator*(double s, cplx a) { return mk(s * a.re, s * a.im); }
BEM_HD cplx operator*(cplx a, double s) { return mk(s * a.re, s * a.im); }
BEM_HD cplx& operator+=(cplx& a, cplx b) { a.re += b.re; a.im += b.im; return a; }
BEM_HD cplx& operator-=(cplx& a, cplx b) { a.re -= b.re; a.im -= b.im; return a; }
BEM_HD cplx& operator*=(cplx& a, double s) { a.re *= s; a.im *= s; return a; }
BEM_HD cplx& operator*=(cplx& a, cplx b) { a = a * b; return a; }
BEM_HD cplx conj(cplx a) { return mk(a.re, -a.im); }
BEM_HD double abs2(cplx a) { return a.re * a.re + a.im * a.im; }
BEM_HD cplx mul_i(cplx a) { return mk(-a.im, a.re); }     // i*a
BEM_HD cplx mul_mi(cplx a) { return mk(a.im, -a.re); }    // -i*a
BEM_HD cplx cdiv(cplx a, cplx b) {
  // Smith's algorithm keeps the quotient accurate when |b| spans a wide range.
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re, d = b.re + b.im * r;
    return mk((a.re + a.im * r) / d, (a.im - a.re * r) / d);
  } else {
    double r = b.re / b.im, d = b.im + b.re * r;
    return mk((a.re * r + a.im) / d, (a.im * r - a.re) / d);
  }
}
BEM_HD cplx crecip(cplx b) { return cdiv(mk(1.0, 0.0), b); }
BEM_HD cplx expi(double a) {  // e^{i a}
  double s, c;
#if defined(__CUDA_ARCH__)
  sincos(a, &s, &c);
#else
  s = sin(a); c = cos(a);
#endif
  return mk(c, s);
}
BEM_HD double rsqrt_(double x) {  // 1/sqrt(x)
#if defined(__CUDA_ARCH__)
  return rsqrt(x);
#else
  return 1.0 / sqrt(x);
#endif
}
BEM_HD cplx cexp_(cplx z) {  // e^{z}
  double e = exp(z.re);
  cplx p = expi(z.im);
  return mk(e * p.re, e * p.im);
}

/*
 * opcount.cpp -- MEASUREMENT INFRASTRUCTURE ONLY (the roofline's numerator, never the product path).
 *
 * Algorithmic FP64 operation counts of the quasi-periodic Green's function as the assembly uses it:
 * the lattice sums of qpgf_oracle.c (the plain-C restatement of qgf2_src/d3_qpgf_d2.c, same terms,
 * same loop nests and stop rules) transcribed term for term onto a counting number type `Fl`, so that
 * running them counts every floating-point operation the algorithm performs:
 *   + - * /  and sqrt: one operation each (the IEEE basic operations); a fused multiply-add is not
 *   used; sign changes, fabs and comparisons are not counted.
 * Special functions are charged by executing compact published methods on the same type:
 *   exp       Cody-Waite reduction by ln 2 (two-part constant) and the Taylor polynomial of degree 13
 *   sin, cos  Cody-Waite reduction by pi/2 (three-part constant), Taylor polynomials of degree 17 / 16
 *   erfcx     J. A. C. Weideman, "Computation of the complex error function", SIAM J. Numer. Anal.
 *             31 (1994) 1497-1518: the rational approximation on the imaginary axis, N = 36
 *   erfc      e^{-x^2} erfcx(x) (x >= 0), 2 - erfc(-x) (x < 0)
 *   w(z)      Weideman's approximation, N = 40, upper half plane; 2 e^{-z^2} - w(-z) below
 * (the coefficient tables come from the caller, computed with Weideman's FFT recipe: opcount.py).
 * Each method is checked against the C library by opcount.py before its counts are used.
 *
 * Entry point: oc_point() evaluates G and grad G at one point with either method choice -- the
 * reference's (d3_qpgf_d2.c:124-176) or the assembly kernels' cost rule (Fourier-domain sum only for
 * |z| > zfac x split parameter) -- and returns the value, the number of lattice terms and the
 * operations counted.
 */
#include <math.h>
#include <stdlib.h>

namespace {

unsigned long long g_ops = 0;

struct Fl {
  double v;
  Fl() : v(0.0) {}
  Fl(double x) : v(x) {}
};
inline Fl operator+(Fl a, Fl b) { g_ops++; return Fl(a.v + b.v); }
inline Fl operator-(Fl a, Fl b) { g_ops++; return Fl(a.v - b.v); }
inline Fl operator*(Fl a, Fl b) { g_ops++; return Fl(a.v * b.v); }
inline Fl operator/(Fl a, Fl b) { g_ops++; return Fl(a.v / b.v); }
inline Fl operator-(Fl a) { return Fl(-a.v); }
inline Fl& operator+=(Fl& a, Fl b) { a = a + b; return a; }
inline bool operator<(Fl a, Fl b) { return a.v < b.v; }
inline bool operator>(Fl a, Fl b) { return a.v > b.v; }
inline bool operator<=(Fl a, Fl b) { return a.v <= b.v; }
inline bool operator>=(Fl a, Fl b) { return a.v >= b.v; }
inline Fl fabs_(Fl a) { return Fl(fabs(a.v)); }
inline Fl sqrt_(Fl a) { g_ops++; return Fl(sqrt(a.v)); }

// exp: x = n ln2 + r, |r| <= ln2 / 2, e^r by Horner on the Taylor series to degree 13 (error ~4e-18)
Fl exp_(Fl x)
{
  if (x.v < -745.0) return Fl(0.0);
  const double LN2_HI = 6.93147180369123816490e-01, LN2_LO = 1.90821492927058770002e-10;
  const Fl n = Fl(nearbyint((x * Fl(1.4426950408889634074)).v));  // round: not an arithmetic op
  const Fl r = (x - n * Fl(LN2_HI)) - n * Fl(LN2_LO);
  double c[14];
  c[0] = 1.0;
  for (int i = 1; i < 14; i++) c[i] = c[i - 1] / i;
  Fl p = Fl(c[13]);
  for (int i = 12; i >= 0; i--) p = p * r + Fl(c[i]);
  return Fl(ldexp(p.v, (int)n.v));  // scaling by 2^n: exponent arithmetic, not counted
}

// sin and cos: x = n pi/2 + r, |r| <= pi/4, Taylor polynomials in r^2
void sincos_(Fl x, Fl& s, Fl& c)
{
  const double P1 = 1.5707963267341256e+00, P2 = 6.0771005065061922e-11, P3 = 2.0222662487959506e-21;
  const Fl n = Fl(nearbyint((x * Fl(0.63661977236758134308)).v));
  const Fl r = ((x - n * Fl(P1)) - n * Fl(P2)) - n * Fl(P3);
  const Fl r2 = r * r;
  double fs[9], fc[9];
  for (int i = 0; i < 9; i++) {  // (-1)^i / (2i+1)!, (-1)^i / (2i)!
    double a = 1.0, b = 1.0;
    for (int j = 1; j <= 2 * i + 1; j++) a /= j;
    for (int j = 1; j <= 2 * i; j++) b /= j;
    fs[i] = (i & 1) ? -a : a;
    fc[i] = (i & 1) ? -b : b;
  }
  Fl ps = Fl(fs[8]), pc = Fl(fc[8]);
  for (int i = 7; i >= 0; i--) { ps = ps * r2 + Fl(fs[i]); pc = pc * r2 + Fl(fc[i]); }
  ps = ps * r;
  const int q = ((int)n.v) & 3;
  Fl sv = (q == 0) ? ps : (q == 1) ? pc : (q == 2) ? -ps : -pc;
  Fl cv = (q == 0) ? pc : (q == 1) ? -ps : (q == 2) ? -pc : ps;
  s = sv;
  c = cv;
}

const double* g_ax = nullptr;  // Weideman coefficients, erfcx (N = 36), highest power first
const double* g_aw = nullptr;  // Weideman coefficients, w(z) (N = 40)
double g_Lx = 0.0, g_Lw = 0.0;
const int NX = 36, NW = 40;
const double ISQPI = 5.6418958354775628695e-1;

Fl erfcx_(Fl x)  // x >= 0
{
  const Fl L = Fl(g_Lx);
  const Fl iv = Fl(1.0) / (L + x);
  const Fl Z = (L - x) * iv;
  Fl p = Fl(g_ax[0]);
  for (int i = 1; i < NX; i++) p = p * Z + Fl(g_ax[i]);
  return Fl(2.0) * p * iv * iv + Fl(ISQPI) * iv;
}
Fl erfc_(Fl x)
{
  if (x.v >= 0.0) return exp_(-(x * x)) * erfcx_(x);
  return Fl(2.0) - exp_(-(x * x)) * erfcx_(-x);
}

struct Cx {
  Fl re, im;
  Cx() {}
  Cx(Fl a, Fl b) : re(a), im(b) {}
};
inline Cx operator+(Cx a, Cx b) { return Cx(a.re + b.re, a.im + b.im); }
inline Cx operator-(Cx a, Cx b) { return Cx(a.re - b.re, a.im - b.im); }
inline Cx operator*(Cx a, Cx b) { return Cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
inline Cx operator*(Cx a, Fl b) { return Cx(a.re * b, a.im * b); }
inline Cx operator/(Cx a, Fl b) { return Cx(a.re / b, a.im / b); }
inline Cx operator/(Cx a, Cx b)  // textbook complex division
{
  const Fl d = b.re * b.re + b.im * b.im;
  return Cx((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d);
}
inline Cx& operator+=(Cx& a, Cx b) { a = a + b; return a; }
inline Cx mul_i(Cx a) { return Cx(-a.im, a.re); }  // i a: no arithmetic
inline Cx neg(Cx a) { return Cx(-a.re, -a.im); }
inline Cx cexp_i(Fl t)  // e^{i t}
{
  Fl s, c;
  sincos_(t, s, c);
  return Cx(c, s);
}
inline Cx cexp_(Cx z)
{
  const Fl m = exp_(z.re);
  Fl s, c;
  sincos_(z.im, s, c);
  return Cx(m * c, m * s);
}

Cx w_upper(Cx z)
{
  const Fl L = Fl(g_Lw);
  const Cx den(L + z.im, -z.re);  // L - i z
  const Cx num(L - z.im, z.re);   // L + i z
  const Cx iv = Cx(Fl(1.0), Fl(0.0)) / den;
  const Cx Z = num * iv;
  Cx p(Fl(g_aw[0]), Fl(0.0));
  for (int i = 1; i < NW; i++) {
    p = p * Z;
    p.re = p.re + Fl(g_aw[i]);
  }
  return (p * (iv * iv)) * Fl(2.0) + iv * Fl(ISQPI);
}
Cx w_(Cx z)
{
  if (z.im.v >= 0.0) return w_upper(z);
  const Cx mz(-z.re, -z.im);
  const Cx e = cexp_(Cx(-(z.re * z.re - z.im * z.im), -(Fl(2.0) * z.re * z.im)));
  return e * Fl(2.0) - w_upper(mz);
}

struct Q {
  double k, vk[3], d1[2], d2[2];
};

int same(Cx a, Cx b, double e)
{
  return (Fl(2.0) * fabs_(a.re - b.re) <= Fl(e) * (fabs_(a.re) + fabs_(b.re))) &&
         (Fl(2.0) * fabs_(a.im - b.im) <= Fl(e) * (fabs_(a.im) + fabs_(b.im)));
}
int small(Cx v, Cx s, double e)
{
  return (fabs_(v.re) <= fabs_(s.re) * Fl(0.1) * Fl(e)) && (fabs_(v.im) <= fabs_(s.im) * Fl(0.1) * Fl(e));
}

// per-lattice constants of qpgf_oracle.c (computed once per lattice there too: not per term)
struct Rc {
  double g1[2], g2[2], idd;
};
Rc recip(const Q* q)
{
  Rc c;
  const double det = q->d1[0] * q->d2[1] - q->d2[0] * q->d1[1];
  c.idd = 1.0 / det;
  c.g1[0] = 2 * M_PI * c.idd * q->d2[1];
  c.g1[1] = -2 * M_PI * c.idd * q->d2[0];
  c.g2[0] = -2 * M_PI * c.idd * q->d1[1];
  c.g2[1] = 2 * M_PI * c.idd * q->d1[0];
  return c;
}

// Ewald real-space sum: qpgf_oracle.c or_ew_real, term for term
int ew_real(const Q* q, const Fl* r, Fl ve, double eps, Cx* G, Cx* dG)
{
  int cc = 0;
  const Cx z0(Fl(0.0), Fl(0.0));
  *G = z0; dG[0] = dG[1] = dG[2] = z0;
  const double ad22 = q->d2[0] * q->d2[0] + q->d2[1] * q->d2[1];
  for (int pass = 0; pass < 3; pass++) {
    int l1 = pass == 0 ? 0 : (pass == 1 ? 1 : -1), st = pass == 2 ? -1 : 1;
    for (; abs(l1) < 100; l1 += st) {
      const Cx oG = *G;
      const int lc = -(int)round((((r[0] + Fl(l1 * q->d1[0])) * Fl(q->d2[0]) + (r[1] + Fl(l1 * q->d1[1])) * Fl(q->d2[1])) /
                                  Fl(ad22)).v);
      for (int side = 0; side < 3; side++) {
        int l2 = side == 0 ? lc : (side == 1 ? lc + 1 : lc - 1), s2 = side == 2 ? -1 : 1;
        for (; abs(l2 - lc) < 100; l2 += s2) {
          const Fl R0 = Fl((double)l1) * Fl(q->d1[0]) + Fl((double)l2) * Fl(q->d2[0]);
          const Fl R1 = Fl((double)l1) * Fl(q->d1[1]) + Fl((double)l2) * Fl(q->d2[1]);
          const Fl px = r[0] + R0, py = r[1] + R1;
          const Fl rl = sqrt_(px * px + py * py + r[2] * r[2]);
          const Fl ke = Fl(q->k) * ve, a = rl / (Fl(2.0) * ve);
          const Cx ce = cexp_i(Fl(q->vk[0]) * R0 + Fl(q->vk[1]) * R1);
          const Fl ef = exp_(ke * ke - a * a);
          const Cx w = w_(Cx(ke, a));
          const Cx F = ((ce / rl) * ef) * w.re;
          const Cx cf = ((ce / (rl * rl)) * ef) * (w.re / rl - Fl(q->k) * w.im + Fl(1.0) / (ve * Fl(sqrt(M_PI))));
          *G += F; dG[0] += cf * px; dG[1] += cf * py; dG[2] += cf;
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
  const Fl f4p = Fl(4.0 * M_PI);
  *G = *G / f4p; dG[0] = dG[0] / (-f4p); dG[1] = dG[1] / (-f4p); dG[2] = dG[2] * (-r[2] / f4p);
  return cc;
}

// Ewald spectral sum: qpgf_oracle.c or_ew_spec
int ew_spec(const Q* q, const Fl* r, Fl ve, double eps, Cx* G, Cx* dG)
{
  const Rc c = recip(q);
  const int nc = (int)round((q->vk[0] * q->d1[0] + q->vk[1] * q->d1[1]) / (2 * M_PI));
  int cc = 0;
  const Cx z0(Fl(0.0), Fl(0.0));
  *G = z0; dG[0] = dG[1] = dG[2] = z0;
  for (int pass = 0; pass < 3; pass++) {
    int n1 = nc + (pass == 0 ? 0 : (pass == 1 ? 1 : -1)), st = pass == 2 ? -1 : 1;
    for (; abs(n1 - nc) < 100; n1 += st) {
      const Cx od = dG[2];
      const int nc2 = (int)round(-((-q->vk[0] + n1 * c.g1[0]) * c.g2[0] + (-q->vk[1] + n1 * c.g1[1]) * c.g2[1]) /
                                 (c.g2[0] * c.g2[0] + c.g2[1] * c.g2[1]));
      int prop = 0;
      for (int side = 0; side < 3; side++) {
        int n2 = side == 0 ? nc2 : (side == 1 ? nc2 + 1 : nc2 - 1), s2 = side == 2 ? -1 : 1;
        for (; abs(n2 - nc2) < 100; n2 += s2) {
          const Fl a0 = Fl(-q->vk[0]) + Fl((double)n1) * Fl(c.g1[0]) + Fl((double)n2) * Fl(c.g2[0]);
          const Fl a1 = Fl(-q->vk[1]) + Fl((double)n1) * Fl(c.g1[1]) + Fl((double)n2) * Fl(c.g2[1]);
          const Fl b2 = Fl(q->k) * Fl(q->k) - a0 * a0 - a1 * a1;
          const Cx ce = cexp_i(a0 * r[0] + a1 * r[1]);
          Cx F, dz;
          int evan;
          if (b2.v > 0) {
            const Fl b = sqrt_(b2), az = r[2] / (Fl(2.0) * ve);
            const Fl ef = exp_(b2 * ve * ve - az * az);
            const Cx ff = cexp_i(b * r[2]), w = w_(Cx(b * ve, az));
            F = ((ce * Fl(2.0)) / b) * Cx(ff.re, ef * w.im + ff.im);
            dz = (ce * Fl(2.0)) * Cx(ef * w.re - ff.re, -ff.im);
            evan = 0;
          } else if (b2.v < 0) {
            const Fl b = sqrt_(-b2), az = r[2] / (Fl(2.0) * ve), eb = exp_(b * r[2]);
            const Fl f1 = eb * erfc_(b * ve + az), f2 = erfc_(b * ve - az) / eb;
            F = neg(mul_i(ce / b)) * (f1 + f2);  // ce / (i b) = -i ce / b
            dz = ce * (f1 - f2);
            evan = 1;
          } else {
            return -3;
          }
          *G += F; dG[0] += F * a0; dG[1] += F * a1; dG[2] += dz;
          cc++;
          if (side == 0) break;
          if (evan) {
            if (small(dz, dG[2], eps)) break;
          } else {
            prop++;
          }
        }
        if (side > 0 && abs(n2 - nc2) >= 100) return -2;
      }
      if (pass == 0) break;
      if (prop == 0 && same(dG[2], od, eps)) break;
    }
    if (pass > 0 && abs(n1 - nc) >= 100) return -2;
  }
  const Fl a = Fl(fabs(c.idd));
  *G = mul_i(*G * (Fl(0.25) * a)); dG[0] = dG[0] * (Fl(-0.25) * a); dG[1] = dG[1] * (Fl(-0.25) * a);
  dG[2] = dG[2] * (Fl(0.25) * a);
  return cc;
}

// Fourier-domain sum: qpgf_oracle.c or_fd
int fd_sum(const Q* q, const Fl* r, double eps, Cx* G, Cx* dG)
{
  if (r[2].v == 0.0) return -4;
  const Rc c = recip(q);
  const int nc = (int)round((q->vk[0] * q->d1[0] + q->vk[1] * q->d1[1]) / (2 * M_PI));
  int cc = 0;
  const Cx z0(Fl(0.0), Fl(0.0));
  *G = z0; dG[0] = dG[1] = dG[2] = z0;
  const Fl az = fabs_(r[2]);
  for (int pass = 0; pass < 3; pass++) {
    int n1 = nc + (pass == 0 ? 0 : (pass == 1 ? 1 : -1)), st = pass == 2 ? -1 : 1;
    for (; abs(n1 - nc) < 100; n1 += st) {
      const Cx od = dG[2];
      const int nc2 = (int)round((q->vk[0] * c.g2[0] + q->vk[1] * c.g2[1] - n1 * (c.g1[0] * c.g2[0] + c.g1[1] * c.g2[1])) /
                                 (c.g2[0] * c.g2[0] + c.g2[1] * c.g2[1]));
      for (int side = 0; side < 3; side++) {
        int n2 = side == 0 ? nc2 : (side == 1 ? nc2 + 1 : nc2 - 1), s2 = side == 2 ? -1 : 1;
        for (; abs(n2 - nc2) < 100; n2 += s2) {
          const Fl a0 = Fl(-q->vk[0]) + Fl((double)n1) * Fl(c.g1[0]) + Fl((double)n2) * Fl(c.g2[0]);
          const Fl a1 = Fl(-q->vk[1]) + Fl((double)n1) * Fl(c.g1[1]) + Fl((double)n2) * Fl(c.g2[1]);
          const Fl b2 = Fl(q->k) * Fl(q->k) - a0 * a0 - a1 * a1;
          Cx dz, F;
          int evan;
          if (b2.v > 0) {
            const Fl b = sqrt_(b2);
            dz = cexp_i(a0 * r[0] + a1 * r[1] + b * az);
            F = dz / b;
            evan = 0;
          } else if (b2.v < 0) {
            const Fl b = sqrt_(-b2);
            dz = cexp_i(a0 * r[0] + a1 * r[1]) * exp_(-(b * az));
            F = neg(mul_i(dz / b));
            evan = 1;
          } else {
            return -2;
          }
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
  const Fl a = Fl(fabs(c.idd));
  *G = mul_i(*G * (Fl(0.5) * a)); dG[0] = dG[0] * (Fl(-0.5) * a); dG[1] = dG[1] * (Fl(-0.5) * a);
  dG[2] = dG[2] * (Fl(-0.5) * a * r[2] / az);
  return cc;
}

}  // namespace

extern "C" {

void oc_set_tables(const double* ax, double Lx, const double* aw, double Lw)
{
  g_ax = ax; g_Lx = Lx; g_aw = aw; g_Lw = Lw;
}

// Special functions alone, for the accuracy checks (value, operations).
double oc_exp(double x, unsigned long long* ops) { g_ops = 0; double v = exp_(Fl(x)).v; *ops = g_ops; return v; }
double oc_erfc(double x, unsigned long long* ops) { g_ops = 0; double v = erfc_(Fl(x)).v; *ops = g_ops; return v; }
void oc_sincos(double x, double* sc, unsigned long long* ops)
{
  g_ops = 0; Fl s, c; sincos_(Fl(x), s, c); sc[0] = s.v; sc[1] = c.v; *ops = g_ops;
}
void oc_w(double x, double y, double* w, unsigned long long* ops)
{
  g_ops = 0; Cx v = w_(Cx(Fl(x), Fl(y))); w[0] = v.re.v; w[1] = v.im.v; *ops = g_ops;
}

// G and grad G at r (p: k, vk[3], d1[2], d2[2]); zfac > 0 selects the assembly kernels' cost rule.
// out: G, dG[3] interleaved re/im; info: [terms, operations, 1 if the Fourier-domain sum ran].
int oc_point(const double* p, const double* rin, double zfac, double* out, unsigned long long* info)
{
  Q q = {p[0], {p[1], p[2], p[3]}, {p[4], p[5]}, {p[6], p[7]}};
  const double eps = 1e-15;
  g_ops = 0;
  // lattice reduction and method choice (qpgf_oracle.c or_qpgf_v1): per point
  const double det = q.d1[0] * q.d2[1] - q.d2[0] * q.d1[1], idd = 1.0 / det;
  const Fl x0 = Fl(rin[0]), x1 = Fl(rin[1]);
  const int l1 = (int)floor(((x0 * Fl(q.d2[1]) - x1 * Fl(q.d2[0])) * Fl(idd) + Fl(0.5)).v);
  const int l2 = (int)floor((-(x0 * Fl(q.d1[1]) - x1 * Fl(q.d1[0])) * Fl(idd) + Fl(0.5)).v);
  Fl r[3] = {x0 - Fl((double)l1) * Fl(q.d1[0]) - Fl((double)l2) * Fl(q.d2[0]),
             x1 - Fl((double)l1) * Fl(q.d1[1]) - Fl((double)l2) * Fl(q.d2[1]), Fl(rin[2])};
  // lattice constants of the selection (once per lattice)
  const double k2 = q.k * q.k, cpd = 2 * M_PI * idd;
  const double ad12 = q.d1[0] * q.d1[0] + q.d1[1] * q.d1[1], ad22 = q.d2[0] * q.d2[0] + q.d2[1] * q.d2[1];
  const int n1 = (int)round((q.vk[0] * q.d1[0] + q.vk[1] * q.d1[1]) / (2 * M_PI));
  const int n2 = (int)round((q.vk[0] * q.d2[0] + q.vk[1] * q.d2[1]) / (2 * M_PI));
  const double ax = -q.vk[0] + n1 * cpd * q.d2[1] - n2 * cpd * q.d1[1], ay = -q.vk[1] - n1 * cpd * q.d2[0] + n2 * cpd * q.d1[0];
  const double bN = sqrt(k2 - ax * ax - ay * ay);
  int m1p = n1, m1m = n1, m2p = n2, m2m = n2;
  if (ad22 < ad12) { m1p += 15; m1m -= 15; } else { m2p += 15; m2m -= 15; }
  const double px = -q.vk[0] + m1p * cpd * q.d2[1] - m2p * cpd * q.d1[1], py = -q.vk[1] - m1p * cpd * q.d2[0] + m2p * cpd * q.d1[0];
  const double mx = -q.vk[0] + m1m * cpd * q.d2[1] - m2m * cpd * q.d1[1], my = -q.vk[1] - m1m * cpd * q.d2[0] + m2m * cpd * q.d1[0];
  double bp = k2 - px * px - py * py, bm = k2 - mx * mx - my * my;
  int fd = 0;
  if (!(bp > 0 || bm > 0)) {
    bp = sqrt(-bp); bm = sqrt(-bm);
    const Fl az = fabs_(r[2]);
    fd = (Fl(bN / bp) * exp_(-(Fl(bp) * az)) < Fl(eps)) && (Fl(bN / bm) * exp_(-(Fl(bm) * az)) < Fl(eps));
  }
  const double adp = sqrt(pow(q.d1[0] + q.d2[0], 2) + pow(q.d1[1] + q.d2[1], 2));
  const double adm = sqrt(pow(q.d1[0] - q.d2[0], 2) + pow(q.d1[1] - q.d2[1], 2));
  Fl ve = Fl(sqrt(fabs(det) / (4 * M_PI) * adp / adm));
  const Fl r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  if (Fl(k2) * ve * ve - r2 / (Fl(4.0) * ve * ve) > Fl(3.0))
    ve = sqrt_(Fl(3.0) + sqrt_(Fl(k2) * r2 + Fl(9.0))) / (Fl(sqrt(2.0)) * Fl(q.k));
  if (zfac > 0.0 && fd && fabs_(r[2]) < Fl(zfac) * ve) fd = 0;
  Cx G, dG[3];
  int err;
  if (fd) {
    err = fd_sum(&q, r, eps, &G, dG);
    if (err < 0) return err - 10;
  } else {
    Cx G2, d2[3];
    const int c1 = ew_real(&q, r, ve, eps, &G, dG);
    if (c1 < 0) return c1 - 20;
    const int c2 = ew_spec(&q, r, ve, eps, &G2, d2);
    if (c2 < 0) return c2 - 20;
    G += G2; dG[0] += d2[0]; dG[1] += d2[1]; dG[2] += d2[2];
    err = c1 + c2;
  }
  if (l1 || l2) {
    const Cx cf = cexp_i(-(Fl(q.vk[0]) * (Fl((double)l1) * Fl(q.d1[0]) + Fl((double)l2) * Fl(q.d2[0])) +
                           Fl(q.vk[1]) * (Fl((double)l1) * Fl(q.d1[1]) + Fl((double)l2) * Fl(q.d2[1]))));
    G = G * cf; dG[0] = dG[0] * cf; dG[1] = dG[1] * cf; dG[2] = dG[2] * cf;
  }
  out[0] = G.re.v; out[1] = G.im.v;
  for (int i = 0; i < 3; i++) { out[2 + 2 * i] = dG[i].re.v; out[3 + 2 * i] = dG[i].im.v; }
  info[0] = (unsigned long long)err;
  info[1] = g_ops;
  info[2] = (unsigned long long)fd;
  return err;
}

}  // extern "C"

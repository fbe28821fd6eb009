// elem.cuh -- element geometry and the per-quadrature-point integrands of the boundary-integral
// coefficients, host+device.
//
// One "pair" is a collocation node (element t, node tn) against a source element s.  The
// reference evaluates each pair with element rules that loop over shape functions outermost
// and re-evaluate the Green's function for every shape function (e.g. q0_bil_dcoef_v2_cc.c:153-197,
// 4 Green's function calls per quadrature point).  Here every quadrature point is visited once and
// its contribution is scattered into all shape-function accumulators, so the Green's function is
// evaluated once per point; the sums are the same quadrature sums.
//
// Geometry (per element id 1..Ne, id 0 unused; GEO_STRIDE doubles each):
//   [0..11]  cr[3][4]  r(zeta,eta) = cr[:,0] + cr[:,1] zeta + cr[:,2] eta + cr[:,3] zeta eta
//   [12..20] cw[3][3]  W(zeta,eta) = cw[:,0] + cw[:,1] zeta + cw[:,2] eta  (|W| = Jacobian)
//   [21..32] ren[4][3] collocation node positions       (d3qd2_setup.c:1309-1349)
//   [33..44] wen[4][3] normal vectors at the nodes
//   [45]     number of vertices (3 or 4)
// These are the reference's element constants (init_elem_const, d3qd2_setup.c:1139-1222).
#pragma once

#include "cplx.cuh"
#include "qpgf.cuh"

#define GEO_STRIDE 48
#define GEO_CR 0
#define GEO_CW 12
#define GEO_REN 21
#define GEO_WEN 33
#define GEO_NN 45

#define EL_I_FP 7.957747154594766788444e-2    // 1/(4 pi)
#define EL_SQ3 1.732050807568877293528e+0     // sqrt(3)
#define EL_I_SPSQ3 3.062938307898844719507e-2 // 1/(6 pi sqrt(3))
#define EL_P44_N 0.5773502691896257645091     // sqrt(1/3)
#define EL_P34_N0 0.2
#define EL_P34_N1 0.3464101615137754587055    // sqrt(3)/5
#define EL_CBD_SDF 0.5                         // near-singular switch (d3qd2_const.h:453)
#define EL_CDFH 1.0e-3                         // finite-difference step (d3qd2_const.h:37)
#define EL_GEPS 1.0e-15
#define EL_DEPS 0.1

struct Elem {
  double cr[3][4];
  double cw[3][3];
  int nn;
};

BEM_HD void load_elem(const double* __restrict__ geo, int id, Elem& e)
{
  const double* g = geo + (size_t)id * GEO_STRIDE;
#pragma unroll
  for (int d = 0; d < 3; d++) {
#pragma unroll
    for (int c = 0; c < 4; c++) e.cr[d][c] = g[GEO_CR + d * 4 + c];
#pragma unroll
    for (int c = 0; c < 3; c++) e.cw[d][c] = g[GEO_CW + d * 3 + c];
  }
  e.nn = (int)g[GEO_NN];
  if (e.nn == 3) {  // lit_copy_elem_const_rw (d3qd2_elem.c:1060-1073) zeroes these
    for (int d = 0; d < 3; d++) { e.cr[d][3] = 0.0; e.cw[d][1] = 0.0; e.cw[d][2] = 0.0; }
  }
}

BEM_HD double vnorm3(const double* v) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
BEM_HD double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
BEM_HD void unit3(double* v)
{
  double a = vnorm3(v);
  if (a != 0.0) { v[0] /= a; v[1] /= a; v[2] /= a; }
}

// node parameter positions (d3qd2_setup.c:1189-1200)
BEM_HD double node_zeta(int nn, int nid)
{
  if (nn == 4) return (nid == 0 || nid == 3) ? -EL_P44_N : EL_P44_N;
  return (nid == 0 || nid == 2) ? -EL_P34_N0 : (nid == 1 ? 2.0 * EL_P34_N0 : 0.0);
}
BEM_HD double node_eta(int nn, int nid)
{
  if (nn == 4) return (nid < 2) ? -EL_P44_N : EL_P44_N;
  return nid == 0 ? -EL_P34_N1 : (nid == 2 ? EL_P34_N1 : 0.0);
}

// unit tangents at an element node (tz_te_bd_node, d3qd2_elem.c:122-143)
BEM_HD void node_tangents(const Elem& e, int nid, double* vtz, double* vte)
{
  if (e.nn == 4) {
    double zt = node_zeta(4, nid), et = node_eta(4, nid);
    for (int i = 0; i < 3; i++) {
      vtz[i] = e.cr[i][1] + e.cr[i][3] * et;
      vte[i] = e.cr[i][2] + e.cr[i][3] * zt;
    }
  } else {
    for (int i = 0; i < 3; i++) { vtz[i] = e.cr[i][1]; vte[i] = e.cr[i][2]; }
  }
  unit3(vtz);
  unit3(vte);
}

// interpolation functions (bil_Nn d3qd2_elem.c:903-915, lit_Nn :1047-1058)
BEM_HD void bil_N4(double zeta, double eta, double* N)
{
  const double i_a = 1.0 / EL_P44_N;
  N[0] = 0.25 * (1.0 - zeta * i_a) * (1.0 - eta * i_a);
  N[1] = 0.25 * (1.0 + zeta * i_a) * (1.0 - eta * i_a);
  N[2] = 0.25 * (1.0 + zeta * i_a) * (1.0 + eta * i_a);
  N[3] = 0.25 * (1.0 - zeta * i_a) * (1.0 + eta * i_a);
}
BEM_HD void lit_N3(double zeta, double eta, double* N)
{
  const double i_a = 0.5 / EL_P34_N0;
  N[0] = 1.0 / 3.0 * (1.0 - i_a * (zeta + EL_SQ3 * eta));
  N[1] = 1.0 / 3.0 * (1.0 + 2.0 * i_a * zeta);
  N[2] = 1.0 / 3.0 * (1.0 - i_a * (zeta - EL_SQ3 * eta));
}

BEM_HD void bil_rw(const Elem& e, double zeta, double eta, double* r, double* w)
{
  for (int i = 0; i < 3; i++) {
    r[i] = e.cr[i][0] + e.cr[i][1] * zeta + e.cr[i][2] * eta + e.cr[i][3] * zeta * eta;
    w[i] = e.cw[i][0] + e.cw[i][1] * zeta + e.cw[i][2] * eta;
  }
}
BEM_HD void lit_r(const Elem& e, double zeta, double eta, double* r)
{
  for (int i = 0; i < 3; i++) r[i] = e.cr[i][0] + e.cr[i][1] * zeta + e.cr[i][2] * eta;
}

// Triangle rule: each GL node pair (a,b) maps to one point in each of the three sub-quads of
// the reference triangle, with Jacobian weight 1 + a/4 + b/4 (q0_lit_dcoef_v2_cc.c:199-218).
BEM_HD void lit_part_point(int part, double a, double b, double& zeta, double& eta)
{
  if (part == 0) {
    zeta = 0.125 * (3.0 + 2.0 * a + 2.0 * b + a * b);
    eta = 0.125 * EL_SQ3 * (-a + b);
  } else if (part == 1) {
    zeta = 0.0625 * (-3.0 + a - 5.0 * b - a * b);
    eta = 0.0625 * EL_SQ3 * (3.0 + 3.0 * a + b + a * b);
  } else {
    zeta = 0.0625 * (-3.0 - 5.0 * a + b - a * b);
    eta = 0.0625 * EL_SQ3 * (-3.0 - a - 3.0 * b - a * b);
  }
}

// Point enumeration of a regular rule with n nodes per direction.  Quad: q in [0, n*n).
// Triangle: q in [0, 3*n*n) (part-major).  Returns zeta, eta and the full weight.
BEM_HD void rule_point(int nn, int n, const double* x, const double* wgt, int q, double& zeta, double& eta, double& w)
{
  if (nn == 4) {
    int i = q / n, j = q - (q / n) * n;
    zeta = x[i]; eta = x[j];
    w = wgt[i] * wgt[j];
  } else {
    int part = q / (n * n);
    int r = q - part * n * n;
    int i = r / n, j = r - (r / n) * n;
    double a = x[i], b = x[j];
    lit_part_point(part, a, b, zeta, eta);
    w = wgt[i] * wgt[j] * (1.0 + 0.25 * a + 0.25 * b);
  }
}

// =============================================================================================
// Periodic (open-domain) pair, "cc" variant: CC[0..8], dC0[8], dC1[8]
// (q0_bil_dcoef_v2_cc_GL/GH q0_bil_dcoef_v2_cc.c:129-281; q0_lit_dcoef_v2_cc_GL
// q0_lit_dcoef_v2_cc.c:156-237 with integrand q0_lit_sdqGHF_v2_cc_zeta_eta :345-381).
struct AccP {
  cplx G[4], H[4];
  double F, dF0, dF1;
};

BEM_HD void accp_zero(AccP& a)
{
  for (int i = 0; i < 4; i++) { a.G[i] = mk(0, 0); a.H[i] = mk(0, 0); }
  a.F = 0; a.dF0 = 0; a.dF1 = 0;
}

// Source point r(zeta, eta) relative to the target rt, and the Jacobian normal W there.
BEM_HD void point_geom(const Elem& e, double zeta, double eta, const double* rt, double* vR, double* vW)
{
  if (e.nn == 4) {
    bil_rw(e, zeta, eta, vR, vW);
  } else {
    lit_r(e, zeta, eta, vR);
    vW[0] = e.cw[0][0]; vW[1] = e.cw[1][0]; vW[2] = e.cw[2][0];
  }
  for (int l = 0; l < 3; l++) vR[l] -= rt[l];
}

// Adds the contribution of one quadrature point; returns the QPGF status (<0: error) or the
// number of lattice terms.
BEM_HD int accp_point(const Elem& e, const QPLattice& L, const double* rt, const double* v0, const double* v1,
                      double zeta, double eta, double w, AccP& a)
{
  double vR[3], vW[3];
  point_geom(e, zeta, eta, rt, vR, vW);
  QPVal g;
  int err = qpgf_eval<QP_V1, true>(L, vR, g);
  // the geometry once more, after the lattice sums: only (zeta, eta, w) stay live across them
  // (the callers keep the element, the target and the sums in shared memory)
  point_geom(e, zeta, eta, rt, vR, vW);
  double aR = vnorm3(vR);
  double i_aR = 1.0 / aR;
  double rdW = dot3(vR, vW) * i_aR;
  double rdv0 = dot3(vR, v0) * i_aR, rdv1 = dot3(vR, v1) * i_aR;
  double Wdv0 = dot3(vW, v0), Wdv1 = dot3(vW, v1);
  cplx hn = g.dG[0] * vW[0] + g.dG[1] * vW[1] + g.dG[2] * vW[2];
  double N[4];
  double i3 = i_aR * i_aR * i_aR;
  if (e.nn == 4) {
    double aW = vnorm3(vW);
    bil_N4(zeta, eta, N);
    cplx gw = g.G * (w * aW);
    cplx hw = hn * w;
    for (int ep = 0; ep < 4; ep++) { a.G[ep] += gw * N[ep]; a.H[ep] += hw * N[ep]; }
  } else {
    lit_N3(zeta, eta, N);
    cplx gw = g.G * w;
    cplx hw = hn * w;
    for (int ep = 0; ep < 3; ep++) { a.G[ep] += gw * N[ep]; a.H[ep] += hw * N[ep]; }
  }
  a.F += w * rdW * i_aR * i_aR;
  a.dF0 += w * i3 * (3.0 * rdv0 * rdW - Wdv0);
  a.dF1 += w * i3 * (3.0 * rdv1 * rdW - Wdv1);
  return err;
}

// Final scalings.  out: CC[9], dCz[9], dCe[9] (only [8] of the derivatives is non-zero).
BEM_HD void accp_finish(const Elem& e, const AccP& a, cplx* CC, cplx* dCz, cplx* dCe)
{
  for (int i = 0; i < 9; i++) { CC[i] = mk(0, 0); dCz[i] = mk(0, 0); dCe[i] = mk(0, 0); }
  if (e.nn == 4) {
    for (int ep = 0; ep < 4; ep++) { CC[ep] = a.G[ep]; CC[ep + 4] = a.H[ep]; }
    CC[8] = mk(a.F * EL_I_FP, 0);
    dCz[8] = mk(a.dF0 * EL_I_FP, 0);
    dCe[8] = mk(a.dF1 * EL_I_FP, 0);
  } else {
    double V[3] = {e.cw[0][0], e.cw[1][0], e.cw[2][0]};
    double aW = vnorm3(V);
    for (int ep = 0; ep < 3; ep++) {
      CC[ep] = a.G[ep] * (1.0 / (24.0) * aW);
      CC[ep + 4] = a.H[ep] * (1.0 / (24.0));
    }
    const double c = 0.0625 * EL_SQ3 * EL_I_SPSQ3;
    CC[8] = mk(a.F * c, 0);
    dCz[8] = mk(a.dF0 * c, 0);
    dCe[8] = mk(a.dF1 * c, 0);
  }
}

// =============================================================================================
// Interior (free-space, complex k) pair: CC[9], dC0[9], dC1[9]
// (bil_dcoef_v2_GL/GH bil_dcoef_v2.c:141-325; lit_dcoef_v2_GL/GH lit_dcoef_v2.c:185-357 with
// integrand lit_sdGL_v2_zeta_eta :381-413).  Negative source ids flip H, F and their
// derivatives (bil_convert_CC / bil_convert_dCC, d3qd2_elem.c:927-947).
struct AccI {
  cplx G[4], H[4], dG0[4], dH0[4], dG1[4], dH1[4];
  double F, dF0, dF1;
};

BEM_HD void acci_zero(AccI& a)
{
  for (int i = 0; i < 4; i++) {
    a.G[i] = mk(0, 0); a.H[i] = mk(0, 0); a.dG0[i] = mk(0, 0); a.dH0[i] = mk(0, 0);
    a.dG1[i] = mk(0, 0); a.dH1[i] = mk(0, 0);
  }
  a.F = 0; a.dF0 = 0; a.dF1 = 0;
}

BEM_HD void acci_point(const Elem& e, cplx k, const double* rt, const double* v0, const double* v1,
                       double zeta, double eta, double w, AccI& a)
{
  double vR[3], vW[3];
  if (e.nn == 4) {
    bil_rw(e, zeta, eta, vR, vW);
  } else {
    lit_r(e, zeta, eta, vR);
    vW[0] = e.cw[0][0]; vW[1] = e.cw[1][0]; vW[2] = e.cw[2][0];
  }
  for (int l = 0; l < 3; l++) vR[l] -= rt[l];
  double aR = vnorm3(vR);
  double i_aR = 1.0 / aR;
  cplx kR = k * aR;
  cplx ca = mul_i(kR);                 // i k R
  cplx cb = mk(ca.re - 1.0, ca.im);    // i k R - 1
  cplx ce = cexp_(ca);                 // e^{i k R}
  double rdW = dot3(vR, vW) * i_aR;
  double rdv0 = dot3(vR, v0) * i_aR, rdv1 = dot3(vR, v1) * i_aR;
  double Wdv0 = dot3(vW, v0), Wdv1 = dot3(vW, v1);
  double i2 = i_aR * i_aR, i3 = i2 * i_aR;
  double aW = (e.nn == 4) ? vnorm3(vW) : 1.0;  // the triangle rule applies |W| at the end
  cplx kR2p3 = kR * kR + 3.0 * cb;             // (kR)^2 + 3 (ikR - 1)
  cplx g = ce * (i_aR * aW);                                   // G
  cplx h = cb * ce * (rdW * i2);                               // H
  cplx dg0 = cb * ce * (i2 * rdv0 * aW);                       // dG/dv0
  cplx dg1 = cb * ce * (i2 * rdv1 * aW);
  cplx dh0 = ce * (kR2p3 * (rdv0 * rdW) - cb * Wdv0) * i3;     // dH/dv0
  cplx dh1 = ce * (kR2p3 * (rdv1 * rdW) - cb * Wdv1) * i3;
  double N[4];
  int ne;
  if (e.nn == 4) { bil_N4(zeta, eta, N); ne = 4; } else { lit_N3(zeta, eta, N); ne = 3; }
  for (int ep = 0; ep < ne; ep++) {
    double wn = w * N[ep];
    a.G[ep] += g * wn;
    a.H[ep] += h * wn;
    a.dG0[ep] += dg0 * wn;
    a.dG1[ep] += dg1 * wn;
    a.dH0[ep] += dh0 * wn;
    a.dH1[ep] += dh1 * wn;
  }
  a.F += w * rdW * i2;
  a.dF0 += w * i3 * (3.0 * rdv0 * rdW - Wdv0);
  a.dF1 += w * i3 * (3.0 * rdv1 * rdW - Wdv1);
}

BEM_HD void acci_finish(const Elem& e, const AccI& a, int negative, cplx* CC, cplx* dCz, cplx* dCe)
{
  for (int i = 0; i < 9; i++) { CC[i] = mk(0, 0); dCz[i] = mk(0, 0); dCe[i] = mk(0, 0); }
  double cg, ch, cf;
  int ne;
  if (e.nn == 4) {
    cg = EL_I_FP; ch = EL_I_FP; cf = EL_I_FP; ne = 4;
  } else {
    double V[3] = {e.cw[0][0], e.cw[1][0], e.cw[2][0]};
    double c = 0.0625 * EL_SQ3 * EL_I_SPSQ3;
    cg = c * vnorm3(V); ch = c; cf = c; ne = 3;
  }
  for (int ep = 0; ep < ne; ep++) {
    CC[ep] = a.G[ep] * cg;
    CC[ep + 4] = a.H[ep] * ch;
    dCz[ep] = a.dG0[ep] * (-cg);
    dCe[ep] = a.dG1[ep] * (-cg);
    dCz[ep + 4] = a.dH0[ep] * ch;
    dCe[ep + 4] = a.dH1[ep] * ch;
  }
  CC[8] = mk(a.F * cf, 0);
  dCz[8] = mk(a.dF0 * cf, 0);
  dCe[8] = mk(a.dF1 * cf, 0);
  if (negative) {
    for (int i = 4; i < 9; i++) { CC[i] = -CC[i]; dCz[i] = -dCz[i]; dCe[i] = -dCe[i]; }
  }
}

// Near-singular switch (d3qd2_elem.c:536-537, 563-564, 851-852, 877-878): a GL result is
// replaced by the 64x64 (GH) result when |dF/dv| exceeds CBD_SDF along either tangent, for
// quads and triangles alike (q0_bil_dcoef_v2_cc_GH :206-281, q0_lit_dcoef_v2_cc_GH :239-320).
BEM_HD int needs_gh(double dFz, double dFe) { return fabs(dFz) > EL_CBD_SDF || fabs(dFe) > EL_CBD_SDF; }

// =============================================================================================
// Polar rule for the self-element (t == s) integrals (q0_bil_coef_bd q0_bil_coef.c:246-338,
// q0_lit_coef_bd q0_lit_coef.c:297-371, bil_coef_bd bil_coef.c:244-342, lit_coef_bd
// lit_coef.c:290-348).  The element is split into sub-triangles at the node (zeta_t, eta_t);
// each sub-triangle gets 2 x 64 Gauss-Legendre nodes in theta and n_r nodes in r from 0 to
// the edge distance rm(theta).
struct PolarSet {
  double r[5], th[5];
  int nsub;  // 4 (quad) or 3 (triangle)
};

// bil_calc_node_r_th (d3qd2_elem.c:1014-1028), lit_calc_node_r_th (:1149-1162)
BEM_HD void polar_setup(int nn, double zeta_t, double eta_t, PolarSet& P)
{
  if (nn == 4) {
    double ztp = 1.0 - zeta_t, ztm = -1.0 - zeta_t, etp = 1.0 - eta_t, etm = -1.0 - eta_t;
    P.r[0] = sqrt(ztm * ztm + etm * etm); P.r[1] = sqrt(ztp * ztp + etm * etm);
    P.r[2] = sqrt(ztp * ztp + etp * etp); P.r[3] = sqrt(ztm * ztm + etp * etp);
    P.r[4] = P.r[0];
    P.th[0] = atan2(etm, ztm); P.th[1] = atan2(etm, ztp);
    P.th[2] = atan2(etp, ztp); P.th[3] = atan2(etp, ztm);
    P.th[4] = P.th[0] + 2.0 * QP_PI;
    P.nsub = 4;
  } else {
    double ztp = 1.0 - zeta_t, ztm = -0.5 - zeta_t, etp = 0.5 * EL_SQ3 - eta_t, etm = -0.5 * EL_SQ3 - eta_t;
    P.r[0] = sqrt(ztm * ztm + etm * etm); P.r[1] = sqrt(ztp * ztp + eta_t * eta_t);
    P.r[2] = sqrt(ztm * ztm + etp * etp);
    P.r[3] = P.r[0];
    P.th[0] = atan2(etm, ztm); P.th[1] = atan2(-eta_t, ztp);
    P.th[2] = atan2(etp, ztm);
    P.th[3] = P.th[0] + 2.0 * QP_PI;
    P.r[4] = 0; P.th[4] = 0;
    P.nsub = 3;
  }
}

// theta node m2 in [0,128) of sub-triangle j: returns theta and its weight
BEM_HD void polar_theta(const PolarSet& P, int j, int m2, const double* xh, const double* wh, double& theta, double& wt)
{
  double th0 = P.th[j], th1 = P.th[j + 1];
  int m = m2 & 63;
  if (m2 < 64) theta = 0.25 * (th1 - th0) * xh[m] + 0.25 * (th1 + 3.0 * th0);
  else theta = 0.25 * (th1 - th0) * xh[m] + 0.25 * (3.0 * th1 + th0);
  wt = 0.25 * (th1 - th0) * wh[m];
}

// distance from the node to the sub-triangle's far edge along theta (q0_bil_sqG_theta :417)
BEM_HD double polar_rm(const PolarSet& P, int j, double theta)
{
  double r0 = P.r[j], r1 = P.r[j + 1], th0 = P.th[j], th1 = P.th[j + 1];
  return r0 * r1 * sin(th1 - th0) / (r0 * sin(theta - th0) - r1 * sin(theta - th1));
}

// bil_check_plane (d3qd2_elem.c:987-996)
BEM_HD int bil_is_plane(const Elem& e)
{
  double bdc = e.cr[0][1] * e.cw[0][2] + e.cr[1][1] * e.cw[1][2] + e.cr[2][1] * e.cw[2][2];
  double ab = sqrt(e.cr[0][1] * e.cr[0][1] + e.cr[1][1] * e.cr[1][1] + e.cr[2][1] * e.cr[2][1]);
  double aC = sqrt(e.cw[0][2] * e.cw[0][2] + e.cw[1][2] * e.cw[1][2] + e.cw[2][2] * e.cw[2][2]);
  return fabs(bdc / (ab * aC)) < EL_GEPS;
}

// K(r, theta) of the bilinear map: r(zeta_t + r c, eta_t + r s) - r(zeta_t, eta_t) = r K
BEM_HD void bil_K(const Elem& e, double zeta_t, double eta_t, double r, double cth, double sth, double* K)
{
  for (int i = 0; i < 3; i++)
    K[i] = e.cr[i][1] * cth + e.cr[i][2] * sth + e.cr[i][3] * (r * cth * sth + zeta_t * sth + eta_t * cth);
}

// Free-space solid-angle term of a curved bilinear self element around (zeta_t, eta_t)
// (q0_bil_coef_bd_F q0_bil_dcoef_v2_cc.c:392-454; the F part of bil_coef_bd bil_coef.c:316-337).
// Serial over all points; used by the finite-difference dF/dt of the periodic self pair.
BEM_HD double bil_self_F(const Elem& e, double zeta_t, double eta_t, const double* xl, const double* wl,
                         const double* xh, const double* wh, int lane, int nlanes)
{
  if (bil_is_plane(e)) return 0.0;
  PolarSet P;
  polar_setup(4, zeta_t, eta_t, P);
  double acc = 0.0;
  for (int q = lane; q < 4 * 128; q += nlanes) {
    int j = q >> 7, m2 = q & 127;
    double theta, wt;
    polar_theta(P, j, m2, xh, wh, theta, wt);
    double rm = polar_rm(P, j, theta);
    double cth = cos(theta), sth = sin(theta);
    double s = 0.0;
    for (int i = 0; i < 12; i++) {
      double r = 0.5 * rm * (xl[i] + 1.0);
      double K[3];
      bil_K(e, zeta_t, eta_t, r, cth, sth, K);
      double aK = vnorm3(K);
      s += wl[i] * (1.0 / (aK * aK * aK) * cth * sth);
    }
    acc += wt * 0.5 * rm * s;
  }
  return acc;  // caller scales by I_FP * bdC after summing lanes
}

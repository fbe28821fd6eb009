// field.cuh -- per-element coefficients of the field representation at a point off the boundary,
// and the solid angle used to find which domain a point lies in (host + device).
//
// A field value at r is  sum_s sum_n ( CC[n] dE(s,n) - CC[n+4] E(s,n) ) / (1 + F)  (open region)
// or / F (closed regions), CC and F being surface integrals over source element s of the Green's
// function, its normal derivative times the shape functions, and the solid-angle kernel.  The
// rules here are the low-order ones the reference uses for field evaluation:
//   type 0: the element's own collocation nodes (4-point rule on quads, the 4-point
//           triangle rule with the centroid on triangles)
//   type 1: 3x3 Gauss rule on quads, 7-point rule on triangles
//   types 2 and 3: 12 x 12 and 64 x 64 Gauss-Legendre rules (field_coef_gl), for points near
//           the boundary
// (q0_bil_coef_4p/_9p q0_bil_coef.c:10-95, q0_lit_coef_4p/_7p q0_lit_coef.c:10-117 for the
// periodic Green's function; bil_coef_4p/_9p bil_coef.c:25-97, lit_coef_4p/_7p lit_coef.c:26-123
// for the free-space one.)  Each quadrature point's Green's function is evaluated once and
// scattered into every shape-function sum.
#pragma once

#include "elem.cuh"

// quadrature tables (init_elem_const, d3qd2_setup.c:1194-1217): the standard 3x3 Gauss-Legendre
// product rule, and the 4- and 7-point triangle rules on the reference triangle with vertices
// (-0.5, -sqrt(3)/2), (1, 0), (-0.5, sqrt(3)/2)
#define FQ_G3N 0.7745966692414833770359   // sqrt(3/5)
#define FQ_G3W0 0.3086419753086419753086  // 25/81
#define FQ_G3W1 0.4938271604938271604938  // 40/81
#define FQ_G3W2 0.7901234567901234567901  // 64/81
#define FQ_T4W0 0.5208333333333333333333  // 25/48
#define FQ_T4W1 0.5625                    // 27/48 (enters with a minus sign)
#define FQ_T7N0 0.3480702390148154917985  // (sqrt(15)+1)/14
#define FQ_T7N1 0.2052130961576726346557  // (sqrt(15)-1)/14
#define FQ_T7N2 0.6028753385763033130539  // sqrt(3) (sqrt(15)+1)/14
#define FQ_T7N3 0.3554395089236065568357  // sqrt(3) (sqrt(15)-1)/14
#define FQ_T7W0 0.1259391805448271525957  // (155-sqrt(15))/1200
#define FQ_T7W1 0.1323941527885061807376  // (155+sqrt(15))/1200
#define FQ_T7W2 0.225                     // 270/1200
#define FQ_I_EP 3.978873577297383394222e-2  // 1/(8 pi)

BEM_HD void fq_gauss9(int i, double& z, double& e, double& w)
{
  // points ordered as the reference's table: 4 corners, 4 edge midpoints, centre
  const double a = FQ_G3N;
  switch (i) {
    case 0: z = -a; e = -a; w = FQ_G3W0; break;
    case 1: z = a; e = -a; w = FQ_G3W0; break;
    case 2: z = a; e = a; w = FQ_G3W0; break;
    case 3: z = -a; e = a; w = FQ_G3W0; break;
    case 4: z = 0.0; e = -a; w = FQ_G3W1; break;
    case 5: z = a; e = 0.0; w = FQ_G3W1; break;
    case 6: z = 0.0; e = a; w = FQ_G3W1; break;
    case 7: z = -a; e = 0.0; w = FQ_G3W1; break;
    default: z = 0.0; e = 0.0; w = FQ_G3W2; break;
  }
}

BEM_HD void fq_tri7(int i, double& z, double& e, double& w)
{
  switch (i) {
    case 0: z = -FQ_T7N0; e = -FQ_T7N2; w = FQ_T7W0; break;
    case 1: z = 2.0 * FQ_T7N0; e = 0.0; w = FQ_T7W0; break;
    case 2: z = -FQ_T7N0; e = FQ_T7N2; w = FQ_T7W0; break;
    case 3: z = FQ_T7N1; e = FQ_T7N3; w = FQ_T7W1; break;
    case 4: z = -2.0 * FQ_T7N1; e = 0.0; w = FQ_T7W1; break;
    case 5: z = FQ_T7N1; e = -FQ_T7N3; w = FQ_T7W1; break;
    default: z = 0.0; e = 0.0; w = FQ_T7W2; break;
  }
}

// Kernel values at one quadrature point.  g = Green's function, hn = its gradient . W (W the
// element's Jacobian normal), tD = (R . W) / |R|^3, R = r(point) - rt.
struct FieldKer {
  cplx g, hn;
  double tD, aW;
};

template <bool PER>
BEM_HD int field_kernel(const QPLattice& L, cplx k, const double* vR, const double* vW, FieldKer& o)
{
  const double aR = vnorm3(vR);
  const double i_aR = 1.0 / aR;
  o.aW = vnorm3(vW);
  o.tD = dot3(vR, vW) * i_aR * i_aR * i_aR;
  if (PER) {
    QPVal v;
    int err = qpgf_eval<QP_V1>(L, vR, v);
    o.g = v.G;
    o.hn = v.dG[0] * vW[0] + v.dG[1] * vW[1] + v.dG[2] * vW[2];
    return err;
  }
  // free space: e^{ikR}/R and its normal derivative, without the 1/(4 pi) applied later
  cplx ca = mul_i(k) * aR;
  cplx ce = (k.im == 0.0) ? expi(k.re * aR) : cexp_(ca);
  o.g = ce * i_aR;
  o.hn = (ca - mk(1.0, 0.0)) * ce * o.tD;
  return 0;
}

// Coefficients of source element `sd` (signed id) at point rt: CC[0..3] (Green's function times
// shape functions), CC[4..7] (normal derivative), F.  Triangles leave CC[3], CC[7] zero.
// Returns 0, a QPGF failure code, or -1 for an unsupported type or a negative id in the
// periodic region (the reference exits there, q0_bil_coef.c:16-19).
// Gauss-Legendre tables for the rules of types 2 and 3: x12, w12, x64, w64.
struct FieldGL {
  const double *x12, *w12, *x64, *w64;
};

// Types 2 (12 x 12 Gauss-Legendre, 3 x 12 x 12 on triangles) and 3 (64 x 64): the same quadrature
// sums as the regular element rules of the assembly (q0_bil_coef_GL/_GH q0_bil_coef.c:97-190,
// q0_lit_coef_GL/_GH q0_lit_coef.c:118-250, bil_coef_GL/_GH bil_coef.c:99-190, lit_coef_GL/_GH
// lit_coef.c:125-260), so they run through accp_point / acci_point and keep their CC part.
template <bool PER>
BEM_HD int field_coef_gl(const double* geo, int sd, const double* rt, cplx k, int type, const FieldGL& gl,
                         const QPLattice& L, cplx* CC, double& F)
{
  const int s = sd < 0 ? -sd : sd;
  Elem el;
  load_elem(geo, s, el);
  const int n = (type == 2) ? 12 : 64;
  const double* x = (type == 2) ? gl.x12 : gl.x64;
  const double* w = (type == 2) ? gl.w12 : gl.w64;
  const int npts = (el.nn == 4) ? n * n : 3 * n * n;
  const double v0[3] = {0.0, 0.0, 0.0};  // tangents of the derivative parts, not needed here
  cplx C9[9], dCz[9], dCe[9];
  int err = 0;
  if (PER) {
    AccP a;
    accp_zero(a);
    for (int q = 0; q < npts; q++) {
      double z, e, wt;
      rule_point(el.nn, n, x, w, q, z, e, wt);
      const int st = accp_point(el, L, rt, v0, v0, z, e, wt, a);
      if (st < 0) err = st;
    }
    accp_finish(el, a, C9, dCz, dCe);
  } else {
    AccI a;
    acci_zero(a);
    for (int q = 0; q < npts; q++) {
      double z, e, wt;
      rule_point(el.nn, n, x, w, q, z, e, wt);
      acci_point(el, k, rt, v0, v0, z, e, wt, a);
    }
    acci_finish(el, a, sd < 0, C9, dCz, dCe);
  }
  for (int i = 0; i < 8; i++) CC[i] = C9[i];
  F = C9[8].re;
  return err;
}

template <bool PER>
BEM_HD int field_coef(const double* geo, int sd, const double* rt, cplx k, int type, const QPLattice& L, cplx* CC,
                      double& F, const FieldGL* gl = nullptr)
{
  for (int i = 0; i < 8; i++) CC[i] = mk(0.0, 0.0);
  F = 0.0;
  if (PER && sd < 0) return -1;
  if (type == 2 || type == 3) {
    if (!gl) return -1;
    return field_coef_gl<PER>(geo, sd, rt, k, type, *gl, L, CC, F);
  }
  if (type != 0 && type != 1) return -1;
  const int s = sd < 0 ? -sd : sd;
  const double* g = geo + (size_t)s * GEO_STRIDE;
  const int nn = (int)g[GEO_NN];
  int err = 0;
  FieldKer q;
  double vR[3], vW[3];
  if (nn == 4) {
    if (type == 0) {
      for (int i = 0; i < 4; i++) {
        for (int l = 0; l < 3; l++) { vR[l] = g[GEO_REN + 3 * i + l] - rt[l]; vW[l] = g[GEO_WEN + 3 * i + l]; }
        int e = field_kernel<PER>(L, k, vR, vW, q);
        if (e < 0) err = e;
        CC[i] = q.g * q.aW;
        CC[i + 4] = q.hn;
        F += q.tD;  // node weights are 1
      }
    } else {
      Elem el;
      load_elem(geo, s, el);
      for (int i = 0; i < 9; i++) {
        double z, e, w, N[4];
        fq_gauss9(i, z, e, w);
        bil_rw(el, z, e, vR, vW);
        for (int l = 0; l < 3; l++) vR[l] -= rt[l];
        int st = field_kernel<PER>(L, k, vR, vW, q);
        if (st < 0) err = st;
        bil_N4(z, e, N);
        cplx gw = q.g * (w * q.aW), hw = q.hn * w;
        for (int ep = 0; ep < 4; ep++) { CC[ep] += gw * N[ep]; CC[ep + 4] += hw * N[ep]; }
        F += w * q.tD;
      }
    }
    const double cg = PER ? 1.0 : EL_I_FP;
    for (int i = 0; i < 8; i++) CC[i] = CC[i] * cg;
    F *= EL_I_FP;
  } else {
    // flat triangle: one normal (the node-0 normal / W at the centroid)
    for (int l = 0; l < 3; l++) vW[l] = (type == 0) ? g[GEO_WEN + l] : g[GEO_CW + 3 * l];
    const double aW = vnorm3(vW);
    if (type == 0) {
      for (int i = 0; i < 4; i++) {
        for (int l = 0; l < 3; l++) vR[l] = g[GEO_REN + 3 * i + l] - rt[l];
        int e = field_kernel<PER>(L, k, vR, vW, q);
        if (e < 0) err = e;
        const double w = (i < 3) ? FQ_T4W0 : -FQ_T4W1;
        if (i < 3) {
          CC[i] += q.g * w;
          CC[i + 4] += q.hn * w;
        } else {  // centroid: every shape function is 1/3 there
          double N[3];
          lit_N3(0.0, 0.0, N);
          for (int ep = 0; ep < 3; ep++) { CC[ep] += q.g * (w * N[ep]); CC[ep + 4] += q.hn * (w * N[ep]); }
        }
        F += w * q.tD;
      }
    } else {
      Elem el;
      load_elem(geo, s, el);
      for (int i = 0; i < 7; i++) {
        double z, e, w, N[3];
        fq_tri7(i, z, e, w);
        lit_r(el, z, e, vR);
        for (int l = 0; l < 3; l++) vR[l] -= rt[l];
        int st = field_kernel<PER>(L, k, vR, vW, q);
        if (st < 0) err = st;
        lit_N3(z, e, N);
        for (int ep = 0; ep < 3; ep++) { CC[ep] += q.g * (w * N[ep]); CC[ep + 4] += q.hn * (w * N[ep]); }
        F += w * q.tD;
      }
    }
    const double cg = PER ? 0.5 * aW : FQ_I_EP * aW;
    const double ch = PER ? 0.5 : FQ_I_EP;
    for (int i = 0; i < 3; i++) { CC[i] = CC[i] * cg; CC[i + 4] = CC[i + 4] * ch; }
    F *= FQ_I_EP;
  }
  if (sd < 0) {  // seen from the other side (bil_convert_CC d3qd2_elem.c:927-936)
    for (int i = 4; i < 8; i++) CC[i] = -CC[i];
    F = -F;
  }
  return err;
}

// ---------------------------------------------------------------------------------------------
// Coefficients and their gradients with respect to the point, for the fields computed from the
// derivatives of the potentials (q0_dcoef_rt_grad d3qd2_elem.c:650-682 and dcoef_rt_grad
// :316-349: q0_bil_dcoef_grad.c, q0_lit_dcoef_grad.c, bil_dcoef_grad.c, lit_dcoef_grad.c, types
// 0-3).  dC[p][n] = d CC[n] / d rt_p; dF[p] = dF / d rt_p.  The periodic kernels need the QPGF's
// second derivatives (qpgf_eval2).
struct GradKer {
  cplx g, h, dg[3], dh[3];
  double tD, dF[3];
};

// Kernel values at one quadrature point, R = r(point) - rt, W the normal used by the rule:
// g, h = G and grad G . W; dg, dh their derivatives with respect to R (the rules apply the sign
// of d/d rt); tD = (R . W) / |R|^3 and its derivative dF.  Free space without the 1/(4 pi).
template <bool PER>
BEM_HD int grad_kernel(const QPLattice& L, cplx k, const double* vR, const double* vW, GradKer& o)
{
  const double aR = vnorm3(vR);
  const double i_aR = 1.0 / aR, i3 = i_aR * i_aR * i_aR;
  const double rdW = dot3(vR, vW) * i_aR;
  o.tD = rdW * i_aR * i_aR;
  for (int p = 0; p < 3; p++) o.dF[p] = i3 * (3.0 * vR[p] * i_aR * rdW - vW[p]);
  if (PER) {
    QPVal2 v;
    const int err = qpgf_eval2(L, vR, v);
    o.g = v.G;
    o.h = v.dG[0] * vW[0] + v.dG[1] * vW[1] + v.dG[2] * vW[2];
    const cplx* d2 = v.d2G;  // xx, yy, zz, xy, yz, zx
    o.dh[0] = d2[0] * vW[0] + d2[3] * vW[1] + d2[5] * vW[2];
    o.dh[1] = d2[3] * vW[0] + d2[1] * vW[1] + d2[4] * vW[2];
    o.dh[2] = d2[5] * vW[0] + d2[4] * vW[1] + d2[2] * vW[2];
    for (int p = 0; p < 3; p++) o.dg[p] = v.dG[p];
    return err;
  }
  const cplx kR = k * aR;
  const cplx ca = mul_i(kR), cb = ca - mk(1.0, 0.0);
  const cplx ce = (k.im == 0.0) ? expi(kR.re) : cexp_(ca);
  o.g = ce * i_aR;
  o.h = cb * ce * o.tD;
  const cplx a3 = kR * kR + 3.0 * cb;
  for (int p = 0; p < 3; p++) {
    o.dg[p] = cb * ce * (i_aR * i_aR * vR[p] * i_aR);
    o.dh[p] = ce * i3 * (a3 * (vR[p] * i_aR * rdW) - cb * vW[p]);
  }
  return 0;
}

template <bool PER>
BEM_HD int field_grad_coef(const double* geo, int sd, const double* rt, cplx k, int type, const QPLattice& L,
                           const FieldGL* gl, cplx* CC, cplx (*dC)[8], double& F, double* dF)
{
  for (int i = 0; i < 8; i++) {
    CC[i] = mk(0.0, 0.0);
    for (int p = 0; p < 3; p++) dC[p][i] = mk(0.0, 0.0);
  }
  F = 0.0;
  dF[0] = dF[1] = dF[2] = 0.0;
  if (PER && sd < 0) return -1;
  if (type < 0 || type > 3 || (type >= 2 && !gl)) return -1;
  const int s = sd < 0 ? -sd : sd;
  const double* g = geo + (size_t)s * GEO_STRIDE;
  Elem el;
  load_elem(geo, s, el);
  const int nn = el.nn;
  int err = 0;
  GradKer q;
  double vR[3], vW[3];
  // one quadrature point: weight w, shape-function values N (nn of them), area factor aW (quads)
  auto add = [&](double w, const double* N, double aW) {
    for (int ep = 0; ep < nn; ep++) {
      const double wn = w * N[ep];
      CC[ep] += q.g * (wn * aW);
      CC[ep + 4] += q.h * wn;
      for (int p = 0; p < 3; p++) {
        dC[p][ep] += q.dg[p] * (wn * aW);
        dC[p][ep + 4] += q.dh[p] * wn;
      }
    }
    F += w * q.tD;
    for (int p = 0; p < 3; p++) dF[p] += w * q.dF[p];
  };
  const int n = (type == 2) ? 12 : 64;
  const double* x = (type == 2) ? (gl ? gl->x12 : nullptr) : (gl ? gl->x64 : nullptr);
  const double* wq = (type == 2) ? (gl ? gl->w12 : nullptr) : (gl ? gl->w64 : nullptr);
  double sG, sH, sdG, sdH, sF;  // end scaling of G, H, dG, dH and F parts
  if (nn == 4) {
    if (type == 0) {  // the element's nodes, node weights 1 (q0_bil_dcoef_grad_4p, bil_dcoef_grad_4p)
      for (int i = 0; i < 4; i++) {
        for (int l = 0; l < 3; l++) { vR[l] = g[GEO_REN + 3 * i + l] - rt[l]; vW[l] = g[GEO_WEN + 3 * i + l]; }
        const int st = grad_kernel<PER>(L, k, vR, vW, q);
        if (st < 0) err = st;
        double N[4] = {0.0, 0.0, 0.0, 0.0};
        N[i] = 1.0;
        add(1.0, N, vnorm3(vW));
      }
    } else {
      const int npts = (type == 1) ? 9 : n * n;
      for (int i = 0; i < npts; i++) {
        double z, e, w, N[4];
        if (type == 1) fq_gauss9(i, z, e, w);
        else rule_point(4, n, x, wq, i, z, e, w);
        bil_rw(el, z, e, vR, vW);
        for (int l = 0; l < 3; l++) vR[l] -= rt[l];
        const int st = grad_kernel<PER>(L, k, vR, vW, q);
        if (st < 0) err = st;
        bil_N4(z, e, N);
        add(w, N, vnorm3(vW));
      }
    }
    sG = PER ? 1.0 : EL_I_FP;
    sH = sG;
    sdG = -sG;
    sdH = PER ? -1.0 : EL_I_FP;
    sF = EL_I_FP;
  } else {
    // flat triangle: one normal for the whole element -- the node-0 normal (4-point rules, and the
    // 7-point periodic rule) or W = cw[:, 0] (7-point free-space rule, Gauss-Legendre rules)
    const bool wen0 = (type == 0) || (type == 1 && PER);
    for (int l = 0; l < 3; l++) vW[l] = wen0 ? g[GEO_WEN + l] : g[GEO_CW + 3 * l];
    const double aV = vnorm3(vW);
    if (type == 0) {  // nodes 0-2 (weight 25/48) and the centroid (weight -27/48, shape functions 1/3)
      for (int i = 0; i < 4; i++) {
        for (int l = 0; l < 3; l++) vR[l] = g[GEO_REN + 3 * i + l] - rt[l];
        const int st = grad_kernel<PER>(L, k, vR, vW, q);
        if (st < 0) err = st;
        double N[3] = {0.0, 0.0, 0.0};
        if (i < 3) N[i] = 1.0;
        else lit_N3(0.0, 0.0, N);
        add((i < 3) ? FQ_T4W0 : -FQ_T4W1, N, 1.0);
      }
    } else {
      const int npts = (type == 1) ? 7 : 3 * n * n;
      for (int i = 0; i < npts; i++) {
        double z, e, w, N[3];
        if (type == 1) fq_tri7(i, z, e, w);
        else rule_point(3, n, x, wq, i, z, e, w);
        lit_r(el, z, e, vR);
        for (int l = 0; l < 3; l++) vR[l] -= rt[l];
        const int st = grad_kernel<PER>(L, k, vR, vW, q);
        if (st < 0) err = st;
        lit_N3(z, e, N);
        add(w, N, 1.0);
      }
    }
    if (type <= 1) {
      const double c = PER ? 0.5 : FQ_I_EP;
      sG = c * aV; sH = c; sdG = -c * aV; sdH = PER ? -c : c;
      sF = FQ_I_EP;
    } else {
      const double c = 0.0625 * EL_SQ3 * EL_I_SPSQ3;
      sG = (PER ? 1.0 / 24.0 : c) * aV; sH = PER ? 1.0 / 24.0 : c;
      sdG = -sG; sdH = PER ? -1.0 / 24.0 : c;
      sF = c;
    }
  }
  for (int i = 0; i < 4; i++) {
    CC[i] = CC[i] * sG;
    CC[i + 4] = CC[i + 4] * sH;
    for (int p = 0; p < 3; p++) { dC[p][i] = dC[p][i] * sdG; dC[p][i + 4] = dC[p][i + 4] * sdH; }
  }
  F *= sF;
  for (int p = 0; p < 3; p++) dF[p] *= sF;
  if (sd < 0) {  // seen from the other side (bil_convert_dCC / lit_convert_dCC, d3qd2_elem.c:938-947)
    for (int i = 4; i < 8; i++) {
      CC[i] = -CC[i];
      for (int p = 0; p < 3; p++) dC[p][i] = -dC[p][i];
    }
    F = -F;
    for (int p = 0; p < 3; p++) dF[p] = -dF[p];
  }
  return err;
}

// Solid angle of a flat triangle (or of a quad split into two triangles along 0-2) seen from the
// origin, vertices given relative to the point (fid_calc_solid_angle, d3qd2_setup.c:1351-1422):
// the spherical excess of the triangle of unit vectors, from the angles between the planes
// through the origin and each edge, signed by the orientation.  flag = -1 when the point lies on
// a vertex or in the plane of a sub-triangle (on the boundary).
BEM_HD double sa_plane_angle(const double* na, const double* nb)
{
  double c[3] = {na[1] * nb[2] - na[2] * nb[1], na[2] * nb[0] - na[0] * nb[2], na[0] * nb[1] - na[1] * nb[0]};
  return atan2(vnorm3(c), -dot3(na, nb));
}
BEM_HD void sa_cross(const double* a, const double* b, double* c)
{
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
BEM_HD double solid_angle(int nv, double r[4][3], int& flag)
{
  flag = 0;
  for (int i = 0; i < nv; i++) {
    double a = vnorm3(r[i]);
    if (a == 0.0) { flag = -1; return 0.0; }
    r[i][0] /= a; r[i][1] /= a; r[i][2] /= a;
  }
  double om = 0.0;
  const int ntri = (nv == 4) ? 2 : 1;
  for (int t = 0; t < ntri; t++) {
    const double* p0 = r[0];
    const double* p1 = r[t == 0 ? 1 : 2];
    const double* p2 = r[t == 0 ? 2 : 3];
    double n01[3], n12[3], n20[3];
    sa_cross(p0, p1, n01);
    sa_cross(p1, p2, n12);
    sa_cross(p2, p0, n20);
    const double ex = sa_plane_angle(n01, n20) + sa_plane_angle(n12, n01) + sa_plane_angle(n20, n12) - QP_PI;
    const double D = dot3(p0, n12);
    if (D > 0.0) om += ex;
    else if (D < 0.0) om -= ex;
    else { flag = -1; return 0.0; }
  }
  return om;
}

// self.cuh -- self-element (t == s) coefficients, host+device.
//
// Each routine sums the points q = lane, lane + nlanes, ... of one quadrature piece into a flat
// accumulator, so a CUDA block (lane = threadIdx.x) and a serial host check (lane 0 of 1) run the
// same code; the kernels reduce the partial sums across the block and call the *_combine step.
//
// Periodic (open) domain -- q0_bil_dcoef_bd_vt2_cc_DV (q0_bil_dcoef_v2_cc.c:292-301) and
// q0_lit_dcoef_bd_vt2_cc_DV (q0_lit_dcoef_v2_cc.c:331-342): polar rule of q0_bil_coef_bd
// (q0_bil_coef.c:246-338) / q0_lit_coef_bd (q0_lit_coef.c:297-371) with one Green's function
// evaluation per point shared by all shape functions, plus the free-space solid angle F and
// its central-difference tangential derivatives (q0_bil_dcoef_v2_cc.c:336-454).
//
// Interior domains -- principal-value method: bil_dcoef_bd_vt2_PV (bil_dcoef_v2.c:334-339) =
// bil_coef_bd (bil_coef.c:244-342) + bil_dcoef_bd_tz0_PV / te0_PV (bil_dcoef.c:369-740, integrands
// :916-1630); lit_dcoef_bd_vt2_PV (lit_dcoef_v2.c:366-371) = lit_coef_bd (lit_coef.c:290-348) +
// lit_dcoef_bd_tz0_PV / te0_PV (lit_dcoef.c:461-638, integrands :858-952).  Pieces:
//   1 polar G (and H, F of curved quads)        2 far part D̄ε, r in [DEPS, rm] (64 nodes)
//   3 near disc Dε, r in [0, DEPS]              4 principal-value correction, theta in [0, pi]
#pragma once

#include "elem.cuh"

BEM_HD cplx ccos_(cplx z) { return mk(cos(z.re) * cosh(z.im), -sin(z.re) * sinh(z.im)); }
BEM_HD cplx csin_(cplx z) { return mk(sin(z.re) * cosh(z.im), cos(z.re) * sinh(z.im)); }
BEM_HD void acc_put(double* v, int i, cplx z) { v[2 * i] += z.re; v[2 * i + 1] += z.im; }
BEM_HD cplx acc_get(const double* v, int i) { return mk(v[2 * i], v[2 * i + 1]); }

struct SelfInfo {
  Elem e;
  cplx k;
  double zt, et;
  PolarSet P;
  int bil, curved;
  double Tz[3], Te[3];  // unnormalised tangents at the node
};

// Self integral around the point (zt, et) of element aid (collocation nodes use their own
// parameters; the boundary field of the force evaluation uses other points of the element).
BEM_HD void self_setup_at(const double* geo, int aid, double zt, double et, cplx k, SelfInfo& S)
{
  load_elem(geo, aid, S.e);
  S.k = k;
  S.zt = zt;
  S.et = et;
  polar_setup(S.e.nn, S.zt, S.et, S.P);
  S.bil = (S.e.nn == 4);
  S.curved = S.bil ? !bil_is_plane(S.e) : 0;
  for (int i = 0; i < 3; i++) {
    S.Tz[i] = S.e.cr[i][1] + S.e.cr[i][3] * S.et;
    S.Te[i] = S.e.cr[i][2] + S.e.cr[i][3] * S.zt;
  }
}

BEM_HD void self_setup(const double* geo, int aid, int tn, cplx k, SelfInfo& S)
{
  load_elem(geo, aid, S.e);
  S.k = k;
  S.zt = node_zeta(S.e.nn, tn);
  S.et = node_eta(S.e.nn, tn);
  polar_setup(S.e.nn, S.zt, S.et, S.P);
  S.bil = (S.e.nn == 4);
  S.curved = S.bil ? !bil_is_plane(S.e) : 0;
  for (int i = 0; i < 3; i++) {
    S.Tz[i] = S.e.cr[i][1] + S.e.cr[i][3] * S.et;
    S.Te[i] = S.e.cr[i][2] + S.e.cr[i][3] * S.zt;
  }
}

BEM_HD void self_K(const SelfInfo& S, double r, double cth, double sth, double* K)
{
  if (S.bil) bil_K(S.e, S.zt, S.et, r, cth, sth, K);
  else for (int i = 0; i < 3; i++) K[i] = S.e.cr[i][1] * cth + S.e.cr[i][2] * sth;
}
BEM_HD double self_aW(const SelfInfo& S, double zeta, double eta)
{
  if (!S.bil) return 1.0;
  double W[3];
  for (int i = 0; i < 3; i++) W[i] = S.e.cw[i][0] + S.e.cw[i][1] * zeta + S.e.cw[i][2] * eta;
  return vnorm3(W);
}
BEM_HD void self_N(const SelfInfo& S, double zeta, double eta, double* N)
{
  if (S.bil) bil_N4(zeta, eta, N);
  else { lit_N3(zeta, eta, N); N[3] = 0.0; }
}

// lit_dNn_pr_cs (lit_dcoef.c:845-855)
BEM_HD double lit_dN(int n, double cth, double sth)
{
  const double i_a = 0.5 / EL_P34_N0;
  if (n == 0) return -2.0 / 3.0 * i_a * (cth + EL_SQ3 * sth);
  if (n == 1) return 4.0 / 3.0 * i_a * cth;
  return -2.0 / 3.0 * i_a * (cth - EL_SQ3 * sth);
}

#define SELF_NV 40  // accumulator length of every piece

// ---- interior pieces -------------------------------------------------------------------------
// piece 1 layout: G[4] 0..7, H[4] 8..15, F 16
BEM_HD void self_int_piece1(const SelfInfo& S, const double* xl, const double* wl, const double* xh, const double* wh,
                            int lane, int nlanes, double* v)
{
  const int n = S.P.nsub * 128 * 12;
  for (int q = lane; q < n; q += nlanes) {
    int ir = q % 12, tq = q / 12, j = tq >> 7, m2 = tq & 127;
    double theta, wt;
    polar_theta(S.P, j, m2, xh, wh, theta, wt);
    double rm = polar_rm(S.P, j, theta);
    double cth = cos(theta), sth = sin(theta);
    double r = 0.5 * rm * (xl[ir] + 1.0);
    double w = wt * 0.5 * rm * wl[ir];
    double zeta = r * cth + S.zt, eta = r * sth + S.et;
    double K[3], N[4];
    self_K(S, r, cth, sth, K);
    self_N(S, zeta, eta, N);
    double aK = vnorm3(K);
    cplx kR = S.k * (aK * r);
    cplx ce = cexp_(mul_i(kR));
    cplx g = ce * (w / aK * self_aW(S, zeta, eta));
    for (int i = 0; i < 4; i++) acc_put(v, i, g * N[i]);
    if (S.curved) {
      double i3 = 1.0 / (aK * aK * aK);
      cplx h = mk(-kR.im - 1.0, kR.re) * ce * (w * i3 * cth * sth);  // (i kR - 1) e^{ikR} cs/|K|^3
      for (int i = 0; i < 4; i++) acc_put(v, 4 + i, h * N[i]);
      v[16] += w * i3 * cth * sth;
    }
  }
}

// piece 2 (D̄ε) layout: dGz[4] 0..7, dGe[4] 8..15, dHz[4] 16..23, dHe[4] 24..31, dFz 32, dFe 33
BEM_HD void self_int_piece2(const SelfInfo& S, const double* xh, const double* wh, int lane, int nlanes, double* v)
{
  const int n = S.P.nsub * 128 * 64;
  for (int q = lane; q < n; q += nlanes) {
    int ir = q & 63, tq = q >> 6, j = tq >> 7, m2 = tq & 127;
    double theta, wt;
    polar_theta(S.P, j, m2, xh, wh, theta, wt);
    double rm = polar_rm(S.P, j, theta);
    double cth = cos(theta), sth = sin(theta);
    double r = 0.5 * (rm - EL_DEPS) * xh[ir] + 0.5 * (rm + EL_DEPS);
    double w = wt * 0.5 * (rm - EL_DEPS) * wh[ir];
    double zeta = r * cth + S.zt, eta = r * sth + S.et;
    double K[3], N[4];
    self_K(S, r, cth, sth, K);
    self_N(S, zeta, eta, N);
    double aK = vnorm3(K), i_aK = 1.0 / aK;
    cplx kR = S.k * (aK * r);
    cplx ca = mul_i(kR);
    cplx cb = mk(ca.re - 1.0, ca.im);
    cplx ce = cexp_(ca);
    double KTz = dot3(K, S.Tz), KTe = dot3(K, S.Te);
    cplx gb = cb * ce * (w * i_aK * i_aK / r * self_aW(S, zeta, eta));
    for (int i = 0; i < 4; i++) {
      acc_put(v, i, gb * (KTz * i_aK * N[i]));
      acc_put(v, 4 + i, gb * (KTe * i_aK * N[i]));
    }
    if (S.curved) {
      double aK2 = aK * aK, i5r = 1.0 / (r * aK2 * aK2 * aK);
      cplx kR2p3 = kR * kR + 3.0 * cb;
      cplx hz = ce * (kR2p3 * (KTz * cth) - cb * aK2) * (w * sth * i5r);
      cplx he = ce * (kR2p3 * (KTe * sth) - cb * aK2) * (w * cth * i5r);
      for (int i = 0; i < 4; i++) { acc_put(v, 8 + i, hz * N[i]); acc_put(v, 12 + i, he * N[i]); }
      v[32] += w * sth * i5r * (3.0 * KTz * cth - aK2);
      v[33] += w * cth * i5r * (3.0 * KTe * sth - aK2);
    }
  }
}

// piece 3 (Dε) layout: dGz[4] 0..7, dGe[4] 8..15, dHz[4] 16..23, dHe[4] 24..31
BEM_HD void self_int_piece3(const SelfInfo& S, const double* xl, const double* wl, const double* xh, const double* wh,
                            int lane, int nlanes, double* v)
{
  const cplx k = S.k;
  if (S.bil) {
    // theta in 4 quarter pieces of [-pi, pi] (64 nodes each), r in [0, DEPS] (12 nodes)
    for (int q = lane; q < 4 * 64 * 12; q += nlanes) {
      int ir = q % 12, tq = q / 12, piece = tq >> 6, m = tq & 63;
      double theta = 0.25 * QP_PI * xh[m] + (-0.75 + 0.5 * piece) * QP_PI;
      double w = 0.25 * QP_PI * wh[m] * 0.5 * EL_DEPS * wl[ir];
      double r = 0.5 * EL_DEPS * (xl[ir] + 1.0);
      double cth = cos(theta), sth = sin(theta);
      double zeta = r * cth + S.zt, eta = r * sth + S.et;
      double K[3], N[4];
      self_K(S, r, cth, sth, K);
      self_N(S, zeta, eta, N);
      double aW = self_aW(S, zeta, eta);
      double aK = vnorm3(K), i_aK = 1.0 / aK;
      cplx kR = k * (aK * r);
      cplx ca = mul_i(kR);
      cplx cb = mk(ca.re - 1.0, ca.im);
      cplx cc = ccos_(kR), cs = csin_(kR);
      double KTz = dot3(K, S.Tz), KTe = dot3(K, S.Te);
      cplx gd = (cb * cs + kR * cc) * (w * i_aK * i_aK / r * aW);
      for (int i = 0; i < 4; i++) {
        acc_put(v, i, gd * (KTz * i_aK * N[i]));
        acc_put(v, 4 + i, gd * (KTe * i_aK * N[i]));
      }
      if (S.curved) {
        double aK2 = aK * aK;
        cplx ce = cexp_(ca);
        cplx cbk = mul_i(k);                 // i k
        cplx kkR3 = k * kR + 3.0 * cbk;      // k kR + 3 i k
        double i4 = 1.0 / (aK2 * aK2), i5r = 1.0 / (aK2 * aK2 * aK * r);
        cplx h0z = ce * (kkR3 * (KTz * cth) - cbk * aK2) * i4;
        cplx h1z = cs * ((3.0 * KTz * cth - aK2) * i5r);
        cplx h0e = ce * (kkR3 * (KTe * sth) - cbk * aK2) * i4;
        cplx h1e = cs * ((3.0 * KTe * sth - aK2) * i5r);
        cplx hz = (h0z - mul_i(h1z)) * (w * sth);
        cplx he = (h0e - mul_i(h1e)) * (w * cth);
        for (int i = 0; i < 4; i++) { acc_put(v, 8 + i, hz * N[i]); acc_put(v, 12 + i, he * N[i]); }
      }
    }
  } else {
    // triangle: closed form in r; theta in 4 quarter pieces (64 nodes each)
    for (int q = lane; q < 4 * 64; q += nlanes) {
      int piece = q >> 6, m = q & 63;
      double theta = 0.25 * QP_PI * xh[m] + (-0.75 + 0.5 * piece) * QP_PI;
      double w = 0.25 * QP_PI * wh[m];
      double cth = cos(theta), sth = sin(theta);
      double K[3];
      self_K(S, 0.0, cth, sth, K);
      double aK = vnorm3(K), i_aK = 1.0 / aK;
      cplx keK = k * (EL_DEPS * aK);
      cplx cc = ccos_(keK), cs = csin_(keK);
      // (keK + i) sin + (2 - i keK) cos - 2
      cplx f = mk(keK.re, keK.im + 1.0) * cs + mk(2.0 + keK.im, -keK.re) * cc - mk(2.0, 0.0);
      double i3 = i_aK * i_aK * i_aK;
      for (int i = 0; i < 3; i++) {
        double dn = lit_dN(i, cth, sth);
        acc_put(v, i, f * (w * dn * i3 * dot3(K, S.Tz) * i_aK));
        acc_put(v, 4 + i, f * (w * dn * i3 * dot3(K, S.Te) * i_aK));
      }
    }
  }
}

// piece 4 (principal-value correction) layout as piece 2
BEM_HD void self_int_piece4(const SelfInfo& S, const double* xl, const double* wl, const double* xh, const double* wh,
                            int lane, int nlanes, double* v)
{
  const cplx k = S.k;
  if (S.bil) {
    for (int q = lane; q < 2 * 64 * 12; q += nlanes) {
      int ir = q % 12, tq = q / 12, piece = tq >> 6, m = tq & 63;
      double theta = 0.25 * QP_PI * xh[m] + (0.25 + 0.5 * piece) * QP_PI;
      double w = 0.25 * QP_PI * wh[m] * 0.5 * EL_DEPS * wl[ir];
      double r = 0.5 * EL_DEPS * (xl[ir] + 1.0);
      double cth = cos(theta), sth = sin(theta);
      double zp = r * cth + S.zt, ep = r * sth + S.et, zm = -r * cth + S.zt, em = -r * sth + S.et;
      double Kp[3], Km[3], Np[4], Nm[4];
      bil_K(S.e, S.zt, S.et, r, cth, sth, Kp);
      bil_K(S.e, S.zt, S.et, -r, cth, sth, Km);
      bil_N4(zp, ep, Np);
      bil_N4(zm, em, Nm);
      double aKp = vnorm3(Kp), aKm = vnorm3(Km), aWp = self_aW(S, zp, ep), aWm = self_aW(S, zm, em);
      cplx ccp = ccos_(k * (aKp * r)), ccm = ccos_(k * (aKm * r));
      double KpTz = dot3(Kp, S.Tz), KmTz = dot3(Km, S.Tz), KpTe = dot3(Kp, S.Te), KmTe = dot3(Km, S.Te);
      double ip2 = 1.0 / (aKp * aKp), im2 = 1.0 / (aKm * aKm);
      for (int i = 0; i < 4; i++) {
        cplx gz = ccp * (ip2 * KpTz / aKp * Np[i] * aWp) - ccm * (im2 * KmTz / aKm * Nm[i] * aWm);
        cplx ge = ccp * (ip2 * KpTe / aKp * Np[i] * aWp) - ccm * (im2 * KmTe / aKm * Nm[i] * aWm);
        acc_put(v, i, gz * (w / r));
        acc_put(v, 4 + i, ge * (w / r));
      }
      if (S.curved) {
        double p2 = aKp * aKp, m2 = aKm * aKm;
        double i5p = 1.0 / (p2 * p2 * aKp), i5m = 1.0 / (m2 * m2 * aKm);
        double az_p = (3.0 * KpTz * cth - p2) * i5p, az_m = (3.0 * KmTz * cth - m2) * i5m;
        double ae_p = (3.0 * KpTe * sth - p2) * i5p, ae_m = (3.0 * KmTe * sth - m2) * i5m;
        for (int i = 0; i < 4; i++) {
          acc_put(v, 8 + i, (ccp * (az_p * Np[i]) - ccm * (az_m * Nm[i])) * (w * sth / r));
          acc_put(v, 12 + i, (ccp * (ae_p * Np[i]) - ccm * (ae_m * Nm[i])) * (w * cth / r));
        }
        v[32] += w * sth / r * (az_p - az_m);
        v[33] += w * cth / r * (ae_p - ae_m);
      }
    }
  } else {
    for (int q = lane; q < 2 * 64; q += nlanes) {
      int piece = q >> 6, m = q & 63;
      double theta = 0.25 * QP_PI * xh[m] + (0.25 + 0.5 * piece) * QP_PI;
      double w = 0.25 * QP_PI * wh[m];
      double cth = cos(theta), sth = sin(theta);
      double K[3];
      self_K(S, 0.0, cth, sth, K);
      double aK = vnorm3(K), i_aK = 1.0 / aK;
      cplx cs = csin_(k * (aK * EL_DEPS));
      double i3 = i_aK * i_aK * i_aK;
      for (int i = 0; i < 3; i++) {
        double dn = lit_dN(i, cth, sth);
        acc_put(v, i, cs * (w * dn * i3 * dot3(K, S.Tz) * i_aK));
        acc_put(v, 4 + i, cs * (w * dn * i3 * dot3(K, S.Te) * i_aK));
      }
    }
  }
}

// Combines the four pieces (R[p] = block-summed accumulator of piece p+1) with the reference's
// factors; `negative` flips H, F and their derivatives (bil_convert_CC / _dCC).
BEM_HD void self_int_combine(const SelfInfo& S, const double* R1, const double* R2, const double* R3, const double* R4,
                             int negative, cplx* CC, cplx* dCz, cplx* dCe)
{
  for (int i = 0; i < 9; i++) { CC[i] = mk(0, 0); dCz[i] = mk(0, 0); dCe[i] = mk(0, 0); }
  const double iaTz = 1.0 / vnorm3(S.Tz), iaTe = 1.0 / vnorm3(S.Te);
  const Elem& e = S.e;
  if (S.bil) {
    double bdC = e.cr[0][1] * e.cw[0][2] + e.cr[1][1] * e.cw[1][2] + e.cr[2][1] * e.cw[2][2];
    for (int i = 0; i < 4; i++) {
      CC[i] = acc_get(R1, i) * EL_I_FP;
      // dG = -I_FP/|T| (D̄ε + i Dε - PV)
      dCz[i] = (acc_get(R2, i) + mul_i(acc_get(R3, i)) - acc_get(R4, i)) * (-EL_I_FP * iaTz);
      dCe[i] = (acc_get(R2, 4 + i) + mul_i(acc_get(R3, 4 + i)) - acc_get(R4, 4 + i)) * (-EL_I_FP * iaTe);
    }
    if (S.curved) {
      for (int i = 0; i < 4; i++) {
        CC[4 + i] = acc_get(R1, 4 + i) * (EL_I_FP * bdC);
        dCz[4 + i] = (acc_get(R2, 8 + i) + acc_get(R3, 8 + i) - acc_get(R4, 8 + i)) * (bdC * EL_I_FP * iaTz);
        dCe[4 + i] = (acc_get(R2, 12 + i) + acc_get(R3, 12 + i) - acc_get(R4, 12 + i)) * (bdC * EL_I_FP * iaTe);
      }
      CC[8] = mk(R1[16] * EL_I_FP * bdC, 0);
      dCz[8] = mk((R2[32] + R4[32]) * bdC * EL_I_FP * iaTz, 0);
      dCe[8] = mk((R2[33] + R4[33]) * bdC * EL_I_FP * iaTe, 0);
    }
  } else {
    double V[3] = {e.cw[0][0], e.cw[1][0], e.cw[2][0]};
    double aW = vnorm3(V);
    cplx ik = crecip(S.k);  // 1/k
    for (int i = 0; i < 3; i++) {
      CC[i] = acc_get(R1, i) * (EL_I_SPSQ3 * aW);
      dCz[i] = (acc_get(R2, i) + mul_i(acc_get(R3, i)) * ik - acc_get(R4, i) * ik) * (-EL_I_SPSQ3 * aW * iaTz);
      dCe[i] = (acc_get(R2, 4 + i) + mul_i(acc_get(R3, 4 + i)) * ik - acc_get(R4, 4 + i) * ik) * (-EL_I_SPSQ3 * aW * iaTe);
    }
  }
  if (negative) {
    for (int i = 4; i < 9; i++) { CC[i] = -CC[i]; dCz[i] = -dCz[i]; dCe[i] = -dCe[i]; }
  }
}

// ---- periodic (open-domain) self pair ----------------------------------------------------------
// Layout: G[4] 0..7, H[4] 8..15 (polar rule with the quasi-periodic Green's function), then the
// free-space solid angle of a curved quad at the node and at its four finite-difference
// neighbours (zeta +- h, eta +- h): 16..20.  Returns the first QPGF failure code (0 if none).
// nf: how many solid-angle centres to evaluate (5 for the derivatives of the assembly, 1 when
// only F at the point is needed).
BEM_HD int self_per_points(const SelfInfo& S, const QPLattice& L, const double* xl, const double* wl, const double* xh,
                           const double* wh, int lane, int nlanes, double* v, int nf = 5)
{
  int err = 0;
  const Elem& e = S.e;
  const int npts = S.P.nsub * 128 * 12;
  for (int q = lane; q < npts; q += nlanes) {
    int ir = q % 12, tq = q / 12, j = tq >> 7, m2 = tq & 127;
    double theta, wt;
    polar_theta(S.P, j, m2, xh, wh, theta, wt);
    double rm = polar_rm(S.P, j, theta);
    double cth = cos(theta), sth = sin(theta);
    double r = 0.5 * rm * (xl[ir] + 1.0);
    double w = wt * 0.5 * rm * wl[ir];
    double zeta = r * cth + S.zt, eta = r * sth + S.et;
    double vR[3], W[3], N[4], K[3];
    self_K(S, r, cth, sth, K);
    for (int i = 0; i < 3; i++) {
      vR[i] = r * K[i];
      W[i] = S.bil ? e.cw[i][0] + e.cw[i][1] * zeta + e.cw[i][2] * eta : e.cw[i][0];
    }
    self_N(S, zeta, eta, N);
    QPVal g;
    int e2 = qpgf_eval<QP_BOTH, true>(L, vR, g);
    if (e2 < 0) err = e2;
    double aW = S.bil ? vnorm3(W) : 1.0;
    cplx gw = g.G * (w * aW * r);
    cplx hw = (g.dG[0] * W[0] + g.dG[1] * W[1] + g.dG[2] * W[2]) * (w * r);
    for (int i = 0; i < 4; i++) { acc_put(v, i, gw * N[i]); acc_put(v, 4 + i, hw * N[i]); }
  }
  if (S.bil && S.curved) {
    const double h = EL_CDFH;
    const double cz[5] = {S.zt, S.zt + h, S.zt - h, S.zt, S.zt};
    const double ce[5] = {S.et, S.et, S.et, S.et + h, S.et - h};
    for (int c = 0; c < nf; c++) v[16 + c] += bil_self_F(e, cz[c], ce[c], xl, wl, xh, wh, lane, nlanes);
  }
  return err;
}

BEM_HD void self_per_combine(const SelfInfo& S, const double* R, cplx* CC, cplx* dCz, cplx* dCe)
{
  for (int i = 0; i < 9; i++) { CC[i] = mk(0, 0); dCz[i] = mk(0, 0); dCe[i] = mk(0, 0); }
  const Elem& e = S.e;
  if (S.bil) {
    for (int i = 0; i < 4; i++) { CC[i] = acc_get(R, i); CC[i + 4] = acc_get(R, 4 + i); }
    double bdC = e.cr[0][1] * e.cw[0][2] + e.cr[1][1] * e.cw[1][2] + e.cr[2][1] * e.cw[2][2];
    double s = EL_I_FP * bdC;
    CC[8] = mk(R[16] * s, 0);
    // dF/dt by central differences (q0_bil_dcoef_bd_tz0_cc_DV :336-362, te0 :364-390)
    dCz[8] = mk(1.0 / vnorm3(S.Tz) * (R[17] * s - R[18] * s) / (2.0 * EL_CDFH), 0);
    dCe[8] = mk(1.0 / vnorm3(S.Te) * (R[19] * s - R[20] * s) / (2.0 * EL_CDFH), 0);
  } else {
    double V[3] = {e.cw[0][0], e.cw[1][0], e.cw[2][0]};
    double aV = vnorm3(V);
    for (int i = 0; i < 3; i++) {
      CC[i] = acc_get(R, i) * (2.0 / (3.0 * EL_SQ3) * aV);
      CC[i + 4] = acc_get(R, 4 + i) * (2.0 / (3.0 * EL_SQ3));
    }
  }
}

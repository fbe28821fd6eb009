// self_interior.cu -- self-element (t == s) coefficients of the interior (free-space, complex k)
// domains, one CTA per collocation node.
//
// Follows the reference's principal-value method (SW_DBIEQ == 0):
//   bilinear: bil_dcoef_bd_vt2_PV (bil_dcoef_v2.c:334-339) = bil_coef_bd (bil_coef.c:244-342)
//             + bil_dcoef_bd_tz0_PV / te0_PV (bil_dcoef.c:369-549, 557-740) with integrands
//             bil_sd{G,Hz,He,Fz,Fe}_{Db,De,DP} (bil_dcoef.c:916-1630);
//   triangle: lit_dcoef_bd_vt2_PV (lit_dcoef_v2.c:366-371) = lit_coef_bd (lit_coef.c:290-348)
//             + lit_dcoef_bd_tz0_PV / te0_PV (lit_dcoef.c:461-638) with integrands
//             lit_sdG_{Db,De,DP} (lit_dcoef.c:858-952).
// The tangential derivative is split into the far part D̄ε (r in [DEPS, rm], 64-point rule),
// the near disc Dε (r in [0, DEPS]) and its principal-value correction (PV); each piece is a
// separate strided loop below and the pieces are combined with the reference's factors.
#include <cuda_runtime.h>

#include "elem.cuh"
#include "bem3_internal.h"

// c_xl, c_wl, c_xh, c_wh: Gauss-Legendre tables defined in assemble.cu (same translation unit,
// see bem3_lib.cu).

#define SI_THREADS 256
#define SI_NW (SI_THREADS / 32)

BEM_HD cplx ccos_(cplx z)  // cos(a+ib) = cos a cosh b - i sin a sinh b
{
  return mk(cos(z.re) * cosh(z.im), -sin(z.re) * sinh(z.im));
}
BEM_HD cplx csin_(cplx z)  // sin(a+ib) = sin a cosh b + i cos a sinh b
{
  return mk(sin(z.re) * cosh(z.im), cos(z.re) * sinh(z.im));
}

// block-wide sum of v[0..n) into out (valid in thread 0 after the call); red = [SI_NW][n]
template <int N>
__device__ void block_sum(double* v, double* red, double* out)
{
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < N; i++) {
    double x = v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    v[i] = x;
  }
  if (lane == 0)
    for (int i = 0; i < N; i++) red[wid * N + i] = v[i];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int i = 0; i < N; i++) {
      double s = 0.0;
      for (int w = 0; w < SI_NW; w++) s += red[w * N + i];
      out[i] = s;
    }
  __syncthreads();
}

__device__ __forceinline__ void put(double* v, int i, cplx z) { v[2 * i] += z.re; v[2 * i + 1] += z.im; }
__device__ __forceinline__ cplx get(const double* v, int i) { return mk(v[2 * i], v[2 * i + 1]); }

// lit_dNn_pr_cs (lit_dcoef.c:845-855)
__device__ __forceinline__ double lit_dN(int n, double cth, double sth)
{
  const double i_a = 0.5 / EL_P34_N0;
  if (n == 0) return -2.0 / 3.0 * i_a * (cth + EL_SQ3 * sth);
  if (n == 1) return 4.0 / 3.0 * i_a * cth;
  return -2.0 / 3.0 * i_a * (cth - EL_SQ3 * sth);
}

__global__ void __launch_bounds__(SI_THREADS) k_self_interior(AssembleArgs A, double3* Fself, int* status)
{
  __shared__ double red[SI_NW * 40];
  __shared__ double res[4][40];
  const int row = blockIdx.x;
  const int t = row >> 2, tn = row & 3;
  const int sd = A.sid[t];
  Elem e;
  load_elem(A.geo, abs(sd), e);
  if (tn == 3 && e.nn == 3) return;
  const cplx k = mk(A.kre, A.kim);
  const double zt = node_zeta(e.nn, tn), et = node_eta(e.nn, tn);
  PolarSet P;
  polar_setup(e.nn, zt, et, P);
  const int bil = (e.nn == 4);
  const int curved = bil ? !bil_is_plane(e) : 0;
  // unnormalised tangents (bil_t_zeta / bil_t_eta; lit_t_zeta / lit_t_eta)
  double Tz[3], Te[3];
  for (int i = 0; i < 3; i++) {
    Tz[i] = e.cr[i][1] + e.cr[i][3] * et;
    Te[i] = e.cr[i][2] + e.cr[i][3] * zt;
  }
  const int ns = P.nsub;
  double v[40];

  // ---- part 1: polar coefficients G (and H, F for curved quads) ------------------------------
  for (int i = 0; i < 40; i++) v[i] = 0.0;
  for (int q = threadIdx.x; q < ns * 128 * 12; q += blockDim.x) {
    int ir = q % 12, tq = q / 12, j = tq >> 7, m2 = tq & 127;
    double theta, wt;
    polar_theta(P, j, m2, c_xh, c_wh, theta, wt);
    double rm = polar_rm(P, j, theta);
    double cth = cos(theta), sth = sin(theta);
    double r = 0.5 * rm * (c_xl[ir] + 1.0);
    double w = wt * 0.5 * rm * c_wl[ir];
    double zeta = r * cth + zt, eta = r * sth + et;
    double K[3], N[4];
    if (bil) { bil_K(e, zt, et, r, cth, sth, K); bil_N4(zeta, eta, N); }
    else { for (int i = 0; i < 3; i++) K[i] = e.cr[i][1] * cth + e.cr[i][2] * sth; lit_N3(zeta, eta, N); N[3] = 0.0; }
    double aK = vnorm3(K);
    cplx kR = k * (aK * r);
    cplx ce = cexp_(mul_i(kR));
    double aW = 1.0;
    if (bil) {
      double W[3];
      for (int i = 0; i < 3; i++) W[i] = e.cw[i][0] + e.cw[i][1] * zeta + e.cw[i][2] * eta;
      aW = vnorm3(W);
    }
    cplx g = ce * (w / aK * aW);
    for (int i = 0; i < 4; i++) put(v, i, g * N[i]);
    if (curved) {
      double i3 = 1.0 / (aK * aK * aK);
      cplx h = mk(-kR.im - 1.0, kR.re) * ce * (w * i3 * cth * sth);  // (i kR - 1) e^{ikR} cs/|K|^3
      for (int i = 0; i < 4; i++) put(v, 4 + i, h * N[i]);
      v[16] += w * i3 * cth * sth;
    }
  }
  block_sum<17>(v, red, res[0]);

  // ---- part 2: far part D̄ε, r in [DEPS, rm] (64-point rule) ---------------------------------
  for (int i = 0; i < 40; i++) v[i] = 0.0;
  // layout: dGz[4] 0..7, dGe[4] 8..15, dHz[4] 16..23, dHe[4] 24..31, dFz 32, dFe 33
  for (int q = threadIdx.x; q < ns * 128 * 64; q += blockDim.x) {
    int ir = q & 63, tq = q >> 6, j = tq >> 7, m2 = tq & 127;
    double theta, wt;
    polar_theta(P, j, m2, c_xh, c_wh, theta, wt);
    double rm = polar_rm(P, j, theta);
    double cth = cos(theta), sth = sin(theta);
    double r = 0.5 * (rm - EL_DEPS) * c_xh[ir] + 0.5 * (rm + EL_DEPS);
    double w = wt * 0.5 * (rm - EL_DEPS) * c_wh[ir];
    double zeta = r * cth + zt, eta = r * sth + et;
    double K[3], N[4];
    if (bil) { bil_K(e, zt, et, r, cth, sth, K); bil_N4(zeta, eta, N); }
    else { for (int i = 0; i < 3; i++) K[i] = e.cr[i][1] * cth + e.cr[i][2] * sth; lit_N3(zeta, eta, N); N[3] = 0.0; }
    double aK = vnorm3(K), i_aK = 1.0 / aK;
    cplx kR = k * (aK * r);
    cplx ca = mul_i(kR);
    cplx cb = mk(ca.re - 1.0, ca.im);
    cplx ce = cexp_(ca);
    double aW = 1.0;
    if (bil) {
      double W[3];
      for (int i = 0; i < 3; i++) W[i] = e.cw[i][0] + e.cw[i][1] * zeta + e.cw[i][2] * eta;
      aW = vnorm3(W);
    }
    double KTz = dot3(K, Tz), KTe = dot3(K, Te);
    cplx gb = cb * ce * (w * i_aK * i_aK / r * aW);
    for (int i = 0; i < 4; i++) {
      put(v, i, gb * (KTz * i_aK * N[i]));
      put(v, 4 + i, gb * (KTe * i_aK * N[i]));
    }
    if (curved) {
      double aK2 = aK * aK, i5r = 1.0 / (r * aK2 * aK2 * aK);
      cplx kR2p3 = kR * kR + 3.0 * cb;
      cplx hz = ce * (kR2p3 * (KTz * cth) - cb * aK2) * (w * sth * i5r);
      cplx he = ce * (kR2p3 * (KTe * sth) - cb * aK2) * (w * cth * i5r);
      for (int i = 0; i < 4; i++) { put(v, 8 + i, hz * N[i]); put(v, 12 + i, he * N[i]); }
      v[32] += w * sth * i5r * (3.0 * KTz * cth - aK2);
      v[33] += w * cth * i5r * (3.0 * KTe * sth - aK2);
    }
  }
  block_sum<34>(v, red, res[1]);

  // ---- part 3: near disc Dε ------------------------------------------------------------------
  for (int i = 0; i < 40; i++) v[i] = 0.0;
  if (bil) {
    // theta in 4 quarter pieces of [-pi, pi] (64 nodes each), r in [0, DEPS] (12 nodes)
    for (int q = threadIdx.x; q < 4 * 64 * 12; q += blockDim.x) {
      int ir = q % 12, tq = q / 12, piece = tq >> 6, m = tq & 63;
      double theta = 0.25 * QP_PI * c_xh[m] + (-0.75 + 0.5 * piece) * QP_PI;
      double w = 0.25 * QP_PI * c_wh[m] * 0.5 * EL_DEPS * c_wl[ir];
      double r = 0.5 * EL_DEPS * (c_xl[ir] + 1.0);
      double cth = cos(theta), sth = sin(theta);
      double zeta = r * cth + zt, eta = r * sth + et;
      double K[3], N[4], W[3];
      bil_K(e, zt, et, r, cth, sth, K);
      bil_N4(zeta, eta, N);
      for (int i = 0; i < 3; i++) W[i] = e.cw[i][0] + e.cw[i][1] * zeta + e.cw[i][2] * eta;
      double aW = vnorm3(W);
      double aK = vnorm3(K), i_aK = 1.0 / aK;
      cplx kR = k * (aK * r);
      cplx ca = mul_i(kR);
      cplx cb = mk(ca.re - 1.0, ca.im);
      cplx cc = ccos_(kR), cs = csin_(kR);
      double KTz = dot3(K, Tz), KTe = dot3(K, Te);
      cplx gd = (cb * cs + kR * cc) * (w * i_aK * i_aK / r * aW);
      for (int i = 0; i < 4; i++) {
        put(v, i, gd * (KTz * i_aK * N[i]));
        put(v, 4 + i, gd * (KTe * i_aK * N[i]));
      }
      if (curved) {
        double aK2 = aK * aK;
        cplx ce = cexp_(ca);
        cplx cbk = mul_i(k);                         // i k
        cplx kkR3 = k * kR + 3.0 * cbk;              // k kR + 3 i k
        double i4 = 1.0 / (aK2 * aK2), i5r = 1.0 / (aK2 * aK2 * aK * r);
        cplx h0z = ce * (kkR3 * (KTz * cth) - cbk * aK2) * i4;
        cplx h1z = cs * ((3.0 * KTz * cth - aK2) * i5r);
        cplx h0e = ce * (kkR3 * (KTe * sth) - cbk * aK2) * i4;
        cplx h1e = cs * ((3.0 * KTe * sth - aK2) * i5r);
        cplx hz = (h0z - mul_i(h1z)) * (w * sth);
        cplx he = (h0e - mul_i(h1e)) * (w * cth);
        for (int i = 0; i < 4; i++) { put(v, 8 + i, hz * N[i]); put(v, 12 + i, he * N[i]); }
      }
    }
  } else {
    // triangle: closed form in r; theta in 4 quarter pieces (64 nodes each)
    for (int q = threadIdx.x; q < 4 * 64; q += blockDim.x) {
      int piece = q >> 6, m = q & 63;
      double theta = 0.25 * QP_PI * c_xh[m] + (-0.75 + 0.5 * piece) * QP_PI;
      double w = 0.25 * QP_PI * c_wh[m];
      double cth = cos(theta), sth = sin(theta);
      double K[3];
      for (int i = 0; i < 3; i++) K[i] = e.cr[i][1] * cth + e.cr[i][2] * sth;
      double aK = vnorm3(K), i_aK = 1.0 / aK;
      cplx keK = k * (EL_DEPS * aK);
      cplx cc = ccos_(keK), cs = csin_(keK);
      // (keK + i) sin + (2 - i keK) cos - 2
      cplx f = mk(keK.re, keK.im + 1.0) * cs + mk(2.0 + keK.im, -keK.re) * cc - mk(2.0, 0.0);
      double i3 = i_aK * i_aK * i_aK;
      for (int i = 0; i < 3; i++) {
        double dn = lit_dN(i, cth, sth);
        put(v, i, f * (w * dn * i3 * dot3(K, Tz) * i_aK));
        put(v, 4 + i, f * (w * dn * i3 * dot3(K, Te) * i_aK));
      }
    }
  }
  block_sum<16>(v, red, res[2]);

  // ---- part 4: principal-value correction on [0, DEPS], theta in [0, pi] -----------------------
  for (int i = 0; i < 40; i++) v[i] = 0.0;
  if (bil) {
    for (int q = threadIdx.x; q < 2 * 64 * 12; q += blockDim.x) {
      int ir = q % 12, tq = q / 12, piece = tq >> 6, m = tq & 63;
      double theta = 0.25 * QP_PI * c_xh[m] + (0.25 + 0.5 * piece) * QP_PI;
      double w = 0.25 * QP_PI * c_wh[m] * 0.5 * EL_DEPS * c_wl[ir];
      double r = 0.5 * EL_DEPS * (c_xl[ir] + 1.0);
      double cth = cos(theta), sth = sin(theta);
      double zp = r * cth + zt, ep = r * sth + et, zm = -r * cth + zt, em = -r * sth + et;
      double Kp[3], Km[3], Wp[3], Wm[3], Np[4], Nm[4];
      bil_K(e, zt, et, r, cth, sth, Kp);
      bil_K(e, zt, et, -r, cth, sth, Km);
      for (int i = 0; i < 3; i++) {
        Wp[i] = e.cw[i][0] + e.cw[i][1] * zp + e.cw[i][2] * ep;
        Wm[i] = e.cw[i][0] + e.cw[i][1] * zm + e.cw[i][2] * em;
      }
      bil_N4(zp, ep, Np);
      bil_N4(zm, em, Nm);
      double aKp = vnorm3(Kp), aKm = vnorm3(Km), aWp = vnorm3(Wp), aWm = vnorm3(Wm);
      cplx ccp = ccos_(k * (aKp * r)), ccm = ccos_(k * (aKm * r));
      double KpTz = dot3(Kp, Tz), KmTz = dot3(Km, Tz), KpTe = dot3(Kp, Te), KmTe = dot3(Km, Te);
      double ip2 = 1.0 / (aKp * aKp), im2 = 1.0 / (aKm * aKm);
      for (int i = 0; i < 4; i++) {
        cplx gz = ccp * (ip2 * KpTz / aKp * Np[i] * aWp) - ccm * (im2 * KmTz / aKm * Nm[i] * aWm);
        cplx ge = ccp * (ip2 * KpTe / aKp * Np[i] * aWp) - ccm * (im2 * KmTe / aKm * Nm[i] * aWm);
        put(v, i, gz * (w / r));
        put(v, 4 + i, ge * (w / r));
      }
      if (curved) {
        double p2 = aKp * aKp, m2 = aKm * aKm;
        double i5p = 1.0 / (p2 * p2 * aKp), i5m = 1.0 / (m2 * m2 * aKm);
        double az_p = (3.0 * KpTz * cth - p2) * i5p, az_m = (3.0 * KmTz * cth - m2) * i5m;
        double ae_p = (3.0 * KpTe * sth - p2) * i5p, ae_m = (3.0 * KmTe * sth - m2) * i5m;
        for (int i = 0; i < 4; i++) {
          put(v, 8 + i, (ccp * (az_p * Np[i]) - ccm * (az_m * Nm[i])) * (w * sth / r));
          put(v, 12 + i, (ccp * (ae_p * Np[i]) - ccm * (ae_m * Nm[i])) * (w * cth / r));
        }
        v[32] += w * sth / r * (az_p - az_m);
        v[33] += w * cth / r * (ae_p - ae_m);
      }
    }
  } else {
    for (int q = threadIdx.x; q < 2 * 64; q += blockDim.x) {
      int piece = q >> 6, m = q & 63;
      double theta = 0.25 * QP_PI * c_xh[m] + (0.25 + 0.5 * piece) * QP_PI;
      double w = 0.25 * QP_PI * c_wh[m];
      double cth = cos(theta), sth = sin(theta);
      double K[3];
      for (int i = 0; i < 3; i++) K[i] = e.cr[i][1] * cth + e.cr[i][2] * sth;
      double aK = vnorm3(K), i_aK = 1.0 / aK;
      cplx cs = csin_(k * (aK * EL_DEPS));
      double i3 = i_aK * i_aK * i_aK;
      for (int i = 0; i < 3; i++) {
        double dn = lit_dN(i, cth, sth);
        put(v, i, cs * (w * dn * i3 * dot3(K, Tz) * i_aK));
        put(v, 4 + i, cs * (w * dn * i3 * dot3(K, Te) * i_aK));
      }
    }
  }
  block_sum<34>(v, red, res[3]);

  if (threadIdx.x != 0) return;
  // ---- combine ----------------------------------------------------------------------------------
  cplx CC[9], dCz[9], dCe[9];
  for (int i = 0; i < 9; i++) { CC[i] = mk(0, 0); dCz[i] = mk(0, 0); dCe[i] = mk(0, 0); }
  const double* R1 = res[0];
  const double* R2 = res[1];
  const double* R3 = res[2];
  const double* R4 = res[3];
  const double iaTz = 1.0 / vnorm3(Tz), iaTe = 1.0 / vnorm3(Te);
  if (bil) {
    double bdC = e.cr[0][1] * e.cw[0][2] + e.cr[1][1] * e.cw[1][2] + e.cr[2][1] * e.cw[2][2];
    for (int i = 0; i < 4; i++) {
      CC[i] = get(R1, i) * EL_I_FP;
      // dG: -I_FP/|T| (D̄ε + i Dε - PV)
      dCz[i] = (get(R2, i) + mul_i(get(R3, i)) - get(R4, i)) * (-EL_I_FP * iaTz);
      dCe[i] = (get(R2, 4 + i) + mul_i(get(R3, 4 + i)) - get(R4, 4 + i)) * (-EL_I_FP * iaTe);
    }
    if (curved) {
      for (int i = 0; i < 4; i++) {
        CC[4 + i] = get(R1, 4 + i) * (EL_I_FP * bdC);
        dCz[4 + i] = (get(R2, 8 + i) + get(R3, 8 + i) - get(R4, 8 + i)) * (bdC * EL_I_FP * iaTz);
        dCe[4 + i] = (get(R2, 12 + i) + get(R3, 12 + i) - get(R4, 12 + i)) * (bdC * EL_I_FP * iaTe);
      }
      CC[8] = mk(R1[16] * EL_I_FP * bdC, 0);
      dCz[8] = mk((R2[32] + R4[32]) * bdC * EL_I_FP * iaTz, 0);
      dCe[8] = mk((R2[33] + R4[33]) * bdC * EL_I_FP * iaTe, 0);
    }
  } else {
    double V[3] = {e.cw[0][0], e.cw[1][0], e.cw[2][0]};
    double aW = vnorm3(V);
    cplx ik = crecip(k);  // 1/k
    for (int i = 0; i < 3; i++) {
      CC[i] = get(R1, i) * (EL_I_SPSQ3 * aW);
      dCz[i] = (get(R2, i) + mul_i(get(R3, i)) * ik - get(R4, i) * ik) * (-EL_I_SPSQ3 * aW * iaTz);
      dCe[i] = (get(R2, 4 + i) + mul_i(get(R3, 4 + i)) * ik - get(R4, 4 + i) * ik) * (-EL_I_SPSQ3 * aW * iaTe);
    }
  }
  if (sd < 0) {
    for (int i = 4; i < 9; i++) { CC[i] = -CC[i]; dCz[i] = -dCz[i]; dCe[i] = -dCe[i]; }
  }
  // store (single thread)
  const size_t N = (size_t)4 * A.ne;
  const size_t col = (size_t)4 * t;
  cplx* G = (cplx*)A.G;
  cplx* H = (cplx*)A.H;
  cplx* dG = (cplx*)A.dG;
  cplx* dH = (cplx*)A.dH;
  for (int i = 0; i < 4; i++) {
    G[(size_t)row * N + col + i] = CC[i];
    H[(size_t)row * N + col + i] = CC[4 + i];
    if (dG) {
      dG[(size_t)(2 * row) * N + col + i] = dCz[i];
      dG[(size_t)(2 * row + 1) * N + col + i] = dCe[i];
    }
    if (dH) {
      dH[(size_t)(2 * row) * N + col + i] = dCz[4 + i];
      dH[(size_t)(2 * row + 1) * N + col + i] = dCe[4 + i];
    }
  }
  Fself[row] = make_double3(CC[8].re, dCz[8].re, dCe[8].re);
  (void)status;
}

void bem3_launch_self_interior(const AssembleArgs& A, double3* Fself, int* d_status, cudaStream_t st)
{
  k_self_interior<<<4 * A.ne, SI_THREADS, 0, st>>>(A, Fself, d_status);
}

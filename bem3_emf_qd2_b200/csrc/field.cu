// field.cu -- domain of a point and the electromagnetic field or the modified electromagnetic
// potentials at points off the boundary (d3qd2_src/d3qd2_field.c:10-87, 203-300,
// d3qd2_src/d3qd2_setup.c:157-238), on the device.
//
//   k_domain_id  one warp per point: solid angles of the domains' boundary elements, summed per
//                domain in the reference's domain order (a point on a vertex or in an element's
//                plane belongs to the domain being scanned)
//   k_field_t    one CTA per point: threads stride over the source elements of the point's domain,
//                each evaluating its element's coefficients (field.cuh) and the weighted sums of
//                the boundary values (E, H: EH_s; or U: mEMP_s); a fixed-shape tree reduction
//                makes the result deterministic.
#include "field.cuh"

struct FieldArgs {
  const double* geo;
  const double* rn;
  const int* ed;
  int MN, ps;
  const int* dlist;  // positive element ids of each domain's list, domain by domain
  const int* dsd;    // sub-domain of each of them
  int doff[BEM3_MAXDOM + 1];
  int ne[BEM3_MAXDOM];
  const int* sid[BEM3_MAXDOM];
  const double* E[BEM3_MAXDOM];
  const double* dE[BEM3_MAXDOM];
  const double* H[BEM3_MAXDOM];
  const double* dH[BEM3_MAXDOM];
  const double* U[BEM3_MAXDOM];   // [ne + 1][4][4] complex (potentials at the nodes)
  const double* dU[BEM3_MAXDOM];
  double kn[2 * BEM3_MAXDOM];
  double vk0, vk1, d1x, d1y, d2x, d2y, i_detd;
  const bem3_wave* waves;
  int nwaves;
};

#define FIELD_THREADS 128
#define TWO_PI 6.28318530717958647692

// unit-cell indices of a point (q0_domain_id_l, d3qd2_setup.c:232-238)
__device__ __forceinline__ void cell_of(const FieldArgs& A, const double* rt, int& l1, int& l2)
{
  l1 = (int)floor((rt[0] * A.d2y - rt[1] * A.d2x) * A.i_detd + 0.5);
  l2 = (int)floor(-(rt[0] * A.d1y - rt[1] * A.d1x) * A.i_detd + 0.5);
}

__global__ void k_domain_id(FieldArgs A, int n, const double* __restrict__ r, int* __restrict__ did,
                            int2* __restrict__ cell)
{
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n) return;
  double rt[3] = {r[3 * w], r[3 * w + 1], r[3 * w + 2]};
  int l1 = 0, l2 = 0;
  if (A.ps) {
    cell_of(A, rt, l1, l2);
    rt[0] -= (double)l1 * A.d1x + (double)l2 * A.d2x;
    rt[1] -= (double)l1 * A.d1y + (double)l2 * A.d2y;
  }
  double og[BEM3_MAXDOM];
  for (int d = 0; d < BEM3_MAXDOM; d++) og[d] = 0.0;
  int result = -1;
  for (int d = 0; d <= A.MN; d++) {
    bool hit = false;
    for (int j = A.doff[d] + lane; j < A.doff[d + 1]; j += 32) {
      const int e = A.dlist[j];
      const int nv = (int)A.geo[(size_t)e * GEO_STRIDE + GEO_NN];
      double rv[4][3];
      for (int v = 0; v < 4; v++) {
        const int node = A.ed[4 * e + v];
        for (int k = 0; k < 3; k++) rv[v][k] = A.rn[3 * node + k] - rt[k];
      }
      int flag;
      const double om = solid_angle(nv, rv, flag);
      if (flag < 0) {
        hit = true;
      } else {
        og[d] += om;
        og[A.dsd[j]] -= om;
      }
    }
    if (__any_sync(0xffffffffu, hit)) { result = d; break; }
    double tot = og[d];
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    if (d == 0 && fabs(tot) < TWO_PI) { result = 0; break; }
    if (tot > TWO_PI) { result = d; break; }
  }
  if (lane == 0) {
    did[w] = result;
    cell[w] = make_int2(l1, l2);
  }
}

template <int NV>
__device__ __forceinline__ void block_sum_n(double (*red)[FIELD_THREADS], double* v)
{
  for (int j = 0; j < NV; j++) red[j][threadIdx.x] = v[j];
  __syncthreads();
  for (int o = FIELD_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int j = 0; j < NV; j++) red[j][threadIdx.x] += red[j][threadIdx.x + o];
    __syncthreads();
  }
}

// Incident plane waves at a point (calc_mipw_EH, m_ipw.c:164-179), added to e, h.
__device__ __forceinline__ void add_incident(const FieldArgs& A, const double* r, cplx* e, cplx* h)
{
  for (int wv = 0; wv < A.nwaves; wv++) {
    const bem3_wave& W = A.waves[wv];
    const double te = W.ki * ((r[0] - W.f[0]) * W.sin_t * W.cos_p + (r[1] - W.f[1]) * W.sin_t * W.sin_p +
                              (r[2] - W.f[2]) * W.cos_t);
    const cplx Ee = expi(te);
    for (int i = 0; i < 3; i++) {
      e[i] += mk(W.e[2 * i], W.e[2 * i + 1]) * Ee * W.E0;
      h[i] += mk(W.h[2 * i], W.h[2 * i + 1]) * Ee * W.E0;
    }
  }
}

// POT false: E, H at the points (EH_s, EH_t, EH_i for mode 0, 1, 2; d3qd2_field.c:203-300),
// Eo and Ho [n][3] complex.  POT true: U[4] (mEMP_s, mEMP_t, mEMP_i; d3qd2_field.c:10-87), Eo
// [n][4] complex, Ho unused.  mode 2 sums nothing: the incident field (or its vector potential
// U = (E_inc, 0)) at every point, whatever its domain.
template <bool POT>
__global__ void __launch_bounds__(FIELD_THREADS) k_field_t(FieldArgs A, const __grid_constant__ QPLattice L, int n, const double* __restrict__ r,
                                                          const int* __restrict__ did, const int2* __restrict__ cell,
                                                          int type, int mode, double* __restrict__ Eo,
                                                          double* __restrict__ Ho, int* status)
{
  constexpr int NO = POT ? 4 : 3;  // complex outputs per vector
  const int p = blockIdx.x;
  const int d = did[p];
  const double r_in[3] = {r[3 * p], r[3 * p + 1], r[3 * p + 2]};
  if (mode == 2) {
    if (threadIdx.x != 0) return;
    cplx e[3], h[3];
    for (int i = 0; i < 3; i++) { e[i] = mk(0, 0); h[i] = mk(0, 0); }
    add_incident(A, r_in, e, h);
    for (int i = 0; i < 3; i++) { Eo[2 * NO * p + 2 * i] = e[i].re; Eo[2 * NO * p + 2 * i + 1] = e[i].im; }
    if (POT) { Eo[2 * NO * p + 6] = 0.0; Eo[2 * NO * p + 7] = 0.0; }
    else for (int i = 0; i < 3; i++) { Ho[6 * p + 2 * i] = h[i].re; Ho[6 * p + 2 * i + 1] = h[i].im; }
    return;
  }
  if (d < 0) {
    if (threadIdx.x < 2 * NO) Eo[2 * NO * p + threadIdx.x] = 0.0;
    if (!POT && threadIdx.x < 6) Ho[6 * p + threadIdx.x] = 0.0;
    return;
  }
  const int2 lc = cell[p];
  double rt[3] = {r_in[0], r_in[1], r_in[2]};
  if (A.ps) {
    rt[0] -= (double)lc.x * A.d1x + (double)lc.y * A.d2x;
    rt[1] -= (double)lc.x * A.d1y + (double)lc.y * A.d2y;
  }
  const bool per = (d == 0 && A.ps == 1);
  const cplx k = mk(A.kn[2 * d], A.kn[2 * d + 1]);
  // POT: a[0..3] = U; else a[0..2] = E, a[3..5] = H
  cplx a[6];
  for (int i = 0; i < 6; i++) a[i] = mk(0, 0);
  double F = 0.0;
  const int ne = A.ne[d];
  const int* sid = A.sid[d];
  const double *bE = A.E[d], *bdE = A.dE[d], *bH = A.H[d], *bdH = A.dH[d];
  const double *bU = A.U[d], *bdU = A.dU[d];
  const FieldGL gl = {c_xl, c_wl, c_xh, c_wh};
  for (int s = threadIdx.x; s < ne; s += FIELD_THREADS) {
    cplx CC[8];
    double f;
    const int st = per ? field_coef<true>(A.geo, sid[s], rt, k, type, L, CC, f, &gl)
                       : field_coef<false>(A.geo, sid[s], rt, k, type, L, CC, f, &gl);
    if (st < 0) record_status(status, st);
    if (POT) {
      const size_t b = (size_t)(4 * (s + 1)) * 4;
      for (int nn = 0; nn < 4; nn++)
        for (int i = 0; i < 4; i++) {
          const size_t q = 2 * (b + 4 * nn + i);
          a[i] += CC[nn] * mk(bdU[q], bdU[q + 1]) - CC[nn + 4] * mk(bU[q], bU[q + 1]);
        }
    } else {
      const size_t b = (size_t)(4 * (s + 1)) * 3;
      for (int nn = 0; nn < 4; nn++) {
        for (int i = 0; i < 3; i++) {
          const size_t q = 2 * (b + 3 * nn + i);
          const cplx vdE = mk(bdE[q], bdE[q + 1]), vE = mk(bE[q], bE[q + 1]);
          const cplx vdH = mk(bdH[q], bdH[q + 1]), vH = mk(bH[q], bH[q + 1]);
          a[i] += CC[nn] * vdE - CC[nn + 4] * vE;
          a[3 + i] += CC[nn] * vdH - CC[nn + 4] * vH;
        }
      }
    }
    F += f;
  }
  constexpr int NV = POT ? 9 : 13;
  __shared__ double red[NV][FIELD_THREADS];
  double v[NV];
  for (int i = 0; i < NV - 1; i++) v[i] = (i & 1) ? a[i >> 1].im : a[i >> 1].re;
  v[NV - 1] = F;
  block_sum_n<NV>(red, v);
  if (threadIdx.x != 0) return;
  const double Ft = red[NV - 1][0];
  const double sc = 1.0 / ((d == 0) ? 1.0 + Ft : Ft);
  cplx o[6];
  for (int i = 0; i < (NV - 1) / 2; i++) o[i] = mk(red[2 * i][0], red[2 * i + 1][0]) * sc;
  if (lc.x != 0 || lc.y != 0) {  // Bloch phase of the cell the point lies in
    const double arg = A.vk0 * ((double)lc.x * A.d1x + (double)lc.y * A.d2x) +
                       A.vk1 * ((double)lc.x * A.d1y + (double)lc.y * A.d2y);
    const cplx ce = expi(arg);
    for (int i = 0; i < (NV - 1) / 2; i++) o[i] = o[i] * ce;
  }
  if (mode == 1 && d == 0) {  // total field: the incident waves at the point itself
    cplx e[3], h[3];
    for (int i = 0; i < 3; i++) { e[i] = mk(0, 0); h[i] = mk(0, 0); }
    add_incident(A, r_in, e, h);
    for (int i = 0; i < 3; i++) {
      o[i] += e[i];
      if (!POT) o[3 + i] += h[i];
    }
  }
  for (int i = 0; i < NO; i++) { Eo[2 * NO * p + 2 * i] = o[i].re; Eo[2 * NO * p + 2 * i + 1] = o[i].im; }
  if (!POT)
    for (int i = 0; i < 3; i++) { Ho[6 * p + 2 * i] = o[3 + i].re; Ho[6 * p + 2 * i + 1] = o[3 + i].im; }
}

// E, H from the derivatives of the potentials (EH_mEMP_s / _t / _i for mode 0, 1, 2;
// d3qd2_field.c:89-201).  One CTA per point; threads stride over the source elements with the
// coefficient-gradient rules (field_grad_coef) and sum U[4], dU[3][4] (d/dr of U), F and dF[3].
// A point whose |dF/dr_p| exceeds 10 (CBD_CDF, d3qd2_const.h:84; it lies too close to the
// boundary for these rules) gets zero fields and did = -did (-99 in the open region), as the
// reference returns.  ch = lambda0 / (2 pi i).
#define EHM_CDF 10.0
#define EHM_OPENDID 99
__global__ void __launch_bounds__(FIELD_THREADS) k_eh_memp(FieldArgs A, const __grid_constant__ QPLattice L, int n,
                                                          const double* __restrict__ r, int* __restrict__ did,
                                                          const int2* __restrict__ cell, int type, int mode, double lambda0,
                                                          double* __restrict__ Eo, double* __restrict__ Ho, int* status)
{
  const int p = blockIdx.x;
  const int d = did[p];
  const double r_in[3] = {r[3 * p], r[3 * p + 1], r[3 * p + 2]};
  if (mode == 2 || d < 0) {
    if (threadIdx.x != 0) return;
    cplx e[3], h[3];
    for (int i = 0; i < 3; i++) { e[i] = mk(0, 0); h[i] = mk(0, 0); }
    if (mode == 2) add_incident(A, r_in, e, h);
    for (int i = 0; i < 3; i++) {
      Eo[6 * p + 2 * i] = e[i].re; Eo[6 * p + 2 * i + 1] = e[i].im;
      Ho[6 * p + 2 * i] = h[i].re; Ho[6 * p + 2 * i + 1] = h[i].im;
    }
    return;
  }
  const int2 lc = cell[p];
  double rt[3] = {r_in[0], r_in[1], r_in[2]};
  if (A.ps) {
    rt[0] -= (double)lc.x * A.d1x + (double)lc.y * A.d2x;
    rt[1] -= (double)lc.x * A.d1y + (double)lc.y * A.d2y;
  }
  const bool per = (d == 0 && A.ps == 1);
  const cplx k = mk(A.kn[2 * d], A.kn[2 * d + 1]);
  cplx U[4], dU[3][4];
  for (int i = 0; i < 4; i++) {
    U[i] = mk(0, 0);
    for (int q = 0; q < 3; q++) dU[q][i] = mk(0, 0);
  }
  double F = 0.0, dF[3] = {0.0, 0.0, 0.0};
  const int ne = A.ne[d];
  const int* sid = A.sid[d];
  const double *bU = A.U[d], *bdU = A.dU[d];
  const FieldGL gl = {c_xl, c_wl, c_xh, c_wh};
  for (int s = threadIdx.x; s < ne; s += FIELD_THREADS) {
    cplx CC[8], dC[3][8];
    double f, df[3];
    const int st = per ? field_grad_coef<true>(A.geo, sid[s], rt, k, type, L, &gl, CC, dC, f, df)
                       : field_grad_coef<false>(A.geo, sid[s], rt, k, type, L, &gl, CC, dC, f, df);
    if (st < 0) record_status(status, st);
    const size_t b = (size_t)(4 * (s + 1)) * 4;
    for (int nn = 0; nn < 4; nn++)
      for (int i = 0; i < 4; i++) {
        const size_t q = 2 * (b + 4 * nn + i);
        const cplx vdU = mk(bdU[q], bdU[q + 1]), vU = mk(bU[q], bU[q + 1]);
        U[i] += CC[nn] * vdU - CC[nn + 4] * vU;
        for (int c = 0; c < 3; c++) dU[c][i] += dC[c][nn] * vdU - dC[c][nn + 4] * vU;
      }
    F += f;
    for (int c = 0; c < 3; c++) dF[c] += df[c];
  }
  constexpr int NV = 36;  // U (8), dU (24), F, dF (3)
  __shared__ double red[NV][FIELD_THREADS];
  double v[NV];
  for (int i = 0; i < 4; i++) {
    v[2 * i] = U[i].re; v[2 * i + 1] = U[i].im;
    for (int c = 0; c < 3; c++) { v[8 + 8 * c + 2 * i] = dU[c][i].re; v[9 + 8 * c + 2 * i] = dU[c][i].im; }
  }
  v[32] = F; v[33] = dF[0]; v[34] = dF[1]; v[35] = dF[2];
  block_sum_n<NV>(red, v);
  if (threadIdx.x != 0) return;
  const double Ft = red[32][0], dFt[3] = {red[33][0], red[34][0], red[35][0]};
  cplx e[3], h[3];
  if (fabs(dFt[0]) > EHM_CDF || fabs(dFt[1]) > EHM_CDF || fabs(dFt[2]) > EHM_CDF) {
    for (int i = 0; i < 6; i++) { Eo[6 * p + i] = 0.0; Ho[6 * p + i] = 0.0; }
    did[p] = (d == 0) ? -EHM_OPENDID : -d;
    return;
  }
  const double iC = 1.0 / ((d == 0) ? 1.0 + Ft : Ft);
  cplx u[4], du[3][4];
  for (int i = 0; i < 4; i++) u[i] = mk(red[2 * i][0], red[2 * i + 1][0]) * iC;
  for (int c = 0; c < 3; c++)
    for (int i = 0; i < 4; i++)
      du[c][i] = (mk(red[8 + 8 * c + 2 * i][0], red[9 + 8 * c + 2 * i][0]) - u[i] * dFt[c]) * iC;
  const cplx ch = mk(0.0, -lambda0 / (2.0 * QP_PI));  // lambda0 / (2 pi i)
  for (int c = 0; c < 3; c++) e[c] = u[c] - du[c][3];
  h[0] = ch * (du[1][2] - du[2][1]);
  h[1] = ch * (du[2][0] - du[0][2]);
  h[2] = ch * (du[0][1] - du[1][0]);
  if (lc.x != 0 || lc.y != 0) {
    const double arg = A.vk0 * ((double)lc.x * A.d1x + (double)lc.y * A.d2x) +
                       A.vk1 * ((double)lc.x * A.d1y + (double)lc.y * A.d2y);
    const cplx ce = expi(arg);
    for (int i = 0; i < 3; i++) { e[i] = e[i] * ce; h[i] = h[i] * ce; }
  }
  if (mode == 1 && d == 0) {
    cplx ei[3], hi[3];
    for (int i = 0; i < 3; i++) { ei[i] = mk(0, 0); hi[i] = mk(0, 0); }
    add_incident(A, r_in, ei, hi);
    for (int i = 0; i < 3; i++) { e[i] += ei[i]; h[i] += hi[i]; }
  }
  for (int i = 0; i < 3; i++) {
    Eo[6 * p + 2 * i] = e[i].re; Eo[6 * p + 2 * i + 1] = e[i].im;
    Ho[6 * p + 2 * i] = h[i].re; Ho[6 * p + 2 * i + 1] = h[i].im;
  }
}

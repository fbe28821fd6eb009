// field.cu -- domain of a point and the electromagnetic field at points off the boundary
// (d3qd2_src/d3qd2_field.c:203-285, d3qd2_src/d3qd2_setup.c:157-238), on the device.
//
//   k_domain_id  one warp per point: solid angles of the domains' boundary elements, summed per
//                domain in the reference's domain order (a point on a vertex or in an element's
//                plane belongs to the domain being scanned)
//   k_field      one CTA per point: threads stride over the source elements of the point's domain,
//                each evaluating its element's coefficients (field.cuh) and the weighted sums of
//                the boundary values; a fixed-shape tree reduction makes the result deterministic.
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

__global__ void __launch_bounds__(FIELD_THREADS) k_field(FieldArgs A, const __grid_constant__ QPLattice L, int n, const double* __restrict__ r,
                                                        const int* __restrict__ did, const int2* __restrict__ cell,
                                                        int type, int total, double* __restrict__ Eo,
                                                        double* __restrict__ Ho, int* status)
{
  const int p = blockIdx.x;
  const int d = did[p];
  if (d < 0) {
    if (threadIdx.x < 6) { Eo[6 * p + threadIdx.x] = 0.0; Ho[6 * p + threadIdx.x] = 0.0; }
    return;
  }
  const double r_in[3] = {r[3 * p], r[3 * p + 1], r[3 * p + 2]};
  const int2 lc = cell[p];
  double rt[3] = {r_in[0], r_in[1], r_in[2]};
  if (A.ps) {
    rt[0] -= (double)lc.x * A.d1x + (double)lc.y * A.d2x;
    rt[1] -= (double)lc.x * A.d1y + (double)lc.y * A.d2y;
  }
  const bool per = (d == 0 && A.ps == 1);
  const cplx k = mk(A.kn[2 * d], A.kn[2 * d + 1]);
  cplx e[3], h[3];
  for (int i = 0; i < 3; i++) { e[i] = mk(0, 0); h[i] = mk(0, 0); }
  double F = 0.0;
  const int ne = A.ne[d];
  const int* sid = A.sid[d];
  const double *bE = A.E[d], *bdE = A.dE[d], *bH = A.H[d], *bdH = A.dH[d];
  const FieldGL gl = {c_xl, c_wl, c_xh, c_wh};
  for (int s = threadIdx.x; s < ne; s += FIELD_THREADS) {
    cplx CC[8];
    double f;
    const int st = per ? field_coef<true>(A.geo, sid[s], rt, k, type, L, CC, f, &gl)
                       : field_coef<false>(A.geo, sid[s], rt, k, type, L, CC, f, &gl);
    if (st < 0) record_status(status, st);
    const size_t b = (size_t)(4 * (s + 1)) * 3;
    for (int nn = 0; nn < 4; nn++) {
      for (int i = 0; i < 3; i++) {
        const size_t q = 2 * (b + 3 * nn + i);
        const cplx vdE = mk(bdE[q], bdE[q + 1]), vE = mk(bE[q], bE[q + 1]);
        const cplx vdH = mk(bdH[q], bdH[q + 1]), vH = mk(bH[q], bH[q + 1]);
        e[i] += CC[nn] * vdE - CC[nn + 4] * vE;
        h[i] += CC[nn] * vdH - CC[nn + 4] * vH;
      }
    }
    F += f;
  }
  __shared__ double red[13][FIELD_THREADS];
  double v[13];
  for (int i = 0; i < 3; i++) { v[2 * i] = e[i].re; v[2 * i + 1] = e[i].im; v[6 + 2 * i] = h[i].re; v[7 + 2 * i] = h[i].im; }
  v[12] = F;
  block_sum_n<13>(red, v);
  if (threadIdx.x != 0) return;
  const double Ft = red[12][0];
  const double sc = 1.0 / ((d == 0) ? 1.0 + Ft : Ft);
  cplx Eo3[3], Ho3[3];
  for (int i = 0; i < 3; i++) {
    Eo3[i] = mk(red[2 * i][0], red[2 * i + 1][0]) * sc;
    Ho3[i] = mk(red[6 + 2 * i][0], red[7 + 2 * i][0]) * sc;
  }
  if (lc.x != 0 || lc.y != 0) {  // Bloch phase of the cell the point lies in
    const double arg = A.vk0 * ((double)lc.x * A.d1x + (double)lc.y * A.d2x) +
                       A.vk1 * ((double)lc.x * A.d1y + (double)lc.y * A.d2y);
    const cplx ce = expi(arg);
    for (int i = 0; i < 3; i++) { Eo3[i] = Eo3[i] * ce; Ho3[i] = Ho3[i] * ce; }
  }
  if (total && d == 0) {  // incident plane waves at the point itself (calc_mipw_EH, m_ipw.c:164-179)
    for (int wv = 0; wv < A.nwaves; wv++) {
      const bem3_wave& W = A.waves[wv];
      const double te = W.ki * ((r_in[0] - W.f[0]) * W.sin_t * W.cos_p + (r_in[1] - W.f[1]) * W.sin_t * W.sin_p +
                                (r_in[2] - W.f[2]) * W.cos_t);
      const cplx Ee = expi(te);
      for (int i = 0; i < 3; i++) {
        Eo3[i] += mk(W.e[2 * i], W.e[2 * i + 1]) * Ee * W.E0;
        Ho3[i] += mk(W.h[2 * i], W.h[2 * i + 1]) * Ee * W.E0;
      }
    }
  }
  for (int i = 0; i < 3; i++) {
    Eo[6 * p + 2 * i] = Eo3[i].re; Eo[6 * p + 2 * i + 1] = Eo3[i].im;
    Ho[6 * p + 2 * i] = Ho3[i].re; Ho[6 * p + 2 * i + 1] = Ho3[i].im;
  }
}

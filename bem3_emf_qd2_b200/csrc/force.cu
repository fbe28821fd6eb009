// force.cu -- radiation force and torque on the objects (force_FN, d3qd2_src/d3qd2_force.c:10-240)
// from the Maxwell stress tensor of the total field on the open region's boundary.
//
//   k_force_points  one CTA per (element of the open region, quadrature point): the total field at
//                   the point -- from the boundary values at element nodes, or else by the boundary
//                   field EH_t_bd (d3qd2_field.c:343-385): every other element's nodal-rule
//                   coefficients plus the singular integral of the element itself around the point
//                   (self.cuh, the rule of the periodic self pairs) -- then the point's weighted
//                   stress contributions T.w and (r - rc) x (T.w)
//   k_force_sum     one CTA: the contributions added in a fixed order
//
// Points and weights per element (bil_force_4p/_9p :56-140, lit_force_4p/_7p :142-240):
//   quads,     type 0: the 4 nodes, weight 1, boundary values;        type 1: 3x3 Gauss points
//   triangles, type 0: the 3 nodes (boundary values) + the centroid;   type 1: the 7-point rule
// and the element's sum is scaled by -1 (quads) or -1/2 (triangles).

struct ForceArgs {
  const double* geo;
  int ne;            // elements of the open region
  const int* sid;    // their signed ids
  const double* E;   // boundary values of the open region, [(ne+1)][4][3] complex
  const double* dE;
  const double* H;
  const double* dH;
  double k0re, k0im; // wave number of the open region
  double epd;        // Re(n0)^2
  double rc[3];      // centre of rotation
  int type;          // 0 or 1
  const bem3_wave* waves;
  int nwaves;
};

#define FORCE_THREADS 128
#define FORCE_MAXPTS 9

__device__ __forceinline__ void force_incident(const ForceArgs& A, const double* x, cplx* e, cplx* h)
{
  for (int i = 0; i < 3; i++) { e[i] = mk(0, 0); h[i] = mk(0, 0); }
  for (int wv = 0; wv < A.nwaves; wv++) {
    const bem3_wave& W = A.waves[wv];
    const double te = W.ki * ((x[0] - W.f[0]) * W.sin_t * W.cos_p + (x[1] - W.f[1]) * W.sin_t * W.sin_p +
                              (x[2] - W.f[2]) * W.cos_t);
    const cplx Ee = expi(te);
    for (int i = 0; i < 3; i++) {
      e[i] += mk(W.e[2 * i], W.e[2 * i + 1]) * Ee * W.E0;
      h[i] += mk(W.h[2 * i], W.h[2 * i + 1]) * Ee * W.E0;
    }
  }
}

// quadrature point i of element (nn vertices) for the rule `type`: parameters, weight, and whether
// the field there comes from the node's boundary values
__device__ __forceinline__ int force_point(int nn, int type, int i, double& z, double& e, double& w, bool& node)
{
  node = false;
  if (nn == 4) {
    if (type == 0) {
      if (i >= 4) return 0;
      z = node_zeta(4, i); e = node_eta(4, i); w = 1.0; node = true;
      return 1;
    }
    if (i >= 9) return 0;
    fq_gauss9(i, z, e, w);
    return 1;
  }
  if (type == 0) {
    if (i >= 4) return 0;
    if (i < 3) { z = node_zeta(3, i); e = node_eta(3, i); w = FQ_T4W0; node = true; }
    else { z = 0.0; e = 0.0; w = -FQ_T4W1; }
    return 1;
  }
  if (i >= 7) return 0;
  fq_tri7(i, z, e, w);
  return 1;
}

template <int NV>
__device__ __forceinline__ void fblock_sum(double (*red)[FORCE_THREADS], double* v)
{
  for (int j = 0; j < NV; j++) red[j][threadIdx.x] = v[j];
  __syncthreads();
  for (int o = FORCE_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int j = 0; j < NV; j++) red[j][threadIdx.x] += red[j][threadIdx.x + o];
    __syncthreads();
  }
}

// Scattered field of the open region at the point r = r(z, e) of its element t (0-based position in the
// domain's list, element id at): every other element's coefficients by the rule `type` (0-3, as
// q0_coef_bd takes them for s != t, d3qd2_elem.c), the element itself by the singular rule around
// (z, e) (the periodic self rule, self.cuh), combined with the boundary values and divided by 1 + F
// (EH_s_bd, d3qd2_field.c:299-341).  Called by every thread of a FORCE_THREADS block; the result is
// valid in thread 0.  red: the block's reduction buffer.
__device__ void bd_field_block(const ForceArgs& A, const QPLattice& L, int t, int at, double z, double e,
                               const double* r, int type, int* status, double (*red)[FORCE_THREADS], cplx* es,
                               cplx* hs)
{
  const cplx k = mk(A.k0re, A.k0im);
  cplx ea[3], ha[3];
  for (int l = 0; l < 3; l++) { ea[l] = mk(0, 0); ha[l] = mk(0, 0); }
  double F = 0.0;
  for (int s = threadIdx.x; s < A.ne; s += FORCE_THREADS) {
    if (s == t) continue;
    cplx CC[8];
    double f;
    const int st = field_coef<true>(A.geo, A.sid[s], r, k, type, L, CC, f);
    if (st < 0) record_status(status, st);
    const size_t b = (size_t)(4 * (s + 1)) * 3;
    for (int n = 0; n < 4; n++)
      for (int l = 0; l < 3; l++) {
        const size_t q = 2 * (b + 3 * n + l);
        ea[l] += CC[n] * mk(A.dE[q], A.dE[q + 1]) - CC[n + 4] * mk(A.E[q], A.E[q + 1]);
        ha[l] += CC[n] * mk(A.dH[q], A.dH[q + 1]) - CC[n + 4] * mk(A.H[q], A.H[q + 1]);
      }
    F += f;
  }
  SelfInfo S;
  self_setup_at(A.geo, at, z, e, k, S);
  double sv[24];
  for (int j = 0; j < 24; j++) sv[j] = 0.0;
  const int st = self_per_points(S, L, c_xl, c_wl, c_xh, c_wh, threadIdx.x, FORCE_THREADS, sv, 1);
  if (st < 0) record_status(status, st);
  double v[37];
  for (int l = 0; l < 3; l++) {
    v[2 * l] = ea[l].re; v[2 * l + 1] = ea[l].im; v[6 + 2 * l] = ha[l].re; v[7 + 2 * l] = ha[l].im;
  }
  v[12] = F;
  for (int j = 0; j < 24; j++) v[13 + j] = sv[j];
  fblock_sum<37>(red, v);
  if (threadIdx.x == 0) {
    double R[24];
    for (int j = 0; j < 24; j++) R[j] = red[13 + j][0];
    cplx CC[9], dCz[9], dCe[9];
    self_per_combine(S, R, CC, dCz, dCe);
    for (int l = 0; l < 3; l++) { es[l] = mk(red[2 * l][0], red[2 * l + 1][0]); hs[l] = mk(red[6 + 2 * l][0], red[7 + 2 * l][0]); }
    const size_t b = (size_t)(4 * (t + 1)) * 3;
    for (int n = 0; n < 4; n++)
      for (int l = 0; l < 3; l++) {
        const size_t q = 2 * (b + 3 * n + l);
        es[l] += CC[n] * mk(A.dE[q], A.dE[q + 1]) - CC[n + 4] * mk(A.E[q], A.E[q + 1]);
        hs[l] += CC[n] * mk(A.dH[q], A.dH[q + 1]) - CC[n + 4] * mk(A.H[q], A.H[q + 1]);
      }
    const double sc = 1.0 / (1.0 + red[12][0] + CC[8].re);
    for (int l = 0; l < 3; l++) { es[l] = es[l] * sc; hs[l] = hs[l] * sc; }
  }
  __syncthreads();
}

// Field on the open region's boundary at n points (element position t[i], parameters ze[2 i], ze[2 i + 1]):
// scattered (total 0, EH_s_bd) or plus the incident field (total 1, EH_t_bd, d3qd2_field.c:343-385).
// One block per point; E, H: [n][3] complex.
__global__ void __launch_bounds__(FORCE_THREADS) k_field_bd(ForceArgs A, const __grid_constant__ QPLattice L, int n,
                                                            const int* __restrict__ tl, const double* __restrict__ ze,
                                                            int type, int total, double* __restrict__ E,
                                                            double* __restrict__ H, int* status)
{
  const int i = blockIdx.x;
  if (i >= n) return;
  const int t = tl[i];
  const int at = abs(A.sid[t]);
  const double z = ze[2 * i], e = ze[2 * i + 1];
  Elem el;
  load_elem(A.geo, at, el);
  double r[3];
  if (el.nn == 4) {
    double w[3];
    bil_rw(el, z, e, r, w);
  } else {
    lit_r(el, z, e, r);
  }
  __shared__ double red[37][FORCE_THREADS];
  cplx es[3], hs[3];
  bd_field_block(A, L, t, at, z, e, r, type, status, red, es, hs);
  if (threadIdx.x != 0) return;
  cplx ei[3], hi[3];
  if (total) force_incident(A, r, ei, hi);
  for (int l = 0; l < 3; l++) {
    const cplx ev = total ? es[l] + ei[l] : es[l], hv = total ? hs[l] + hi[l] : hs[l];
    E[6 * (size_t)i + 2 * l] = ev.re; E[6 * (size_t)i + 2 * l + 1] = ev.im;
    H[6 * (size_t)i + 2 * l] = hv.re; H[6 * (size_t)i + 2 * l + 1] = hv.im;
  }
}

__global__ void __launch_bounds__(FORCE_THREADS) k_force_points(ForceArgs A, const __grid_constant__ QPLattice L,
                                                               double* __restrict__ out, int* status)
{
  const int t = blockIdx.x / FORCE_MAXPTS, i = blockIdx.x % FORCE_MAXPTS;
  double* o = out + 6 * (size_t)blockIdx.x;
  const int at = abs(A.sid[t]);
  const double* g = A.geo + (size_t)at * GEO_STRIDE;
  const int nn = (int)g[GEO_NN];
  double z, e, wq;
  bool node;
  if (!force_point(nn, A.type, i, z, e, wq, node)) {
    if (threadIdx.x < 6) o[threadIdx.x] = 0.0;
    return;
  }
  Elem el;
  load_elem(A.geo, at, el);
  double r[3], w[3];
  if (node) {
    for (int l = 0; l < 3; l++) { r[l] = g[GEO_REN + 3 * i + l]; w[l] = g[GEO_WEN + 3 * i + l]; }
  } else if (nn == 4) {
    bil_rw(el, z, e, r, w);
  } else {
    lit_r(el, z, e, r);
    for (int l = 0; l < 3; l++) w[l] = el.cw[l][0];
  }
  __shared__ double red[37][FORCE_THREADS];
  __shared__ double ehs[12];
  if (node) {
    if (threadIdx.x == 0) {
      cplx ei[3], hi[3];
      force_incident(A, r, ei, hi);
      const size_t b = (size_t)(4 * (t + 1) + i) * 3;
      for (int l = 0; l < 3; l++) {
        const cplx ev = mk(A.E[2 * (b + l)], A.E[2 * (b + l) + 1]) + ei[l];
        const cplx hv = mk(A.H[2 * (b + l)], A.H[2 * (b + l) + 1]) + hi[l];
        ehs[2 * l] = ev.re; ehs[2 * l + 1] = ev.im; ehs[6 + 2 * l] = hv.re; ehs[7 + 2 * l] = hv.im;
      }
    }
    __syncthreads();
  } else {
    // boundary field at r (EH_t_bd): other elements by the nodal rule, the element itself by the
    // singular rule around (z, e)
    cplx es[3], hs[3];
    bd_field_block(A, L, t, at, z, e, r, 0, status, red, es, hs);
    if (threadIdx.x == 0) {
      cplx ei[3], hi[3];
      force_incident(A, r, ei, hi);
      for (int l = 0; l < 3; l++) {
        const cplx ev = es[l] + ei[l], hv = hs[l] + hi[l];
        ehs[2 * l] = ev.re; ehs[2 * l + 1] = ev.im; ehs[6 + 2 * l] = hv.re; ehs[7 + 2 * l] = hv.im;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  // Maxwell stress tensor of the total field and the point's weighted contributions
  cplx ev[3], hv[3];
  for (int l = 0; l < 3; l++) { ev[l] = mk(ehs[2 * l], ehs[2 * l + 1]); hv[l] = mk(ehs[6 + 2 * l], ehs[7 + 2 * l]); }
  const double aE2 = abs2(ev[0]) + abs2(ev[1]) + abs2(ev[2]);
  const double aH2 = abs2(hv[0]) + abs2(hv[1]) + abs2(hv[2]);
  const double Tc = 0.25 * (A.epd * aE2 + aH2);
  double T[9];
  for (int j = 0; j < 3; j++)
    for (int k2 = 0; k2 < 3; k2++)
      T[3 * j + k2] = 0.5 * (A.epd * (ev[j] * conj(ev[k2])).re + (hv[j] * conj(hv[k2])).re);
  T[0] -= Tc; T[4] -= Tc; T[8] -= Tc;
  const double sgn = (nn == 4) ? -1.0 : -0.5;
  const double d0 = r[0] - A.rc[0], d1 = r[1] - A.rc[1], d2 = r[2] - A.rc[2];
  for (int j = 0; j < 3; j++) {
    o[j] = sgn * ((T[3 * j + 0] * w[0] + T[3 * j + 1] * w[1] + T[3 * j + 2] * w[2]) * wq);
    o[3 + j] = sgn * (((d1 * T[3 * j + 2] - d2 * T[3 * j + 1]) * w[0] + (d2 * T[3 * j + 0] - d0 * T[3 * j + 2]) * w[1] +
                       (d0 * T[3 * j + 1] - d1 * T[3 * j + 0]) * w[2]) * wq);
  }
}

// Sum of the contributions of all points in a fixed order (one CTA).
__global__ void __launch_bounds__(FORCE_THREADS) k_force_sum(const double* __restrict__ in, int n, double* out)
{
  __shared__ double red[6][FORCE_THREADS];
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int p = threadIdx.x; p < n; p += FORCE_THREADS)
    for (int j = 0; j < 6; j++) v[j] += in[6 * (size_t)p + j];
  fblock_sum<6>(red, v);
  if (threadIdx.x == 0)
    for (int j = 0; j < 6; j++) out[j] = red[j][0];
}

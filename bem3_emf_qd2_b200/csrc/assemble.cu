// assemble.cu -- sm_100a kernels for the coefficient-matrix assembly of one domain
// (the reference's create_cmatrix_domain, d3qd2_src/d3qd2_solve_bieq.c:165-256).
//
// Output layout is the reference's (d3qd2_solve_bieq.c:213-236), N = 4 * Ne_d:
//   G, H   [N][N]     row (t,tn) = 4 t + tn, column (s,i) = 4 s + i        (complex)
//   dG, dH [2N][N]    row 2 (4 t + tn) + {0: d/dt_zeta, 1: d/dt_eta}       (complex)
//   dF     [N][3]     (F or 1+F, dF/dt_zeta, dF/dt_eta)                   (double)
// with 0-based t, s indexing sb[did].sid.  Rows tn = 3 of triangles are left zero, as in
// the reference.
//
// Work decomposition (all FP64, no tensor cores -- none of this is a contraction):
//   k_self_periodic / k_self_interior : one CTA per self pair (t == s), polar rule;
//   k_reg_periodic : one warp per regular pair, lanes over the 144 (quad) / 432 (triangle)
//                    Gauss points, one quasi-periodic Green's function per point;
//   k_reg_interior : one thread per regular pair (free-space kernel, uniform cost);
//   k_gh_*         : pairs whose GL dF/dv exceeds CBD_SDF, recomputed with the 64x64 rule from a
//                    compacted device work list (no host round trip);
//   k_rowsum       : deterministic per-row sums of F, dF/dt over s, H diagonal += (1+)F.
// Regular pairs run in row chunks so that the per-pair F scratch stays bounded.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "self.cuh"
#include "bem3_internal.h"

// ------------------------------------------------------------------------------------------
// Constant tables: Gauss-Legendre nodes (12, 64) and the open-domain lattice.
__constant__ double c_xl[12], c_wl[12], c_xh[64], c_wh[64];

// ------------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int warp_min_i(int v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
template <int N>
__device__ __forceinline__ void warp_sum_arr(double* v)
{
#pragma unroll
  for (int i = 0; i < N; i++) v[i] = warp_sum(v[i]);
}

__device__ __forceinline__ void record_status(int* status, int err)
{
  if (err < 0) atomicCAS(status, 0, err);
}

struct PairIdx {
  int row, s, t, tn;
};
__device__ __forceinline__ PairIdx pair_of(long long p, int ne)
{
  PairIdx q;
  q.row = (int)(p / ne);
  q.s = (int)(p - (long long)q.row * ne);
  q.t = q.row >> 2;
  q.tn = q.row & 3;
  return q;
}

__device__ __forceinline__ void target_info(const double* __restrict__ geo, const int* __restrict__ sid, int t, int tn,
                                            double* rt, double* vtz, double* vte, int& tnn)
{
  int at = abs(sid[t]);
  Elem et;
  load_elem(geo, at, et);
  tnn = et.nn;
  node_tangents(et, tn, vtz, vte);
  const double* g = geo + (size_t)at * GEO_STRIDE + GEO_REN + tn * 3;
  rt[0] = g[0]; rt[1] = g[1]; rt[2] = g[2];
}

// AccP <-> flat array (19 doubles)
__device__ __forceinline__ void accp_pack(const AccP& a, double* v)
{
  for (int i = 0; i < 4; i++) { v[2 * i] = a.G[i].re; v[2 * i + 1] = a.G[i].im; v[8 + 2 * i] = a.H[i].re; v[9 + 2 * i] = a.H[i].im; }
  v[16] = a.F; v[17] = a.dF0; v[18] = a.dF1;
}
__device__ __forceinline__ void accp_unpack(const double* v, AccP& a)
{
  for (int i = 0; i < 4; i++) { a.G[i] = mk(v[2 * i], v[2 * i + 1]); a.H[i] = mk(v[8 + 2 * i], v[9 + 2 * i]); }
  a.F = v[16]; a.dF0 = v[17]; a.dF1 = v[18];
}
// AccI <-> flat array (51 doubles)
__device__ __forceinline__ void acci_pack(const AccI& a, double* v)
{
  for (int i = 0; i < 4; i++) {
    v[2 * i] = a.G[i].re; v[2 * i + 1] = a.G[i].im;
    v[8 + 2 * i] = a.H[i].re; v[9 + 2 * i] = a.H[i].im;
    v[16 + 2 * i] = a.dG0[i].re; v[17 + 2 * i] = a.dG0[i].im;
    v[24 + 2 * i] = a.dH0[i].re; v[25 + 2 * i] = a.dH0[i].im;
    v[32 + 2 * i] = a.dG1[i].re; v[33 + 2 * i] = a.dG1[i].im;
    v[40 + 2 * i] = a.dH1[i].re; v[41 + 2 * i] = a.dH1[i].im;
  }
  v[48] = a.F; v[49] = a.dF0; v[50] = a.dF1;
}
__device__ __forceinline__ void acci_unpack(const double* v, AccI& a)
{
  for (int i = 0; i < 4; i++) {
    a.G[i] = mk(v[2 * i], v[2 * i + 1]); a.H[i] = mk(v[8 + 2 * i], v[9 + 2 * i]);
    a.dG0[i] = mk(v[16 + 2 * i], v[17 + 2 * i]); a.dH0[i] = mk(v[24 + 2 * i], v[25 + 2 * i]);
    a.dG1[i] = mk(v[32 + 2 * i], v[33 + 2 * i]); a.dH1[i] = mk(v[40 + 2 * i], v[41 + 2 * i]);
  }
  a.F = v[48]; a.dF0 = v[49]; a.dF1 = v[50];
}

// Store one pair's coefficients in the reference layout.  Done by lanes of a warp (lane l
// stores item l) or by a single thread (lane = -1 stores all).
__device__ __forceinline__ void store_pair(const AssembleArgs& A, int row, int s, const cplx* CC, const cplx* dCz,
                                           const cplx* dCe, double3* Fp, long long fidx, int lane)
{
  const size_t N = (size_t)4 * A.ne;
  const size_t col = (size_t)4 * s;
  cplx* G = (cplx*)A.G;
  cplx* H = (cplx*)A.H;
  cplx* dG = (cplx*)A.dG;
  cplx* dH = (cplx*)A.dH;
  for (int it = (lane < 0 ? 0 : lane); it < 25; it += (lane < 0 ? 1 : 32)) {
    if (it < 4) G[(size_t)row * N + col + it] = CC[it];
    else if (it < 8) H[(size_t)row * N + col + it - 4] = CC[it];
    else if (it < 12) { if (dG) dG[(size_t)(2 * row) * N + col + it - 8] = dCz[it - 8]; }
    else if (it < 16) { if (dG) dG[(size_t)(2 * row + 1) * N + col + it - 12] = dCe[it - 12]; }
    else if (it < 20) { if (dH) dH[(size_t)(2 * row) * N + col + it - 16] = dCz[it - 12]; }
    else if (it < 24) { if (dH) dH[(size_t)(2 * row + 1) * N + col + it - 20] = dCe[it - 16]; }
    else Fp[fidx] = make_double3(CC[8].re, dCz[8].re, dCe[8].re);
  }
}

// ==========================================================================================
#ifndef REGP_MIN_BLOCKS
#define REGP_MIN_BLOCKS 2  // 2 x 256 threads per SM: 128 registers (measured fastest with register-resident sums)
#endif
// Per-warp pair data in shared memory: the source element and the collocation node with its
// tangents, read by all lanes.  With them and the lanes' sums in shared memory, only a lane's
// current quadrature point stays live in registers across the (out-of-line) lattice sums.
struct RegWarp {
  Elem es;
  double rt[3], vtz[3], vte[3];
};
#define REGP_PAIRS 2  // pairs per warp: 2 x 144 Gauss points = 9 per lane, no ragged last step
#define REGP_SMEM_BYTES (sizeof(RegWarp) * 8 * REGP_PAIRS + sizeof(AccP) * 256 * REGP_PAIRS)

// One warp's unit of regular periodic work: the pairs first, first + 1, ... (REGP_PAIRS of them,
// those < np) of the chunk that starts at pair p0 of the domain.  Lane l takes the points l, l + 32,
// ... of the pairs' concatenated point lists.  sw: the warp's REGP_PAIRS pair slots; sacc: the
// block's per-thread accumulators (shared memory).
__device__ __forceinline__ void reg_periodic_unit(const AssembleArgs& A, const QPLattice& L, long long p0, long long np,
                                                  long long first, double3* Fp, unsigned* gh_list, unsigned* gh_count,
                                                  unsigned gh_cap, int* status, RegWarp* sw, AccP (*sacc)[256], int lane)
{
  int npts[REGP_PAIRS];
  PairIdx q[REGP_PAIRS];
  __syncwarp();  // a warp that runs several units reuses its slots: the last unit's reads are done
#pragma unroll
  for (int j = 0; j < REGP_PAIRS; j++) {
    npts[j] = 0;
    if (first + j >= np) continue;
    q[j] = pair_of(p0 + first + j, A.ne);
    const int at = abs(A.sid[q[j].t]);
    const int tnn = (int)A.geo[(size_t)at * GEO_STRIDE + GEO_NN];
    if ((q[j].tn == 3 && tnn == 3) || q[j].s == q[j].t) continue;
    RegWarp& W = sw[j];
    if (lane == 0) {
      int tn_unused;
      target_info(A.geo, A.sid, q[j].t, q[j].tn, W.rt, W.vtz, W.vte, tn_unused);
      load_elem(A.geo, abs(A.sid[q[j].s]), W.es);
    }
    const int sn = (int)A.geo[(size_t)abs(A.sid[q[j].s]) * GEO_STRIDE + GEO_NN];
    npts[j] = (sn == 4) ? 144 : 432;
    accp_zero(sacc[j][threadIdx.x]);
  }
  __syncwarp();
  const int ntot = npts[0] + (REGP_PAIRS > 1 ? npts[1] : 0);
  int err = 0, nterms = 0;
  for (int k = lane; k < ntot; k += 32) {
    const int j = (k < npts[0]) ? 0 : 1;
    const int kk = j ? k - npts[0] : k;
    const RegWarp& W = sw[j];
    double z, e, wt;
    rule_point(W.es.nn, 12, c_xl, c_wl, kk, z, e, wt);
    int e2 = accp_point(W.es, L, W.rt, W.vtz, W.vte, z, e, wt, sacc[j][threadIdx.x]);
    if (e2 < 0) err = e2;
    else nterms += e2;
  }
  err = warp_min_i(err);
  if (lane == 0) record_status(status, err);
  if (A.terms) {
    double tc = warp_sum((double)nterms);
    if (lane == 0) atomicAdd(A.terms, (unsigned long long)tc);
  }
#pragma unroll 1
  for (int j = 0; j < REGP_PAIRS; j++) {
    if (npts[j] == 0) continue;  // uniform across the warp
    // Warp totals of the 19 sums (AccP is 19 doubles: G, H interleaved re/im, F, dF0, dF1): lane
    // i < 19 adds component i over the warp's 32 shared-memory slots, then writes it to slot 0,
    // which every lane reads for the one item it stores.  No per-thread arrays: the scaled
    // coefficients never leave registers or shared memory.
    double* acc = reinterpret_cast<double*>(&sacc[j][threadIdx.x & ~31]);
    static_assert(sizeof(AccP) == 19 * sizeof(double), "AccP is read as 19 doubles");
    __syncwarp();  // every lane's last accumulation is visible to the others
    double tot = 0.0;
    if (lane < 19) {
      double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
      for (int t = 0; t < 32; t += 4) {
        s0 += acc[(t + 0) * 19 + lane];
        s1 += acc[(t + 1) * 19 + lane];
        s2 += acc[(t + 2) * 19 + lane];
        s3 += acc[(t + 3) * 19 + lane];
      }
      tot = (s0 + s1) + (s2 + s3);
    }
    __syncwarp();
    if (lane < 19) acc[lane] = tot;
    __syncwarp();
    // the scalings of accp_finish: quads as summed; triangles G |W| / 24, H / 24
    double gs = 1.0, hs = 1.0, fs = EL_I_FP;
    if (sw[j].es.nn != 4) {
      const double V[3] = {sw[j].es.cw[0][0], sw[j].es.cw[1][0], sw[j].es.cw[2][0]};
      gs = 1.0 / (24.0) * vnorm3(V);
      hs = 1.0 / (24.0);
      fs = 0.0625 * EL_SQ3 * EL_I_SPSQ3;
    }
    const double dFz = acc[17] * fs, dFe = acc[18] * fs;
    const long long pi = first + j;
    if (needs_gh(dFz, dFe)) {
      if (lane == 0) {
        unsigned slot = atomicAdd(gh_count, 1u);
        if (slot < gh_cap) gh_list[slot] = (unsigned)pi;
        else record_status(status, -900);
      }
      continue;
    }
    // lane it stores item it of store_pair's order: G[0..3], H[0..3], the (zero) dG and dH rows, F
    const size_t N = (size_t)4 * A.ne, col = (size_t)4 * q[j].s, row = (size_t)q[j].row;
    const int it = lane;
    if (it < 4) {
      ((cplx*)A.G)[row * N + col + it] = mk(acc[2 * it] * gs, acc[2 * it + 1] * gs);
    } else if (it < 8) {
      ((cplx*)A.H)[row * N + col + it - 4] = mk(acc[2 * it] * hs, acc[2 * it + 1] * hs);
    } else if (it < 16) {
      if (A.dG) ((cplx*)A.dG)[(2 * row + (it >= 12)) * N + col + (it & 3)] = mk(0, 0);
    } else if (it < 24) {
      if (A.dH) ((cplx*)A.dH)[(2 * row + (it >= 20)) * N + col + (it & 3)] = mk(0, 0);
    } else if (it == 24) {
      Fp[pi] = make_double3(acc[16] * fs, dFz, dFe);
    }
    __syncwarp();  // slot 0 is rewritten by the next pair's accumulation only after every read
  }
}

// Regular periodic pairs of one chunk: one warp per REGP_PAIRS consecutive pairs.
__global__ void __launch_bounds__(256, REGP_MIN_BLOCKS) k_reg_periodic(AssembleArgs A, const __grid_constant__ QPLattice L,
                                                                       long long p0, long long np, double3* Fp,
                                                                       unsigned* gh_list, unsigned* gh_count,
                                                                       unsigned gh_cap, int* status)
{
  extern __shared__ __align__(16) unsigned char regp_smem[];  // REGP_SMEM_BYTES
  RegWarp(*sw)[REGP_PAIRS] = reinterpret_cast<RegWarp(*)[REGP_PAIRS]>(regp_smem);
  AccP(*sacc)[256] = reinterpret_cast<AccP(*)[256]>(regp_smem + sizeof(RegWarp) * 8 * REGP_PAIRS);
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const long long first = w * REGP_PAIRS;  // pair index within the chunk
  if (first >= np) return;  // uniform across the warp
  reg_periodic_unit(A, L, p0, np, first, Fp, gh_list, gh_count, gh_cap, status, sw[wib], sacc, lane);
}

// Near-singular periodic pair w of the chunk starting at pair p0, 64x64 rule, by the whole CTA
// (256 threads; red, serr: its shared reduction slots).  Every thread of the CTA calls it.
__device__ __forceinline__ void gh_periodic_pair(const AssembleArgs& A, const QPLattice& L, long long p0, long long w,
                                                 double3* Fp, int* status, double (*red)[19], int* serr)
{
  {
    PairIdx q = pair_of(p0 + w, A.ne);
    int tnn;
    double rt[3], vtz[3], vte[3];
    target_info(A.geo, A.sid, q.t, q.tn, rt, vtz, vte, tnn);
    Elem es;
    load_elem(A.geo, abs(A.sid[q.s]), es);
    AccP a;
    accp_zero(a);
    int err = 0;
    const int npts = (es.nn == 4) ? 4096 : 3 * 4096;
    for (int k = threadIdx.x; k < npts; k += blockDim.x) {
      double z, e, wt;
      rule_point(es.nn, 64, c_xh, c_wh, k, z, e, wt);
      int e2 = accp_point(es, L, rt, vtz, vte, z, e, wt, a);
      if (e2 < 0) err = e2;
    }
    double v[19];
    accp_pack(a, v);
    warp_sum_arr<19>(v);
    err = warp_min_i(err);
    int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { for (int i = 0; i < 19; i++) red[wid][i] = v[i]; serr[wid] = err; }
    __syncthreads();
    if (wid == 0) {
      for (int i = 0; i < 19; i++) v[i] = (lane < 8) ? red[lane][i] : 0.0;
      warp_sum_arr<19>(v);
      int e3 = warp_min_i(lane < 8 ? serr[lane] : 0);
      if (lane == 0) record_status(status, e3);
      accp_unpack(v, a);
      cplx CC[9], dCz[9], dCe[9];
      accp_finish(es, a, CC, dCz, dCe);
      store_pair(A, q.row, q.s, CC, dCz, dCe, Fp, w, lane);
    }
    __syncthreads();
  }
}

// Near-singular periodic pairs of one chunk: one CTA per listed pair.  The list holds at most
// gh_cap entries (the counter keeps counting past it; the regular kernel then reports -900).
__global__ void __launch_bounds__(256, 2) k_gh_periodic(AssembleArgs A, const __grid_constant__ QPLattice L, long long p0, double3* Fp,
                                                     const unsigned* gh_list, const unsigned* gh_count, unsigned gh_cap,
                                                     int* status)
{
  __shared__ double red[8][19];
  __shared__ int serr[8];
  const unsigned n = min(*gh_count, gh_cap);
  for (unsigned it = blockIdx.x; it < n; it += gridDim.x) gh_periodic_pair(A, L, p0, gh_list[it], Fp, status, red, serr);
}

// ==========================================================================================
// Regular interior pair w of the chunk starting at pair p0, by one thread.
__device__ __forceinline__ void reg_interior_pair(const AssembleArgs& A, long long p0, long long w, double3* Fp,
                                                  unsigned* gh_list, unsigned* gh_count, unsigned gh_cap, int* status)
{
  long long p = p0 + w;
  PairIdx q = pair_of(p, A.ne);
  int tnn;
  double rt[3], vtz[3], vte[3];
  target_info(A.geo, A.sid, q.t, q.tn, rt, vtz, vte, tnn);
  if ((q.tn == 3 && tnn == 3) || q.s == q.t) return;
  int sd = A.sid[q.s];
  Elem es;
  load_elem(A.geo, abs(sd), es);
  const int npts = (es.nn == 4) ? 144 : 432;
  const cplx k = mk(A.kre, A.kim);
  AccI a;
  acci_zero(a);
  for (int kq = 0; kq < npts; kq++) {
    double z, e, wt;
    rule_point(es.nn, 12, c_xl, c_wl, kq, z, e, wt);
    acci_point(es, k, rt, vtz, vte, z, e, wt, a);
  }
  cplx CC[9], dCz[9], dCe[9];
  acci_finish(es, a, sd < 0, CC, dCz, dCe);
  if (needs_gh(dCz[8].re, dCe[8].re)) {
    unsigned slot = atomicAdd(gh_count, 1u);
    if (slot < gh_cap) gh_list[slot] = (unsigned)w;
    else record_status(status, -900);
    return;
  }
  store_pair(A, q.row, q.s, CC, dCz, dCe, Fp, w, -1);
}

// Regular interior pairs of one chunk: one thread per pair.
__global__ void __launch_bounds__(128) k_reg_interior(AssembleArgs A, long long p0, long long np, double3* Fp,
                                                      unsigned* gh_list, unsigned* gh_count, unsigned gh_cap, int* status)
{
  long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= np) return;
  reg_interior_pair(A, p0, w, Fp, gh_list, gh_count, gh_cap, status);
}

// Near-singular interior pair w of the chunk starting at pair p0, 64x64 rule, by one warp.
__device__ __forceinline__ void gh_interior_pair(const AssembleArgs& A, long long p0, long long w, double3* Fp, int lane)
{
  const cplx k = mk(A.kre, A.kim);
  {
    PairIdx q = pair_of(p0 + w, A.ne);
    int tnn;
    double rt[3], vtz[3], vte[3];
    target_info(A.geo, A.sid, q.t, q.tn, rt, vtz, vte, tnn);
    int sd = A.sid[q.s];
    Elem es;
    load_elem(A.geo, abs(sd), es);
    const int npts = (es.nn == 4) ? 4096 : 3 * 4096;
    AccI a;
    acci_zero(a);
    for (int kq = lane; kq < npts; kq += 32) {
      double z, e, wt;
      rule_point(es.nn, 64, c_xh, c_wh, kq, z, e, wt);
      acci_point(es, k, rt, vtz, vte, z, e, wt, a);
    }
    double v[51];
    acci_pack(a, v);
    warp_sum_arr<51>(v);
    acci_unpack(v, a);
    cplx CC[9], dCz[9], dCe[9];
    acci_finish(es, a, sd < 0, CC, dCz, dCe);
    store_pair(A, q.row, q.s, CC, dCz, dCe, Fp, w, lane);
  }
}

// Near-singular interior pairs of one chunk: one warp per listed pair (at most gh_cap of them).
__global__ void __launch_bounds__(256) k_gh_interior(AssembleArgs A, long long p0, double3* Fp, const unsigned* gh_list,
                                                     const unsigned* gh_count, unsigned gh_cap)
{
  const unsigned n = min(*gh_count, gh_cap);
  const int lane = threadIdx.x & 31;
  const unsigned wglob = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nw = (gridDim.x * blockDim.x) >> 5;
  for (unsigned it = wglob; it < n; it += nw) gh_interior_pair(A, p0, gh_list[it], Fp, lane);
}

// ==========================================================================================
// Row sums (d3qd2_solve_bieq.c:222-236): F, dF/dtz, dF/dte over all s (regular pairs from the
// chunk scratch, the self pair from Fself), then H[row][4t+tn] += (did==0 ? 1 : 0) + F.
// One warp per row; lane-strided partial sums and a fixed-shape reduction (deterministic).
// fr: the row's F terms (ne of them, indexed by s).
__device__ __forceinline__ void rowsum_row(const AssembleArgs& A, int row, const double3* fr, const double3* Fself, int lane)
{
  int t = row >> 2, tn = row & 3;
  int at = abs(A.sid[t]);
  int tnn = (int)A.geo[(size_t)at * GEO_STRIDE + GEO_NN];
  if (tn == 3 && tnn == 3) return;
  double f0 = 0, f1 = 0, f2 = 0;
  for (int s = lane; s < A.ne; s += 32) {
    if (s == t) continue;
    double3 v = fr[s];
    f0 += v.x; f1 += v.y; f2 += v.z;
  }
  f0 = warp_sum(f0); f1 = warp_sum(f1); f2 = warp_sum(f2);
  if (lane == 0) {
    double3 sv = Fself[row];
    f0 += sv.x; f1 += sv.y; f2 += sv.z;
    double diag = (A.did == 0) ? 1.0 + f0 : f0;
    cplx* H = (cplx*)A.H;
    size_t N = (size_t)4 * A.ne;
    H[(size_t)row * N + 4 * (size_t)t + tn].re += diag;
    if (A.dF) {
      A.dF[3 * (size_t)row + 0] = diag;
      A.dF[3 * (size_t)row + 1] = f1;
      A.dF[3 * (size_t)row + 2] = f2;
    }
  }
}

__global__ void k_rowsum(AssembleArgs A, int row0, int nrows, const double3* Fp, const double3* Fself)
{
  int wr = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (wr >= nrows) return;
  rowsum_row(A, row0 + wr, Fp + (size_t)wr * A.ne, Fself, lane);
}

// ==========================================================================================
// Self pairs of the periodic domain (q0_bil_dcoef_bd_vt2_cc_DV q0_bil_dcoef_v2_cc.c:292-301 and
// q0_lit_dcoef_bd_vt2_cc_DV q0_lit_dcoef_v2_cc.c:331-342).  One CTA per (t, tn); the point loop
// and the combination are self_per_points / self_per_combine (self.cuh).
#define SELF_THREADS 256
// Row `row` (= 4 t + tn) of the periodic domain, by the whole CTA (SELF_THREADS threads).
__device__ __forceinline__ void self_periodic_row(const AssembleArgs& A, const QPLattice& L, int row, double3* Fself,
                                                  int* status, double (*red)[24], int* serr)
{
  const int t = row >> 2, tn = row & 3;
  SelfInfo S;
  self_setup(A.geo, abs(A.sid[t]), tn, mk(0.0, 0.0), S);
  if (tn == 3 && S.e.nn == 3) return;
  double v[24];
  for (int i = 0; i < 24; i++) v[i] = 0.0;
  int err = self_per_points(S, L, c_xl, c_wl, c_xh, c_wh, threadIdx.x, blockDim.x, v);
  warp_sum_arr<24>(v);
  err = warp_min_i(err);
  int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { for (int i = 0; i < 24; i++) red[wid][i] = v[i]; serr[wid] = err; }
  __syncthreads();
  if (wid != 0) return;
  for (int i = 0; i < 24; i++) v[i] = (lane < SELF_THREADS / 32) ? red[lane][i] : 0.0;
  warp_sum_arr<24>(v);
  int e3 = warp_min_i(lane < SELF_THREADS / 32 ? serr[lane] : 0);
  if (lane != 0) return;
  record_status(status, e3);
  cplx CC[9], dCz[9], dCe[9];
  self_per_combine(S, v, CC, dCz, dCe);
  store_pair(A, row, t, CC, dCz, dCe, Fself, row, -1);
}

__global__ void __launch_bounds__(SELF_THREADS, 2) k_self_periodic(AssembleArgs A, const __grid_constant__ QPLattice L, double3* Fself, int* status)
{
  __shared__ double red[SELF_THREADS / 32][24];
  __shared__ int serr[SELF_THREADS / 32];
  self_periodic_row(A, L, blockIdx.x, Fself, status, red, serr);
}

// ==========================================================================================
// Host side
static void gauleg_host(int n, double* x, double* w)
{
  // Gauss-Legendre nodes on [-1,1] by Newton iteration on P_n from the Chebyshev-like initial
  // guess, with the stop tolerance of the reference's gauleg (com_src/gauleg.c:3-36) so that the
  // tables agree bit for bit (near-singular pairs are sensitive to the last bits of the nodes).
  for (int i = 0; i < (n + 1) / 2; i++) {
    double z = cos(QP_PI * (i + 0.75) / (n + 0.5)), z1, pp;
    for (int it = 0; it < 100; it++) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; j++) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
      if (fabs(z - z1) <= 3.0e-16) break;
    }
    x[i] = -z;
    x[n - 1 - i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    w[n - 1 - i] = w[i];
  }
}

static int g_tables_ready[64];

static int ensure_tables(void)
{
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && g_tables_ready[dev]) return 0;
  double xl[12], wl[12], xh[64], wh[64];
  gauleg_host(12, xl, wl);
  gauleg_host(64, xh, wh);
  if (cudaMemcpyToSymbol(c_xl, xl, sizeof xl) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_wl, wl, sizeof wl) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_xh, xh, sizeof xh) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_wh, wh, sizeof wh) != cudaSuccess) return -1;
  // k_reg_periodic keeps ~80 KB of shared memory per block (dynamic, above the 48 KB static
  // limit): allow it, and ask for the largest carve-out so the L1 split does not cut occupancy
  if (cudaFuncSetAttribute(k_reg_periodic, cudaFuncAttributePreferredSharedMemoryCarveout,
                           (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess ||
      cudaFuncSetAttribute(k_reg_periodic, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)REGP_SMEM_BYTES) !=
          cudaSuccess)
    return -1;
  if (dev < 64) g_tables_ready[dev] = 1;
  return 0;
}

extern "C" void bem3_gauss_legendre(int n, double* x, double* w) { gauleg_host(n, x, w); }

// Scratch layout of bem3_assemble_run for a chunk of `rows` rows, each part starting on a 256-byte
// boundary: self-pair F sums (4 ne double3), the work-list counters (256 B), the chunk's per-pair F
// terms (rows * ne double3), the near-singular work list (rows * ne / 8 + 4096 u32).
static inline size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }
struct ScratchLayout {
  size_t fself, counters, fp, gh_list, end;
  unsigned gh_cap;
};
static ScratchLayout scratch_layout(int ne, int rows)
{
  ScratchLayout l;
  const size_t np = (size_t)rows * ne;
  l.gh_cap = (unsigned)(np / 8 + 4096);
  l.fself = 0;
  l.counters = round256((size_t)4 * ne * sizeof(double3));
  l.fp = l.counters + 256;
  l.gh_list = l.fp + round256(np * sizeof(double3));
  l.end = l.gh_list + round256((size_t)l.gh_cap * sizeof(unsigned));
  return l;
}
size_t bem3_scratch_bytes(int ne, int rows) { return scratch_layout(ne, rows).end; }

// Runs the whole domain on `stream` using caller-provided scratch (see bem3_scratch_bytes).
// Returns 0, or a negative code (see bem3_qd2_b200.h).
// Adds a chunk's near-singular count to the domain's total (no host round trip per chunk).
__global__ void k_acc_count(const unsigned* __restrict__ cnt, unsigned long long* __restrict__ total)
{
  *total += *cnt;
}

int bem3_assemble_run(const AssembleArgs& A, const QPLattice* L, void* scratch, size_t scratch_bytes, int rows_per_chunk,
                      int* d_status, cudaStream_t st, AssembleStats* stats, const ChunkHook* hook)
{
  if (ensure_tables() != 0) return BEM3_ERR_CUDA;
  const int ne = A.ne;
  const int nrows = 4 * ne;
  if (rows_per_chunk <= 0 || rows_per_chunk > nrows) rows_per_chunk = nrows;
  const ScratchLayout lay = scratch_layout(ne, rows_per_chunk);
  if (lay.end > scratch_bytes) return BEM3_ERR_SCRATCH;  // every part below ends inside the scratch
  char* base = (char*)scratch;
  double3* Fself = (double3*)(base + lay.fself);
  unsigned* gh_count = (unsigned*)(base + lay.counters);                          // this chunk's list length
  unsigned long long* gh_total = (unsigned long long*)(base + lay.counters + 8);  // the domain's total
  double3* Fp = (double3*)(base + lay.fp);
  unsigned* gh_list = (unsigned*)(base + lay.gh_list);
  const unsigned gh_cap = lay.gh_cap;

  const size_t N = (size_t)nrows;
  if (cudaMemsetAsync(A.G, 0, N * N * 16, st) != cudaSuccess) return BEM3_ERR_CUDA;
  if (cudaMemsetAsync(A.H, 0, N * N * 16, st) != cudaSuccess) return BEM3_ERR_CUDA;
  if (A.dG && cudaMemsetAsync(A.dG, 0, 2 * N * N * 16, st) != cudaSuccess) return BEM3_ERR_CUDA;
  if (A.dH && cudaMemsetAsync(A.dH, 0, 2 * N * N * 16, st) != cudaSuccess) return BEM3_ERR_CUDA;
  if (A.dF && cudaMemsetAsync(A.dF, 0, N * 3 * sizeof(double), st) != cudaSuccess) return BEM3_ERR_CUDA;
  cudaMemsetAsync(Fself, 0, N * sizeof(double3), st);
  cudaMemsetAsync(gh_total, 0, sizeof(unsigned long long), st);

  int launches = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  const bool timing = stats && stats->time_kernels;
  if (timing) { cudaEventCreate(&ev0); cudaEventCreate(&ev1); }
  // profiling only: the duration of the kernels launched since tic() goes to class_ms[cls]
  auto tic = [&]() { if (timing) cudaEventRecord(ev0, st); };
  auto toc = [&](int cls) -> float {
    float ms = 0.f;
    if (timing) {
      cudaEventRecord(ev1, st);
      cudaEventSynchronize(ev1);
      cudaEventElapsedTime(&ms, ev0, ev1);
      stats->class_ms[cls] += ms;
    }
    return ms;
  };
  // self pairs
  tic();
  if (A.periodic) k_self_periodic<<<nrows, SELF_THREADS, 0, st>>>(A, *L, Fself, d_status);
  else bem3_launch_self_interior(A, Fself, d_status, st);
  toc(0);
  launches++;

  for (int r0 = 0; r0 < nrows; r0 += rows_per_chunk) {
    int nr = (r0 + rows_per_chunk <= nrows) ? rows_per_chunk : nrows - r0;
    long long p0 = (long long)r0 * ne, np = (long long)nr * ne;
    cudaMemsetAsync(gh_count, 0, sizeof(unsigned), st);
    if (A.periodic) {
      long long threads = (np + REGP_PAIRS - 1) / REGP_PAIRS * 32;
      unsigned blocks = (unsigned)((threads + 255) / 256);
      tic();
      k_reg_periodic<<<blocks, 256, REGP_SMEM_BYTES, st>>>(A, *L, p0, np, Fp, gh_list, gh_count, gh_cap, d_status);
      const float ms = toc(1);
      if (timing) {
        stats->reg_periodic_ms += ms;
        stats->reg_periodic_launches++;
      }
      tic();
      k_gh_periodic<<<148 * 4, 256, 0, st>>>(A, *L, p0, Fp, gh_list, gh_count, gh_cap, d_status);
      toc(2);
    } else {
      unsigned blocks = (unsigned)((np + 127) / 128);
      tic();
      k_reg_interior<<<blocks, 128, 0, st>>>(A, p0, np, Fp, gh_list, gh_count, gh_cap, d_status);
      toc(1);
      tic();
      k_gh_interior<<<148 * 4, 256, 0, st>>>(A, p0, Fp, gh_list, gh_count, gh_cap);
      toc(2);
    }
    tic();
    k_rowsum<<<(nr * 32 + 255) / 256, 256, 0, st>>>(A, r0, nr, Fp, Fself);
    toc(3);
    k_acc_count<<<1, 1, 0, st>>>(gh_count, gh_total);
    launches += 4;
    if (hook) hook->fn(hook->user, r0, nr, st);
  }
  if (timing) { cudaEventDestroy(ev0); cudaEventDestroy(ev1); }
  if (stats) {
    stats->launches += launches;
    stats->d_gh_total = gh_total;
  }
  if (cudaGetLastError() != cudaSuccess) return BEM3_ERR_CUDA;
  return 0;
}

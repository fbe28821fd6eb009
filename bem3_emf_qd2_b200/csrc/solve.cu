// solve.cu -- device solve stage after the assembly (d3qd2_src/d3qd2_solve_bieq.c:258-1030):
//   k_build_rows    global system of the modified potentials, 8 NN unknowns
//                   (create_matrix_csr_dac :284-421; dense rows instead of the CSR temp files)
//   cuSOLVER LU     replaces PARDISO (d3qd2_mkl_solver.c:18-148)
//   k_store_bv      scatter to U, dU per domain (tmatrix_bd_store :456-544)
//   k_eh_interior   E, H on the boundary from U, dU and the tangential-derivative rows
//                   (q1_solve_eh_bv :931-1030 with dudt_fcm :617-637, inv_matrix_33 :639-660)
//   k_deh_system    per-domain system G [dE dH] = H [E H] (solve_deh_bv :662-791), cuSOLVER LU
// Every array below is device memory.  Complex values are interleaved (re, im) doubles.
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include "elem.cuh"
#include "bem3_internal.h"
#include "bem3_solve.h"

__device__ __forceinline__ cplx ldc(const double* p, size_t i) { return mk(p[2 * i], p[2 * i + 1]); }
__device__ __forceinline__ void stc(double* p, size_t i, cplx v) { p[2 * i] = v.re; p[2 * i + 1] = v.im; }

// unit normal at an element node (n_bd_node, d3qd2_elem.c:38-44)
__device__ __forceinline__ void node_normal(const double* geo, int aeid, int l, double* vn)
{
  const double* g = geo + (size_t)aeid * GEO_STRIDE + GEO_WEN + 3 * l;
  vn[0] = g[0]; vn[1] = g[1]; vn[2] = g[2];
  unit3(vn);
}

// One CTA per global row.  Row order as create_tmatrix_csr (:271-273): did, cid (0..3), t, tn,
// skipping tn = 3 of triangles.  rowmap[r] = (did, cid, t, tn) packed by the host.
__global__ void k_build_rows(SolveDev S, const int4* __restrict__ rowmap, double* __restrict__ A, double* __restrict__ B,
                             long long na)
{
  const long long r = blockIdx.x;
  const int4 m = rowmap[r];
  const int did = m.x, cid = m.y, t = m.z, tn = m.w;
  const int ne = S.ne[did];
  const size_t N = (size_t)4 * ne;
  const double* G = S.G[did] + 2 * ((size_t)(4 * t + tn) * N);
  const double* H = S.H[did] + 2 * ((size_t)(4 * t + tn) * N);
  const int* sid = S.sid_h[did];
  double* Arow = A + 2 * (size_t)r * (size_t)na;  // row-major, complex
  const size_t nn = (size_t)S.NN;
  cplx bsum = mk(0, 0);
  for (int s = threadIdx.x; s < ne; s += blockDim.x) {
    const int sd = sid[s];
    const int asd = abs(sd);
    const int mdid = S.md[asd], sdid = S.sd[asd];
    const int nv = (int)S.geo[(size_t)asd * GEO_STRIDE + GEO_NN];
    const int* eni = S.eni + 4 * asd;
    if (did == mdid) {
      for (int l = 0; l < nv; l++) {
        stc(Arow, nn * (cid + 0) + eni[l], ldc(H, 4 * s + l));
        stc(Arow, nn * (cid + 4) + eni[l], -ldc(G, 4 * s + l));
      }
    } else {
      cplx k1 = mk(S.kn[2 * mdid], S.kn[2 * mdid + 1]), k2 = mk(S.kn[2 * sdid], S.kn[2 * sdid + 1]);
      cplx k12 = k1 * k1, k22 = k2 * k2;
      cplx delt = k12 - k22, beps = cdiv(k12, k22), sigm = mk(1.0 - beps.re, -beps.im);
      for (int l = 0; l < nv; l++) {
        double vn[3];
        node_normal(S.geo, asd, l, vn);
        cplx g = ldc(G, 4 * s + l), h = ldc(H, 4 * s + l);
        const double* ui = S.Ui + 2 * ((size_t)(4 * asd + l) * 4);
        const double* dui = S.dUi + 2 * ((size_t)(4 * asd + l) * 4);
        if (cid < 3) {
          stc(Arow, nn * cid + eni[l], h);
          stc(Arow, nn * 3 + eni[l], delt * (vn[cid] * g));
          stc(Arow, nn * (cid + 4) + eni[l], g);
          if (mdid == 0) bsum = bsum - h * ldc(ui, cid) - g * ldc(dui, cid);
        } else {
          stc(Arow, nn * 0 + eni[l], sigm * (vn[0] * g));
          stc(Arow, nn * 1 + eni[l], sigm * (vn[1] * g));
          stc(Arow, nn * 2 + eni[l], sigm * (vn[2] * g));
          stc(Arow, nn * 3 + eni[l], h);
          stc(Arow, nn * 7 + eni[l], beps * g);
          if (mdid == 0) {
            cplx nu = ldc(ui, 0) * vn[0] + ldc(ui, 1) * vn[1] + ldc(ui, 2) * vn[2];
            bsum = bsum - sigm * g * nu;
          }
        }
      }
    }
  }
  // deterministic block reduction of the right-hand side
  __shared__ double red[2][256];
  red[0][threadIdx.x] = bsum.re;
  red[1][threadIdx.x] = bsum.im;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red[0][threadIdx.x] += red[0][threadIdx.x + o];
      red[1][threadIdx.x] += red[1][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) stc(B, r, mk(red[0][0], red[1][0]));
}

// tmatrix_bd_store (:456-544): one thread per (domain position s, node l).
__global__ void k_store_bv(SolveDev S, int d, const double* __restrict__ X)
{
  const int ne = S.ne[d];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 4 * ne) return;
  const int s = q >> 2, l = q & 3;
  const int sd = S.sid_h[d][s], asd = abs(sd);
  const int mdid = S.md[asd], sdid = S.sd[asd];
  const int nv = (int)S.geo[(size_t)asd * GEO_STRIDE + GEO_NN];
  if (l >= nv) return;
  const size_t nn = (size_t)S.NN;
  const int e = S.eni[4 * asd + l];
  double* U = S.U[d] + 2 * ((size_t)(4 * (s + 1) + l) * 4);
  double* dU = S.dU[d] + 2 * ((size_t)(4 * (s + 1) + l) * 4);
  if (d == mdid) {
    for (int i = 0; i < 4; i++) {
      stc(U, i, ldc(X, nn * i + e));
      stc(dU, i, ldc(X, nn * (i + 4) + e));
    }
    return;
  }
  cplx k1 = mk(S.kn[2 * mdid], S.kn[2 * mdid + 1]), k2 = mk(S.kn[2 * sdid], S.kn[2 * sdid + 1]);
  cplx k12 = k1 * k1, k22 = k2 * k2;
  cplx delt = k12 - k22, beps = cdiv(k12, k22), sigm = mk(1.0 - beps.re, -beps.im);
  double n[3];
  node_normal(S.geo, asd, l, n);
  cplx tU[4], tUi[3];
  tU[3] = ldc(X, nn * 3 + e);
  const double* ui = S.Ui + 2 * ((size_t)(4 * asd + l) * 4);
  const double* dui = S.dUi + 2 * ((size_t)(4 * asd + l) * 4);
  for (int i = 0; i < 3; i++) {
    tU[i] = ldc(X, nn * i + e);
    cplx u = tU[i];
    cplx du = -(ldc(X, nn * (i + 4) + e) + delt * tU[3] * n[i]);
    if (mdid == 0) {
      tUi[i] = ldc(ui, i);
      u += tUi[i];
      du -= ldc(dui, i);
    }
    stc(U, i, u);
    stc(dU, i, du);
  }
  stc(U, 3, tU[3]);
  cplx dphi = -(beps * ldc(X, nn * 7 + e) + sigm * (tU[0] * n[0] + tU[1] * n[1] + tU[2] * n[2]));
  if (mdid == 0) dphi -= sigm * (tUi[0] * n[0] + tUi[1] * n[1] + tUi[2] * n[2]);
  stc(dU, 3, dphi);
}

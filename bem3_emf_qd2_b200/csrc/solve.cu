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

// inv_matrix_33 (:639-660): rows of the inverse of [vn; vtz; vte] as the reference lays them out
__device__ __forceinline__ void inv33(const double* vn, const double* vtz, const double* vte, double* ma)
{
  double i_det = 1.0 / (vn[0] * vtz[1] * vte[2] + vn[1] * vtz[2] * vte[0] + vn[2] * vtz[0] * vte[1] -
                        (vn[2] * vtz[1] * vte[0] + vn[1] * vtz[0] * vte[2] + vn[0] * vtz[2] * vte[1]));
  ma[0] = vtz[1] * vte[2] - vtz[2] * vte[1];
  ma[1] = -vn[1] * vte[2] + vn[2] * vte[1];
  ma[2] = vn[1] * vtz[2] - vn[2] * vtz[1];
  ma[3] = -vtz[0] * vte[2] + vtz[2] * vte[0];
  ma[4] = vn[0] * vte[2] - vn[2] * vte[0];
  ma[5] = -vn[0] * vtz[2] + vn[2] * vtz[0];
  ma[6] = vtz[0] * vte[1] - vtz[1] * vte[0];
  ma[7] = -vn[0] * vte[1] + vn[1] * vte[0];
  ma[8] = vn[0] * vtz[1] - vn[1] * vtz[0];
  for (int i = 0; i < 9; i++) ma[i] *= i_det;
}

// q1_solve_eh_bv (:931-1030) for interior domain d: one warp per collocation node (t, tn).
// dudt_fcm (:617-637) is the two row dot products over the domain's tangential-derivative rows.
__global__ void k_eh_interior(SolveDev S, int d)
{
  const int ne = S.ne[d];
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= 4 * ne) return;
  const int t = w >> 2, tn = w & 3;
  const int at = S.sid_h[d][t], atd = abs(at);
  Elem el;
  load_elem(S.geo, atd, el);
  if (tn == 3 && el.nn == 3) return;
  const size_t N = (size_t)4 * ne;
  const double* rz = S.dG[d] + 2 * ((size_t)(2 * (4 * t + tn) + 0) * N);
  const double* re = S.dG[d] + 2 * ((size_t)(2 * (4 * t + tn) + 1) * N);
  const double* hz = S.dH[d] + 2 * ((size_t)(2 * (4 * t + tn) + 0) * N);
  const double* he = S.dH[d] + 2 * ((size_t)(2 * (4 * t + tn) + 1) * N);
  const double* U = S.U[d];
  const double* dU = S.dU[d];
  cplx dUz[4], dUe[4];
  for (int i = 0; i < 4; i++) { dUz[i] = mk(0, 0); dUe[i] = mk(0, 0); }
  for (int c = lane; c < 4 * ne; c += 32) {
    const int s = c >> 2, sn = c & 3;
    cplx gz = ldc(rz, c), ge = ldc(re, c), hzz = ldc(hz, c), hee = ldc(he, c);
    const size_t b = (size_t)(4 * (s + 1) + sn) * 4;
    for (int i = 0; i < 4; i++) {
      cplx du = ldc(dU, b + i), u = ldc(U, b + i);
      dUz[i] += gz * du - hzz * u;
      dUe[i] += ge * du - hee * u;
    }
  }
  for (int i = 0; i < 4; i++) {
    for (int o = 16; o > 0; o >>= 1) {
      dUz[i].re += __shfl_xor_sync(0xffffffffu, dUz[i].re, o);
      dUz[i].im += __shfl_xor_sync(0xffffffffu, dUz[i].im, o);
      dUe[i].re += __shfl_xor_sync(0xffffffffu, dUe[i].re, o);
      dUe[i].im += __shfl_xor_sync(0xffffffffu, dUe[i].im, o);
    }
  }
  if (lane != 0) return;
  const double* tdF = S.dF[d] + 3 * (size_t)(4 * t + tn);
  const size_t me = (size_t)(4 * (t + 1) + tn) * 4;
  for (int i = 0; i < 4; i++) {
    cplx u = ldc(U, me + i);
    dUz[i] = (dUz[i] - u * tdF[1]) * (1.0 / tdF[0]);
    dUe[i] = (dUe[i] - u * tdF[2]) * (1.0 / tdF[0]);
  }
  double vtz[3], vte[3], vn[3], a[9];
  node_tangents(el, tn, vtz, vte);
  const double sig = at < 0 ? -1.0 : 1.0;
  const double* wn = S.geo + (size_t)atd * GEO_STRIDE + GEO_WEN + 3 * tn;
  for (int i = 0; i < 3; i++) vn[i] = sig * wn[i];
  unit3(vn);
  inv33(vn, vtz, vte, a);
  const cplx ch = mk(S.ch_re, S.ch_im);
  cplx dUt[4], Ut[4];
  for (int i = 0; i < 4; i++) { dUt[i] = ldc(dU, me + i); Ut[i] = ldc(U, me + i); }
  const size_t me3 = (size_t)(4 * (t + 1) + tn) * 3;
  for (int i = 0; i < 3; i++)
    stc(S.E[d], me3 + i, -(dUt[3] * a[i * 3 + 0] + dUz[3] * a[i * 3 + 1] + dUe[3] * a[i * 3 + 2]) + Ut[i]);
  // H = ch * curl of the potential, written with the rows of a (:987-992)
  cplx Hv[3];
  Hv[0] = ch * ((dUt[2] * a[3] + dUz[2] * a[4] + dUe[2] * a[5]) - (dUt[1] * a[6] + dUz[1] * a[7] + dUe[1] * a[8]));
  Hv[1] = ch * ((dUt[0] * a[6] + dUz[0] * a[7] + dUe[0] * a[8]) - (dUt[2] * a[0] + dUz[2] * a[1] + dUe[2] * a[2]));
  Hv[2] = ch * ((dUt[1] * a[0] + dUz[1] * a[1] + dUe[1] * a[2]) - (dUt[0] * a[3] + dUz[0] * a[4] + dUe[0] * a[5]));
  for (int i = 0; i < 3; i++) stc(S.H_[d], me3 + i, Hv[i]);
  // open-region side of the same node (scattered field, :995-1020)
  if (S.md[atd] == 0) {
    const int s0 = S.pos0[atd];
    const size_t o4 = (size_t)(4 * (s0 + 1) + tn) * 4, o3 = (size_t)(4 * (s0 + 1) + tn) * 3;
    const double* pz = S.dEiz + 2 * ((size_t)(4 * atd + tn) * 3);
    const double* pe = S.dEie + 2 * ((size_t)(4 * atd + tn) * 3);
    cplx dU0[4], U0[4], gz[3], ge[3];
    for (int i = 0; i < 4; i++) { dU0[i] = ldc(S.dU[0], o4 + i); U0[i] = ldc(S.U[0], o4 + i); }
    for (int i = 0; i < 3; i++) { gz[i] = dUz[i] - ldc(pz, i); ge[i] = dUe[i] - ldc(pe, i); }
    for (int i = 0; i < 3; i++)
      stc(S.E[0], o3 + i, -(-dU0[3] * a[i * 3 + 0] + dUz[3] * a[i * 3 + 1] + dUe[3] * a[i * 3 + 2]) + U0[i]);
    cplx H0[3];
    H0[0] = ch * ((-dU0[2] * a[3] + gz[2] * a[4] + ge[2] * a[5]) - (-dU0[1] * a[6] + gz[1] * a[7] + ge[1] * a[8]));
    H0[1] = ch * ((-dU0[0] * a[6] + gz[0] * a[7] + ge[0] * a[8]) - (-dU0[2] * a[0] + gz[2] * a[1] + ge[2] * a[2]));
    H0[2] = ch * ((-dU0[1] * a[0] + gz[1] * a[1] + ge[1] * a[2]) - (-dU0[0] * a[3] + gz[0] * a[4] + ge[0] * a[5]));
    for (int i = 0; i < 3; i++) stc(S.H_[0], o3 + i, H0[i]);
  }
}

// solve_deh_bv (:662-791), system of domain d: rows and columns run over the domain's element
// nodes in order (triangle node 3 skipped).  cmap[c] = 4 s + sn for compacted index c.
// A row-major (transposed for the column-major solver), B column-major [6][nn].
__global__ void k_deh_system(SolveDev S, int d, const int* __restrict__ cmap, int nn, double* A, double* B)
{
  const int c = blockIdx.x;  // compacted row
  const int src = cmap[c];   // 4 t + tn
  const int ne = S.ne[d];
  const size_t N = (size_t)4 * ne;
  const double* G = S.G[d] + 2 * ((size_t)src * N);
  const double* H = S.H[d] + 2 * ((size_t)src * N);
  double* Ar = A ? A + 2 * (size_t)c * nn : nullptr;  // A == nullptr: right-hand sides only
  cplx acc[6];
  for (int j = 0; j < 6; j++) acc[j] = mk(0, 0);
  for (int r = threadIdx.x; r < nn; r += blockDim.x) {
    const int col = cmap[r];
    if (Ar) stc(Ar, r, ldc(G, col));
    const int s = col >> 2, sn = col & 3;
    cplx h = ldc(H, col);
    const size_t b3 = (size_t)(4 * (s + 1) + sn) * 3;
    for (int i = 0; i < 3; i++) {
      acc[i] += h * ldc(S.E[d], b3 + i);
      acc[3 + i] += h * ldc(S.H_[d], b3 + i);
    }
  }
  __shared__ double red[12][256];
  for (int j = 0; j < 6; j++) { red[2 * j][threadIdx.x] = acc[j].re; red[2 * j + 1][threadIdx.x] = acc[j].im; }
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int j = 0; j < 12; j++) red[j][threadIdx.x] += red[j][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int j = 0; j < 6; j++) stc(B, (size_t)j * nn + c, mk(red[2 * j][0], red[2 * j + 1][0]));
}

__global__ void k_deh_store(SolveDev S, int d, const int* __restrict__ cmap, int nn, const double* X)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nn) return;
  const int col = cmap[c];
  const int s = col >> 2, sn = col & 3;
  const size_t b3 = (size_t)(4 * (s + 1) + sn) * 3;
  for (int i = 0; i < 3; i++) {
    stc(S.dE[d], b3 + i, ldc(X, (size_t)i * nn + c));
    stc(S.dH_[d], b3 + i, ldc(X, (size_t)(3 + i) * nn + c));
  }
}

// ==========================================================================================
// Host orchestration of the solve stage
#include <vector>

namespace {

// Device buffer from the stream-ordered allocator on the calling thread's default stream: freeing
// it does not synchronise the device (cudaFree would wait for every stream), so contexts used from
// different host threads do not stall each other.  Every user of a buffer has finished, in that
// stream's order, before the buffer goes out of scope.
struct DevBuf {
  void* p = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { if (p) cudaFreeAsync(p, cudaStreamPerThread); }
  int alloc(size_t bytes)
  {
    if (p) { cudaFreeAsync(p, cudaStreamPerThread); p = nullptr; }
    return cudaMallocAsync(&p, bytes, cudaStreamPerThread) == cudaSuccess ? 0 : BEM3_ERR_CUDA;
  }
  template <class T> T* as() { return (T*)p; }
};

template <class T>
int upload(DevBuf& b, const T* src, size_t n)
{
  if (b.alloc(n * sizeof(T) + 16)) return BEM3_ERR_CUDA;
  return cudaMemcpy(b.p, src, n * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess ? 0 : BEM3_ERR_CUDA;
}

// Dense LU solve of A x = B on the device for row-major A (n x n) and column-major B (n x nrhs):
// the solver sees A^T (column-major), so the transposed solve gives A x = B.
int lu_solve_rowmajor(cusolverDnHandle_t h, double* A, int n, double* B, int nrhs)
{
  int lwork = 0;
  if (cusolverDnZgetrf_bufferSize(h, n, n, (cuDoubleComplex*)A, n, &lwork) != CUSOLVER_STATUS_SUCCESS) return BEM3_ERR_SOLVE;
  DevBuf work, ipiv, info;
  if (work.alloc(sizeof(cuDoubleComplex) * (size_t)(lwork > 0 ? lwork : 1)) || ipiv.alloc(sizeof(int) * (size_t)n) ||
      info.alloc(sizeof(int)))
    return BEM3_ERR_CUDA;
  if (cusolverDnZgetrf(h, n, n, (cuDoubleComplex*)A, n, work.as<cuDoubleComplex>(), ipiv.as<int>(), info.as<int>()) !=
      CUSOLVER_STATUS_SUCCESS)
    return BEM3_ERR_SOLVE;
  int hinfo = 0;
  cudaMemcpy(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost);
  if (hinfo != 0) return BEM3_ERR_SOLVE;
  if (cusolverDnZgetrs(h, CUBLAS_OP_T, n, nrhs, (const cuDoubleComplex*)A, n, ipiv.as<int>(), (cuDoubleComplex*)B, n,
                       info.as<int>()) != CUSOLVER_STATUS_SUCCESS)
    return BEM3_ERR_SOLVE;
  cudaMemcpy(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost);
  return hinfo == 0 ? 0 : BEM3_ERR_SOLVE;
}

}  // namespace


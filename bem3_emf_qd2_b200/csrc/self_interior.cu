// self_interior.cu -- self-element (t == s) coefficients of the interior (free-space, complex k)
// domains: one CTA per collocation node; the quadrature pieces and their combination are the
// host+device functions of self.cuh (principal-value method of the reference, SW_DBIEQ == 0).
#include <cuda_runtime.h>

#include "self.cuh"
#include "bem3_internal.h"

// c_xl, c_wl, c_xh, c_wh: Gauss-Legendre tables defined in assemble.cu (same translation unit,
// see bem3_lib.cu).

#define SI_THREADS 256
#define SI_NW (SI_THREADS / 32)

// block-wide sum of v[0..N) into out (valid in thread 0 after the call); red = [SI_NW][N]
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

// Row `row` (= 4 t + tn) of an interior domain, by the whole CTA (SI_THREADS threads); red, res:
// its shared reduction buffers.
__device__ __forceinline__ void self_interior_row(const AssembleArgs& A, int row, double3* Fself, double* red,
                                                  double (*res)[SELF_NV])
{
  const int t = row >> 2, tn = row & 3;
  const int sd = A.sid[t];
  SelfInfo S;
  self_setup(A.geo, abs(sd), tn, mk(A.kre, A.kim), S);
  if (tn == 3 && S.e.nn == 3) return;
  double v[SELF_NV];

  for (int i = 0; i < SELF_NV; i++) v[i] = 0.0;
  self_int_piece1(S, c_xl, c_wl, c_xh, c_wh, threadIdx.x, blockDim.x, v);
  block_sum<17>(v, red, res[0]);

  for (int i = 0; i < SELF_NV; i++) v[i] = 0.0;
  self_int_piece2(S, c_xh, c_wh, threadIdx.x, blockDim.x, v);
  block_sum<34>(v, red, res[1]);

  for (int i = 0; i < SELF_NV; i++) v[i] = 0.0;
  self_int_piece3(S, c_xl, c_wl, c_xh, c_wh, threadIdx.x, blockDim.x, v);
  block_sum<32>(v, red, res[2]);

  for (int i = 0; i < SELF_NV; i++) v[i] = 0.0;
  self_int_piece4(S, c_xl, c_wl, c_xh, c_wh, threadIdx.x, blockDim.x, v);
  block_sum<34>(v, red, res[3]);

  if (threadIdx.x != 0) return;
  cplx CC[9], dCz[9], dCe[9];
  self_int_combine(S, res[0], res[1], res[2], res[3], sd < 0, CC, dCz, dCe);
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
}

__global__ void __launch_bounds__(SI_THREADS) k_self_interior(AssembleArgs A, double3* Fself)
{
  __shared__ double red[SI_NW * SELF_NV];
  __shared__ double res[4][SELF_NV];
  self_interior_row(A, blockIdx.x, Fself, red, res);
}

void bem3_launch_self_interior(const AssembleArgs& A, double3* Fself, int* d_status, cudaStream_t st)
{
  (void)d_status;  // the free-space integrals have no failure mode to report
  k_self_interior<<<4 * A.ne, SI_THREADS, 0, st>>>(A, Fself);
}

// mesh.cu -- element set-up on the device: the packed geometry record (GEO_* layout of elem.cuh) of
// every element, from the node coordinates and the element vertex lists, for meshes that are built
// or deformed on the device.  It computes what the reference's init_elem_const
// (d3qd2_src/d3qd2_setup.c:1139-1186: the map coefficients cr and the Jacobian-normal coefficients
// cw) and init_boundary_data (:1309-1349: collocation nodes and their normals) compute, with every
// sum and product rounded on its own (no contraction into fused multiply-adds) in the reference's
// operation order, so the record is bit-identical to the host set-up's (bem3_pack_geometry of the
// constants the reference-format readers produce).
#include <cuda_runtime.h>

#include "elem.cuh"
#include "bem3_internal.h"

namespace {

__device__ __forceinline__ double fa(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fs(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double fm(double a, double b) { return __dmul_rn(a, b); }

// one thread per element id 0..Ne (id 0: the unused zero record).  c13 = 1/3 and ic3 = 1/sqrt(3)
// come from the host, rounded as the host set-up rounds them.
__global__ void k_mesh_pack(int Ne, int Nn, const double* __restrict__ rn, const int* __restrict__ ed, double c13,
                            double ic3, double* __restrict__ geo, int* __restrict__ status)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > Ne) return;
  double* g = geo + (size_t)i * GEO_STRIDE;
  for (int k = 0; k < GEO_STRIDE; k++) g[k] = 0.0;
  if (i == 0) return;
  int v[4];
  for (int j = 0; j < 4; j++) v[j] = ed[4 * (size_t)i + j];
  const bool quad = v[3] != 0;
  const int nv = quad ? 4 : 3;
  for (int j = 0; j < nv; j++)
    if (v[j] < 1 || v[j] > Nn) {  // a vertex outside the node table: record it, read nothing
      atomicCAS(status, 0, BEM3_ERR_ARG);
      return;
    }
  double rc[3][4];
  for (int d = 0; d < 3; d++)
    for (int j = 0; j < 4; j++) rc[d][j] = (j < nv) ? rn[3 * (size_t)v[j] + d] : 0.0;
  double cr[3][4], cw[3][3];
  for (int d = 0; d < 3; d++)
    for (int c = 0; c < 3; c++) cw[d][c] = 0.0;
  if (quad) {
    for (int d = 0; d < 3; d++) {
      const double r0 = rc[d][0], r1 = rc[d][1], r2 = rc[d][2], r3 = rc[d][3];
      cr[d][0] = fm(0.25, fa(fa(fa(r0, r1), r2), r3));
      cr[d][1] = fm(0.25, fs(fa(fa(-r0, r1), r2), r3));
      cr[d][2] = fm(0.25, fa(fa(fs(-r0, r1), r2), r3));
      cr[d][3] = fm(0.25, fs(fa(fs(r0, r1), r2), r3));
    }
    const int ra[3] = {1, 2, 0}, rb[3] = {2, 0, 1};
    for (int row = 0; row < 3; row++) {
      const double* A = rc[ra[row]];
      const double* B = rc[rb[row]];
      cw[row][0] = fm(0.125, fs(fm(fs(A[0], A[2]), fs(B[1], B[3])), fm(fs(A[1], A[3]), fs(B[0], B[2]))));
      cw[row][1] = fm(0.125, fs(fm(fs(A[2], A[3]), fs(B[0], B[1])), fm(fs(A[0], A[1]), fs(B[2], B[3]))));
      cw[row][2] = fm(0.125, fs(fm(fs(A[1], A[2]), fs(B[0], B[3])), fm(fs(A[0], A[3]), fs(B[1], B[2]))));
    }
  } else {
    for (int d = 0; d < 3; d++) {
      const double r0 = rc[d][0], r1 = rc[d][1], r2 = rc[d][2];
      cr[d][0] = fm(c13, fa(fa(r0, r1), r2));
      cr[d][1] = fm(c13, fs(fa(-r0, fm(2.0, r1)), r2));
      cr[d][2] = fm(ic3, fs(r2, r0));
      cr[d][3] = 0.0;
    }
    cw[0][0] = fs(fm(fs(rc[1][1], rc[1][0]), fs(rc[2][2], rc[2][0])), fm(fs(rc[2][1], rc[2][0]), fs(rc[1][2], rc[1][0])));
    cw[1][0] = fs(fm(fs(rc[2][1], rc[2][0]), fs(rc[0][2], rc[0][0])), fm(fs(rc[0][1], rc[0][0]), fs(rc[2][2], rc[2][0])));
    cw[2][0] = fs(fm(fs(rc[0][1], rc[0][0]), fs(rc[1][2], rc[1][0])), fm(fs(rc[1][1], rc[1][0]), fs(rc[0][2], rc[0][0])));
  }
  for (int d = 0; d < 3; d++) {
    for (int c = 0; c < 4; c++) g[GEO_CR + d * 4 + c] = cr[d][c];
    for (int c = 0; c < 3; c++) g[GEO_CW + d * 3 + c] = cw[d][c];
  }
  // collocation nodes r(zeta_j, eta_j) and the Jacobian normals there (the node parameters of
  // node_zeta / node_eta; the fourth node of a triangle sits at its first map coefficient)
  for (int j = 0; j < 4; j++) {
    const double z = node_zeta(nv, j), e = node_eta(nv, j);
    for (int d = 0; d < 3; d++) {
      double r, w;
      if (quad) {
        r = fa(fa(fa(cr[d][0], fm(cr[d][1], z)), fm(cr[d][2], e)), fm(fm(cr[d][3], z), e));
        w = fa(fa(cw[d][0], fm(cw[d][1], z)), fm(cw[d][2], e));
      } else {
        r = fa(fa(cr[d][0], fm(cr[d][1], z)), fm(cr[d][2], e));
        w = cw[d][0];
      }
      g[GEO_REN + j * 3 + d] = r;
      g[GEO_WEN + j * 3 + d] = w;
    }
  }
  g[GEO_NN] = (double)nv;
}

}  // namespace

extern "C" int bem3_mesh_pack_dev(int Ne, int Nn, const double* rn_dev, const int* ed_dev, double* geo_dev, void* stream)
{
  if (Ne <= 0 || Nn <= 0 || !rn_dev || !ed_dev || !geo_dev) return BEM3_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  int* dstatus = nullptr;
  if (cudaMallocAsync((void**)&dstatus, sizeof(int), st) != cudaSuccess) return BEM3_ERR_CUDA;
  int rc = BEM3_ERR_CUDA;
  int hs = 0;
  const double c13 = 1.0 / 3.0, ic3 = 1.0 / sqrt(3.0);
  if (cudaMemsetAsync(dstatus, 0, sizeof(int), st) == cudaSuccess) {
    k_mesh_pack<<<(unsigned)((Ne + 1 + 255) / 256), 256, 0, st>>>(Ne, Nn, rn_dev, ed_dev, c13, ic3, geo_dev, dstatus);
    if (cudaGetLastError() == cudaSuccess &&
        cudaMemcpyAsync(&hs, dstatus, sizeof(int), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
        cudaStreamSynchronize(st) == cudaSuccess)
      rc = hs;
  }
  cudaFreeAsync(dstatus, st);
  return rc;
}

// Host build of the device math headers (Faddeeva, QPGF) for CPU-side checks against the
// reference oracle.  Test infrastructure: the product runs these functions only on the GPU.
#include <stdint.h>
#include "qpgf.cuh"

extern "C" {

void hm_faddeeva(int n, const double* z, double* w)
{
  for (int i = 0; i < n; i++) {
    cplx v = faddeeva_w(z[2 * i], z[2 * i + 1]);
    w[2 * i] = v.re;
    w[2 * i + 1] = v.im;
  }
}

// p = k, vk[3], vd1[2], vd2[2] (the reference's QPD2 order); out = qG, dqG[3] interleaved re/im
void hm_qpgf(int n, const double* r, const double* p, int mode, double* out, int* ret)
{
  QPLattice L;
  qp_lattice_init(L, p[0], p[1], p[2], p[4], p[5], p[6], p[7]);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n; i++) {
    QPVal v;
    int e = (mode == 0) ? qpgf_eval<QP_V1>(L, r + 3 * i, v) : qpgf_eval<QP_BOTH>(L, r + 3 * i, v);
    ret[i] = e;
    out[8 * i + 0] = v.G.re; out[8 * i + 1] = v.G.im;
    for (int c = 0; c < 3; c++) { out[8 * i + 2 + 2 * c] = v.dG[c].re; out[8 * i + 3 + 2 * c] = v.dG[c].im; }
  }
}

}

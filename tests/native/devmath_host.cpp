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

// e^{x^2} erfc(x) as the assembly's spectral terms evaluate it (qp_erfcx)
void hm_erfcx(int n, const double* x, double* out)
{
  for (int i = 0; i < n; i++) out[i] = qp_erfcx(x[i]);
}

// Second derivatives: out = qG, dqG[3], d2qG[6] interleaved re/im (20 doubles per point)
void hm_qpgf2(int n, const double* r, const double* p, double* out, int* ret)
{
  QPLattice L;
  qp_lattice_init(L, p[0], p[1], p[2], p[4], p[5], p[6], p[7]);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n; i++) {
    QPVal2 v;
    ret[i] = qpgf_eval2(L, r + 3 * i, v);
    double* o = out + 20 * (size_t)i;
    o[0] = v.G.re; o[1] = v.G.im;
    for (int c = 0; c < 3; c++) { o[2 + 2 * c] = v.dG[c].re; o[3 + 2 * c] = v.dG[c].im; }
    for (int c = 0; c < 6; c++) { o[8 + 2 * c] = v.d2G[c].re; o[9 + 2 * c] = v.d2G[c].im; }
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

#include "elem.cuh"

extern "C" {

// One regular (t != s) pair with the device element rules, evaluated serially on the host.
// geo: packed geometry; td, sd: signed element ids; tn: collocation node; periodic: 1 for the
// open domain; n: 12 (GL) or 64 (GH); p: QPD2 order; out: CC[9], dCz[9], dCe[9] (re/im pairs).
// Returns 1 when the GL result asks for the near-singular rule, else 0.
int hm_pair_regular(const double* geo, int td, int tn, int sd, int periodic, double kre, double kim,
                    const double* p, int n, const double* x, const double* w, double* out)
{
  QPLattice L;
  qp_lattice_init(L, p[0], p[1], p[2], p[4], p[5], p[6], p[7]);
  static thread_local QPProp prop[QP_PROP_CAP];
  L.nprop = qp_prop_list(L, prop, QP_PROP_CAP);
  L.prop = prop;
  Elem et, es;
  load_elem(geo, td < 0 ? -td : td, et);
  load_elem(geo, sd < 0 ? -sd : sd, es);
  double vtz[3], vte[3];
  node_tangents(et, tn, vtz, vte);
  const double* rt = geo + (size_t)(td < 0 ? -td : td) * GEO_STRIDE + GEO_REN + tn * 3;
  int npts = (es.nn == 4) ? n * n : 3 * n * n;
  cplx CC[9], dCz[9], dCe[9];
  if (periodic) {
    AccP a;
    accp_zero(a);
    for (int q = 0; q < npts; q++) {
      double z, e, wt;
      rule_point(es.nn, n, x, w, q, z, e, wt);
      accp_point(es, L, rt, vtz, vte, z, e, wt, a);
    }
    accp_finish(es, a, CC, dCz, dCe);
  } else {
    AccI a;
    acci_zero(a);
    for (int q = 0; q < npts; q++) {
      double z, e, wt;
      rule_point(es.nn, n, x, w, q, z, e, wt);
      acci_point(es, mk(kre, kim), rt, vtz, vte, z, e, wt, a);
    }
    acci_finish(es, a, sd < 0, CC, dCz, dCe);
  }
  for (int i = 0; i < 9; i++) {
    out[2 * i] = CC[i].re; out[2 * i + 1] = CC[i].im;
    out[18 + 2 * i] = dCz[i].re; out[19 + 2 * i] = dCz[i].im;
    out[36 + 2 * i] = dCe[i].re; out[37 + 2 * i] = dCe[i].im;
  }
  return needs_gh(dCz[8].re, dCe[8].re);
}

}

#include "self.cuh"

extern "C" {

// Interior self pair (t == s) evaluated serially with the device pieces; out as hm_pair_regular.
void hm_self_interior(const double* geo, int sd, int tn, double kre, double kim, const double* xl, const double* wl,
                      const double* xh, const double* wh, double* out)
{
  SelfInfo S;
  self_setup(geo, sd < 0 ? -sd : sd, tn, mk(kre, kim), S);
  double R[4][SELF_NV];
  for (int p = 0; p < 4; p++) for (int i = 0; i < SELF_NV; i++) R[p][i] = 0.0;
  self_int_piece1(S, xl, wl, xh, wh, 0, 1, R[0]);
  self_int_piece2(S, xh, wh, 0, 1, R[1]);
  self_int_piece3(S, xl, wl, xh, wh, 0, 1, R[2]);
  self_int_piece4(S, xl, wl, xh, wh, 0, 1, R[3]);
  cplx CC[9], dCz[9], dCe[9];
  self_int_combine(S, R[0], R[1], R[2], R[3], sd < 0, CC, dCz, dCe);
  for (int i = 0; i < 9; i++) {
    out[2 * i] = CC[i].re; out[2 * i + 1] = CC[i].im;
    out[18 + 2 * i] = dCz[i].re; out[19 + 2 * i] = dCz[i].im;
    out[36 + 2 * i] = dCe[i].re; out[37 + 2 * i] = dCe[i].im;
  }
}

}

extern "C" {

// Periodic self pair evaluated serially with the device routine; p: QPD2 order.
int hm_self_periodic(const double* geo, int sd, int tn, const double* p, const double* xl, const double* wl,
                     const double* xh, const double* wh, double* out)
{
  QPLattice L;
  qp_lattice_init(L, p[0], p[1], p[2], p[4], p[5], p[6], p[7]);
  static thread_local QPProp prop[QP_PROP_CAP];
  L.nprop = qp_prop_list(L, prop, QP_PROP_CAP);
  L.prop = prop;
  SelfInfo S;
  self_setup(geo, sd < 0 ? -sd : sd, tn, mk(0.0, 0.0), S);
  double v[24];
  for (int i = 0; i < 24; i++) v[i] = 0.0;
  int err = self_per_points(S, L, xl, wl, xh, wh, 0, 1, v);
  cplx CC[9], dCz[9], dCe[9];
  self_per_combine(S, v, CC, dCz, dCe);
  for (int i = 0; i < 9; i++) {
    out[2 * i] = CC[i].re; out[2 * i + 1] = CC[i].im;
    out[18 + 2 * i] = dCz[i].re; out[19 + 2 * i] = dCz[i].im;
    out[36 + 2 * i] = dCe[i].re; out[37 + 2 * i] = dCe[i].im;
  }
  return err;
}

}

#include "field.cuh"

extern "C" {

// Field coefficients of source element sd at point rt with the device rules (field.cuh);
// out = CC[0..7] re/im pairs then F.  Returns the status of field_coef.
// gl: x12, w12, x64, w64 (152 doubles) for types 2 and 3.
int hm_field_coef(const double* geo, int sd, const double* rt, int periodic, double kre, double kim, int type,
                  const double* p, const double* gl, double* out)
{
  QPLattice L;
  qp_lattice_init(L, p[0], p[1], p[2], p[4], p[5], p[6], p[7]);
  static thread_local QPProp prop[QP_PROP_CAP];
  L.nprop = qp_prop_list(L, prop, QP_PROP_CAP);
  L.prop = prop;
  const FieldGL tabs = {gl, gl + 12, gl + 24, gl + 88};
  cplx CC[8];
  double F;
  int st = periodic ? field_coef<true>(geo, sd, rt, mk(kre, kim), type, L, CC, F, &tabs)
                    : field_coef<false>(geo, sd, rt, mk(kre, kim), type, L, CC, F, &tabs);
  for (int i = 0; i < 8; i++) { out[2 * i] = CC[i].re; out[2 * i + 1] = CC[i].im; }
  out[16] = F;
  return st;
}

// field_grad_coef: out = CC[8], dC[3][8] (re/im pairs, 64 doubles), F, dF[3]
int hm_field_grad_coef(const double* geo, int sd, const double* rt, int periodic, double kre, double kim, int type,
                       const double* p, const double* gl, double* out)
{
  QPLattice L;
  qp_lattice_init(L, p[0], p[1], p[2], p[4], p[5], p[6], p[7]);
  const FieldGL tabs = {gl, gl + 12, gl + 24, gl + 88};
  cplx CC[8], dC[3][8];
  double F, dF[3];
  int st = periodic ? field_grad_coef<true>(geo, sd, rt, mk(kre, kim), type, L, &tabs, CC, dC, F, dF)
                    : field_grad_coef<false>(geo, sd, rt, mk(kre, kim), type, L, &tabs, CC, dC, F, dF);
  for (int i = 0; i < 8; i++) { out[2 * i] = CC[i].re; out[2 * i + 1] = CC[i].im; }
  for (int q = 0; q < 3; q++)
    for (int i = 0; i < 8; i++) { out[16 + 16 * q + 2 * i] = dC[q][i].re; out[17 + 16 * q + 2 * i] = dC[q][i].im; }
  out[64] = F;
  for (int q = 0; q < 3; q++) out[65 + q] = dF[q];
  return st;
}

// Solid angle of an element seen from rt (vertices rn[ed[e][v]]), as the domain search uses it.
double hm_solid_angle(const double* rn, const int* ed, int e, int nv, const double* rt, int* flag)
{
  double rv[4][3];
  for (int v = 0; v < 4; v++)
    for (int k = 0; k < 3; k++) rv[v][k] = rn[3 * ed[4 * e + v] + k] - rt[k];
  return solid_angle(nv, rv, *flag);
}

}

extern "C" void hm_faddeeva_fast(int n, const double* z, double* w)
{
  for (int i = 0; i < n; i++) {
    cplx v = faddeeva_w_t<true>(z[2 * i], z[2 * i + 1]);
    w[2 * i] = v.re;
    w[2 * i + 1] = v.im;
  }
}

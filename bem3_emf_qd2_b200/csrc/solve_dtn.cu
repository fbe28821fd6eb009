// solve_dtn.cu -- the global system of the modified potentials solved through per-domain
// Dirichlet-to-Neumann maps, half the size of the reference's system.
//
// The reference solves one sparse system of 8 NN unknowns (U and dU = dU/dn at every element node,
// 4 components each; create_matrix_csr_dac d3qd2_solve_bieq.c:284-421).  Its rows are, for every
// domain d, component c and node i of d:
//     sum_j H_d[i,j] U_c(j) + G_d[i,j] q^d_c(j) = b^d_c(i)
// where q^d is the normal derivative as domain d sees it: -dU at nodes whose element has d as main
// domain, and dU + delt n_c U_3 (c < 3) or beps dU_3 + sigm n.U (c = 3) at nodes whose element
// has d as sub domain (delt = k_m^2 - k_s^2, beps = k_m^2 / k_s^2, sigm = 1 - beps of the element).
// Every element node lies between exactly two domains.  When the domains can be split into two
// classes such that every element separates a domain of one class from a domain of the other
// (the domain graph is bipartite: nested layers, separate particles), the equations of each
// domain d of the first class give q^d = G_d^-1 (b^d - H_d U) = g^d - K_d U with the same matrices
// for all four components, so dU at every node is a function of U alone.  Substituting it into
// the equations of the other class leaves 4 NN equations in the 4 NN potentials U:
//     H_e U_c + G_e (K^ U_c + local_c(U)) = b^e_c + G_e (alpha g^)_c
// with K^ the rows of the K_d belonging to e's nodes.  After the solve, dU follows from the same
// relations.  The solution is the reference's (same equations, different elimination order).
#include <cublas_v2.h>

struct DtnNode {   // one global element node
  int elem;        // element id (1..Ne)
  int l;           // node within the element
  int de, le;      // eliminated domain and the node's index among that domain's nodes
  int dn, ln;      // kept domain and index among its nodes
};

struct DtnArgs {
  const DtnNode* node;   // [NN]
  const double* geo;
  const int* md;
  const int* sd;
  const double* kn;
  int NN;
};

__device__ __forceinline__ void dtn_consts(const DtnArgs& A, int m, cplx& delt, cplx& beps, cplx& sigm, double* n)
{
  const DtnNode q = A.node[m];
  const int mdid = A.md[q.elem], sdid = A.sd[q.elem];
  cplx k1 = mk(A.kn[2 * mdid], A.kn[2 * mdid + 1]), k2 = mk(A.kn[2 * sdid], A.kn[2 * sdid + 1]);
  cplx k12 = k1 * k1, k22 = k2 * k2;
  delt = k12 - k22;
  beps = cdiv(k12, k22);
  sigm = mk(1.0 - beps.re, -beps.im);
  node_normal(A.geo, q.elem, q.l, n);
}

// Compact a domain's 4ne x 4ne row-major matrix to its n nodes, column-major (dst[c n + r]).
__global__ void k_compact_cm(const double* __restrict__ src, int N, const int* __restrict__ cmap, int n,
                             double* __restrict__ dst)
{
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)n * n) return;
  const int r = (int)(q % n), c = (int)(q / n);
  const size_t s = (size_t)cmap[r] * N + cmap[c];
  dst[2 * q] = src[2 * s];
  dst[2 * q + 1] = src[2 * s + 1];
}

// Right-hand sides b^d_c(i) of domain d's rows (the bsum of k_build_rows), column-major n x 4.
__global__ void k_dtn_rhs(SolveDev S, int d, const int* __restrict__ cmap, int n, double* __restrict__ B)
{
  const int c = blockIdx.y;
  const int i = blockIdx.x;  // compacted row
  const int src = cmap[i];
  const int ne = S.ne[d];
  const size_t N = (size_t)4 * ne;
  const double* G = S.G[d] + 2 * ((size_t)src * N);
  const double* H = S.H[d] + 2 * ((size_t)src * N);
  cplx bsum = mk(0, 0);
  for (int s = threadIdx.x; s < ne; s += blockDim.x) {
    const int sdd = S.sid_h[d][s];
    const int asd = abs(sdd);
    const int mdid = S.md[asd], sdid = S.sd[asd];
    if (d == mdid || mdid != 0) continue;  // only sub-domain elements on the open region carry b
    const int nv = (int)S.geo[(size_t)asd * GEO_STRIDE + GEO_NN];
    cplx k1 = mk(S.kn[2 * mdid], S.kn[2 * mdid + 1]), k2 = mk(S.kn[2 * sdid], S.kn[2 * sdid + 1]);
    cplx beps = cdiv(k1 * k1, k2 * k2);
    cplx sigm = mk(1.0 - beps.re, -beps.im);
    for (int l = 0; l < nv; l++) {
      double vn[3];
      node_normal(S.geo, asd, l, vn);
      cplx g = ldc(G, 4 * s + l), h = ldc(H, 4 * s + l);
      const double* ui = S.Ui + 2 * ((size_t)(4 * asd + l) * 4);
      const double* dui = S.dUi + 2 * ((size_t)(4 * asd + l) * 4);
      if (c < 3) {
        bsum = bsum - h * ldc(ui, c) - g * ldc(dui, c);
      } else {
        cplx nu = ldc(ui, 0) * vn[0] + ldc(ui, 1) * vn[1] + ldc(ui, 2) * vn[2];
        bsum = bsum - sigm * g * nu;
      }
    }
  }
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
  if (threadIdx.x == 0) stc(B, (size_t)c * n + i, mk(red[0][0], red[1][0]));
}

// K^ of kept domain e (column-major ne_n x NN) and, with scale, alpha K^ for the phi rows.
// gnode[j]: global node of e's j-th node.  K[d]: K_d column-major n_d x n_d (device pointers).
struct KPtrs {
  const double* K[BEM3_MAXDOM];
  int n[BEM3_MAXDOM];
};
__global__ void k_dtn_khat(DtnArgs A, KPtrs KP, const int* __restrict__ gnode, int n_e, int e, int alpha,
                           double* __restrict__ Kh)
{
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)n_e * A.NN) return;
  const int j = (int)(q % n_e), m = (int)(q / n_e);
  const DtnNode qj = A.node[gnode[j]];
  const DtnNode qm = A.node[m];
  cplx v = mk(0, 0);
  if (qm.de == qj.de) {
    const int nd = KP.n[qj.de];
    v = ldc(KP.K[qj.de], (size_t)qm.le * nd + qj.le);
    if (alpha) {
      cplx delt, beps, sigm;
      double nrm[3];
      dtn_consts(A, gnode[j], delt, beps, sigm, nrm);
      const bool main_in_e = (A.md[qj.elem] == e);
      v = main_in_e ? cdiv(v, beps) : v * beps;
    }
  }
  stc(Kh, q, v);
}

// alpha g^ of kept domain e, column-major n_e x 4: g of each node's eliminated domain.
__global__ void k_dtn_ghat(DtnArgs A, KPtrs GP, const int* __restrict__ gnode, int n_e, int e, double* __restrict__ Gh)
{
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 4 * n_e) return;
  const int j = q % n_e, c = q / n_e;
  const DtnNode qj = A.node[gnode[j]];
  const int nd = GP.n[qj.de];
  cplx v = ldc(GP.K[qj.de], (size_t)c * nd + qj.le);
  if (c == 3) {
    cplx delt, beps, sigm;
    double nrm[3];
    dtn_consts(A, gnode[j], delt, beps, sigm, nrm);
    v = (A.md[qj.elem] == e) ? cdiv(v, beps) : v * beps;
  }
  stc(Gh, q, v);
}

// Rows of kept domain e in the reduced matrix (column-major, lda = 4 NN), rows row0 + c n_e + j.
__global__ void k_dtn_rows(DtnArgs A, int e, const int* __restrict__ gnode, int n_e, const double* __restrict__ Hc,
                           const double* __restrict__ Gc, const double* __restrict__ P, const double* __restrict__ Q,
                           double* __restrict__ Ared, long long lda, long long row0)
{
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long ncol = 4LL * A.NN;
  if (q >= (long long)4 * n_e * ncol) return;
  const int rr = (int)(q % (4LL * n_e));  // row within e's block: c n_e + j
  const long long col = q / (4LL * n_e);
  const int c = rr / n_e, j = rr % n_e;
  const int cp = (int)(col / A.NN), m = (int)(col % A.NN);
  const DtnNode qm = A.node[m];
  const bool in_e = (qm.dn == e);
  cplx v = mk(0, 0);
  if (cp == c) {
    v = ldc(c < 3 ? P : Q, (size_t)m * n_e + j);
    if (in_e) v += ldc(Hc, (size_t)qm.ln * n_e + j);
  } else if (in_e && (c == 3 || cp == 3)) {
    cplx delt, beps, sigm;
    double nrm[3];
    dtn_consts(A, m, delt, beps, sigm, nrm);
    const cplx g = ldc(Gc, (size_t)qm.ln * n_e + j);
    if (c < 3) {  // delt n_c U_3 inside q^e_c
      v = g * (delt * nrm[c]);
    } else {      // sigma^ n.U inside q^e_3
      const bool main_in_e = (A.md[qm.elem] == e);
      const cplx sh = main_in_e ? cdiv(sigm, beps) : sigm;
      v = g * (sh * nrm[cp]);
    }
  }
  stc(Ared, (size_t)col * lda + row0 + rr, v);
}

// U of eliminated domain d's nodes, column-major n_d x 4, from the reduced solution x (c NN + m).
__global__ void k_dtn_gather_u(const int* __restrict__ gnode, int n_d, int NN, const double* __restrict__ x,
                               double* __restrict__ Ud)
{
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 4 * n_d) return;
  const int j = q % n_d, c = q / n_d;
  stc(Ud, q, ldc(x, (size_t)c * NN + gnode[j]));
}

// dU of eliminated domain d's nodes into the full solution vector X (8 NN, c NN + m layout),
// from KU = K_d U_d and g = g^d (both column-major n_d x 4); copies U as well.
__global__ void k_dtn_du(DtnArgs A, int d, const int* __restrict__ gnode, int n_d, const double* __restrict__ KU,
                         const double* __restrict__ g, const double* __restrict__ x, double* __restrict__ X)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_d) return;
  const int m = gnode[j];
  const size_t NN = (size_t)A.NN;
  cplx U[4];
  for (int c = 0; c < 4; c++) {
    U[c] = ldc(x, c * NN + m);
    stc(X, c * NN + m, U[c]);
  }
  const DtnNode qm = A.node[m];
  if (A.md[qm.elem] == d) {  // main in d: q = -dU
    for (int c = 0; c < 4; c++) stc(X, (4 + c) * NN + m, ldc(KU, (size_t)c * n_d + j) - ldc(g, (size_t)c * n_d + j));
    return;
  }
  cplx delt, beps, sigm;
  double nrm[3];
  dtn_consts(A, m, delt, beps, sigm, nrm);
  for (int c = 0; c < 3; c++) {
    cplx q = ldc(g, (size_t)c * n_d + j) - ldc(KU, (size_t)c * n_d + j);
    stc(X, (4 + c) * NN + m, q - delt * U[3] * nrm[c]);
  }
  cplx q3 = ldc(g, (size_t)3 * n_d + j) - ldc(KU, (size_t)3 * n_d + j);
  cplx nU = U[0] * nrm[0] + U[1] * nrm[1] + U[2] * nrm[2];
  stc(X, 7 * NN + m, cdiv(q3 - sigm * nU, beps));
}

// Y (n x 4, column-major) += G_d,compact X, G_d read in place from the domain's row-major
// 4ne x 4ne matrix through cmap; one CTA per row.
__global__ void k_compact_matvec4(const double* __restrict__ G, int N, const int* __restrict__ cmap, int n,
                                  const double* __restrict__ X, double* __restrict__ Y)
{
  const int i = blockIdx.x;
  const double* row = G + 2 * ((size_t)cmap[i] * N);
  cplx acc[4];
  for (int c = 0; c < 4; c++) acc[c] = mk(0, 0);
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const cplx g = ldc(row, cmap[j]);
    for (int c = 0; c < 4; c++) acc[c] += g * ldc(X, (size_t)c * n + j);
  }
  __shared__ double red[8][256];
  for (int c = 0; c < 4; c++) { red[2 * c][threadIdx.x] = acc[c].re; red[2 * c + 1][threadIdx.x] = acc[c].im; }
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 8; k++) red[k][threadIdx.x] += red[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 4; c++) stc(Y, (size_t)c * n + i, ldc(Y, (size_t)c * n + i) + mk(red[2 * c][0], red[2 * c + 1][0]));
}

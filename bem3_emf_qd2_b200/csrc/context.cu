// context.cu -- device-resident problems (bem3_ctx_*) and the solve stage's host orchestration
// (solve_bieq, d3qd2_src/d3qd2_solve_bieq.c:36-84).
#include <math.h>
#include <stdlib.h>

// What a solve leaves on the device so that a new incident field needs only right-hand sides:
// the matrices of every domain, each domain's compacted G factorised, and the factorised system
// of the potentials (reduced or full).
struct SolveState {
  int method = 0;  // factors held: 0 none, 1 the full 8 NN system, 2 the reduced 4 NN system
  DevBuf G[BEM3_MAXDOM], H[BEM3_MAXDOM], dG[BEM3_MAXDOM], dH[BEM3_MAXDOM], dF[BEM3_MAXDOM];
  int n[BEM3_MAXDOM] = {};                 // element nodes of each domain
  DevBuf gnode[BEM3_MAXDOM], cmap[BEM3_MAXDOM];
  DevBuf Gc[BEM3_MAXDOM], Gpiv[BEM3_MAXDOM];  // compacted G_d, LU-factorised (column-major)
  std::vector<int> elim;                   // reduced form: eliminated domains
  DevBuf nodes;                            // DtnNode[NN]
  DevBuf K[BEM3_MAXDOM];                   // K_d = G_d^-1 H_d of the eliminated domains
  DevBuf A, Apiv;                          // the factorised system of the potentials
  size_t bytes = 0;                        // device memory held
};

struct bem3_ctx_s {
  int dev = 0;
  int MN = 0, Ne = 0, NN = 0, Nn = 0, ps = 0, nwaves = 0;
  double lambda0 = 0.0;
  bem3_qpd2 qd;
  QPLattice L;
  std::vector<int> nv;                 // [(Ne+1)]
  std::vector<std::vector<int>> sid;   // per domain, signed ids
  std::vector<double> kn;              // [2 (MN+1)]
  std::vector<int> doff;               // domain-id lists: offsets [MN+2]
  std::vector<int> eni_h, md_h, sd_h;  // host copies for the solve's index tables
  int solver = 0;                      // 0 auto, 1 full 8 NN system, 2 reduced 4 NN system
  DevBuf geo, md, sd, eni, knd, Ui, dUi, dEiz, dEie, pos0, rn, ed, waves, dlist, dsd;
  DevBuf dsid[BEM3_MAXDOM];
  DevBuf U[BEM3_MAXDOM], dU[BEM3_MAXDOM], E[BEM3_MAXDOM], H[BEM3_MAXDOM], dE[BEM3_MAXDOM], dH[BEM3_MAXDOM];
  DevBuf status;
  DevBuf prop;  // the lattice's propagating orders (the optimised lattice sums of the self rule)
  SolveState* st = nullptr;
  double phase_ms[3] = {0.0, 0.0, 0.0};  // last solve: assembly, factorisation, right-hand sides + fields
  ~bem3_ctx_s() { delete st; }
};

namespace {

size_t bv4_bytes(int ne) { return (size_t)(ne + 1) * 4 * 4 * 16; }
size_t bv3_bytes(int ne) { return (size_t)(ne + 1) * 4 * 3 * 16; }

SolveDev solve_view(bem3_ctx c)
{
  SolveDev S;
  memset(&S, 0, sizeof S);
  S.MN = c->MN; S.NN = c->NN; S.Ne = c->Ne;
  S.geo = c->geo.as<double>(); S.md = c->md.as<int>(); S.sd = c->sd.as<int>(); S.eni = c->eni.as<int>();
  S.kn = c->knd.as<double>(); S.Ui = c->Ui.as<double>(); S.dUi = c->dUi.as<double>();
  S.dEiz = c->dEiz.as<double>(); S.dEie = c->dEie.as<double>(); S.pos0 = c->pos0.as<int>();
  S.ch_re = 0.0; S.ch_im = -c->lambda0 / (2.0 * QP_PI);  // lambda0 / (2 pi i)
  for (int d = 0; d <= c->MN; d++) {
    S.ne[d] = (int)c->sid[d].size();
    S.sid_h[d] = c->dsid[d].as<int>();
    S.U[d] = c->U[d].as<double>(); S.dU[d] = c->dU[d].as<double>(); S.E[d] = c->E[d].as<double>();
    S.H_[d] = c->H[d].as<double>(); S.dE[d] = c->dE[d].as<double>(); S.dH_[d] = c->dH[d].as<double>();
  }
  return S;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) { if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev); }
  ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

}  // namespace

extern "C" int bem3_ctx_create(const bem3_problem* P, bem3_ctx* out)
{
  if (!P || !out || P->MN < 0 || P->MN + 1 > BEM3_MAXDOM || P->Ne <= 0 || P->NN <= 0 || P->Nn <= 0 || !P->rn ||
      !P->ed || !P->md || !P->sd || !P->eni || !P->Ne_d || !P->sid || !P->kn || !P->Ui || !P->dUi || !P->dEiz ||
      !P->dEie || (P->nwaves > 0 && !P->waves) || P->mesh.Ne != P->Ne)
    return BEM3_ERR_ARG;
  *out = nullptr;
  bem3_ctx c = new bem3_ctx_s();
  int rc = 0;
  auto fail = [&](int e) { delete c; return e; };
  cudaGetDevice(&c->dev);
  c->MN = P->MN; c->Ne = P->Ne; c->NN = P->NN; c->Nn = P->Nn; c->ps = P->ps; c->nwaves = P->nwaves;
  c->lambda0 = P->lambda0;
  c->qd = P->qd;
  memset(&c->L, 0, sizeof c->L);
  if (P->ps == 1) {
    if (qp_lattice_init(c->L, P->qd.k, P->qd.vk[0], P->qd.vk[1], P->qd.vd1[0], P->qd.vd1[1], P->qd.vd2[0],
                        P->qd.vd2[1]) != 0)
      return fail(BEM3_ERR_LATTICE);
    std::vector<QPProp> pl(QP_PROP_CAP);
    const int np = qp_prop_list(c->L, pl.data(), QP_PROP_CAP);
    if (np < 0) return fail(BEM3_ERR_LATTICE);
    if ((rc = upload(c->prop, pl.data(), (size_t)(np > 0 ? np : 1)))) return fail(rc);
    c->L.prop = c->prop.as<QPProp>();
    c->L.nprop = np;
  }
  const int Ne = P->Ne, MN = P->MN;
  c->nv.assign(P->mesh.nv, P->mesh.nv + Ne + 1);
  c->eni_h.assign(P->eni, P->eni + 4 * (size_t)(Ne + 1));
  c->md_h.assign(P->md, P->md + Ne + 1);
  c->sd_h.assign(P->sd, P->sd + Ne + 1);
  c->kn.assign(P->kn, P->kn + 2 * (MN + 1));
  c->sid.resize(MN + 1);
  for (int d = 0; d <= MN; d++) {
    if (P->Ne_d[d] <= 0 || !P->sid[d]) return fail(BEM3_ERR_ARG);
    c->sid[d].assign(P->sid[d], P->sid[d] + P->Ne_d[d]);
    for (int s : c->sid[d])
      if (s == 0 || abs(s) > Ne) return fail(BEM3_ERR_ARG);
  }
  for (int e = 1; e <= Ne; e++) {
    if (P->md[e] < 0 || P->md[e] > MN || P->sd[e] < 0 || P->sd[e] > MN) return fail(BEM3_ERR_ARG);
    for (int v = 0; v < 4; v++)
      if (P->ed[4 * e + v] < 0 || P->ed[4 * e + v] > P->Nn) return fail(BEM3_ERR_ARG);
  }
  std::vector<double> geo((size_t)(Ne + 1) * GEO_STRIDE);
  if ((rc = bem3_pack_geometry(&P->mesh, geo.data()))) return fail(rc);
  if ((rc = upload(c->geo, geo.data(), geo.size())) || (rc = upload(c->md, P->md, (size_t)Ne + 1)) ||
      (rc = upload(c->sd, P->sd, (size_t)Ne + 1)) || (rc = upload(c->eni, P->eni, (size_t)(Ne + 1) * 4)) ||
      (rc = upload(c->knd, P->kn, (size_t)2 * (MN + 1))) || (rc = upload(c->Ui, P->Ui, (size_t)(Ne + 1) * 32)) ||
      (rc = upload(c->dUi, P->dUi, (size_t)(Ne + 1) * 32)) || (rc = upload(c->dEiz, P->dEiz, (size_t)(Ne + 1) * 24)) ||
      (rc = upload(c->dEie, P->dEie, (size_t)(Ne + 1) * 24)) || (rc = upload(c->rn, P->rn, (size_t)(P->Nn + 1) * 3)) ||
      (rc = upload(c->ed, P->ed, (size_t)(Ne + 1) * 4)))
    return fail(rc);
  if (P->nwaves > 0 && (rc = upload(c->waves, P->waves, (size_t)P->nwaves))) return fail(rc);
  std::vector<int> pos0((size_t)Ne + 1, -1);
  for (size_t s = 0; s < c->sid[0].size(); s++)
    if (c->sid[0][s] > 0) pos0[c->sid[0][s]] = (int)s;
  if ((rc = upload(c->pos0, pos0.data(), pos0.size()))) return fail(rc);
  // domain-id lists: the positive ids of each domain, in list order, with their sub-domains
  std::vector<int> dl, ds;
  c->doff.assign(MN + 2, 0);
  for (int d = 0; d <= MN; d++) {
    c->doff[d] = (int)dl.size();
    for (int s : c->sid[d])
      if (s > 0) { dl.push_back(s); ds.push_back(P->sd[s]); }
  }
  c->doff[MN + 1] = (int)dl.size();
  if (dl.empty()) return fail(BEM3_ERR_ARG);
  if ((rc = upload(c->dlist, dl.data(), dl.size())) || (rc = upload(c->dsd, ds.data(), ds.size()))) return fail(rc);
  for (int d = 0; d <= MN; d++) {
    const int ne = (int)c->sid[d].size();
    if ((rc = upload(c->dsid[d], c->sid[d].data(), (size_t)ne))) return fail(rc);
    if (c->U[d].alloc(bv4_bytes(ne)) || c->dU[d].alloc(bv4_bytes(ne)) || c->E[d].alloc(bv3_bytes(ne)) ||
        c->H[d].alloc(bv3_bytes(ne)) || c->dE[d].alloc(bv3_bytes(ne)) || c->dH[d].alloc(bv3_bytes(ne)))
      return fail(BEM3_ERR_CUDA);
    cudaMemset(c->U[d].p, 0, bv4_bytes(ne)); cudaMemset(c->dU[d].p, 0, bv4_bytes(ne));
    cudaMemset(c->E[d].p, 0, bv3_bytes(ne)); cudaMemset(c->H[d].p, 0, bv3_bytes(ne));
    cudaMemset(c->dE[d].p, 0, bv3_bytes(ne)); cudaMemset(c->dH[d].p, 0, bv3_bytes(ne));
  }
  if (c->status.alloc(sizeof(int))) return fail(BEM3_ERR_CUDA);
  if (cudaStreamSynchronize(cudaStreamPerThread) != cudaSuccess) return fail(BEM3_ERR_CUDA);
  *out = c;
  return 0;
}

extern "C" void bem3_ctx_destroy(bem3_ctx c)
{
  if (!c) return;
  DeviceGuard g(c->dev);
  delete c;
}

extern "C" int bem3_ctx_get_bv(bem3_ctx c, bem3_bv* out)
{
  if (!c || !out) return BEM3_ERR_ARG;
  DeviceGuard g(c->dev);
  for (int d = 0; d <= c->MN; d++) {
    const int ne = (int)c->sid[d].size();
    if ((out[d].U && cudaMemcpy(out[d].U, c->U[d].p, bv4_bytes(ne), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (out[d].dU && cudaMemcpy(out[d].dU, c->dU[d].p, bv4_bytes(ne), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (out[d].E && cudaMemcpy(out[d].E, c->E[d].p, bv3_bytes(ne), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (out[d].H && cudaMemcpy(out[d].H, c->H[d].p, bv3_bytes(ne), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (out[d].dE && cudaMemcpy(out[d].dE, c->dE[d].p, bv3_bytes(ne), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (out[d].dH && cudaMemcpy(out[d].dH, c->dH[d].p, bv3_bytes(ne), cudaMemcpyDeviceToHost) != cudaSuccess))
      return BEM3_ERR_CUDA;
  }
  return 0;
}

extern "C" int bem3_ctx_set_bv(bem3_ctx c, const bem3_bv* bv)
{
  if (!c || !bv) return BEM3_ERR_ARG;
  DeviceGuard g(c->dev);
  for (int d = 0; d <= c->MN; d++) {
    const int ne = (int)c->sid[d].size();
    if (!bv[d].U || !bv[d].dU || !bv[d].E || !bv[d].H || !bv[d].dE || !bv[d].dH) return BEM3_ERR_ARG;
    if (cudaMemcpy(c->U[d].p, bv[d].U, bv4_bytes(ne), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->dU[d].p, bv[d].dU, bv4_bytes(ne), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->E[d].p, bv[d].E, bv3_bytes(ne), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->H[d].p, bv[d].H, bv3_bytes(ne), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->dE[d].p, bv[d].dE, bv3_bytes(ne), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->dH[d].p, bv[d].dH, bv3_bytes(ne), cudaMemcpyHostToDevice) != cudaSuccess)
      return BEM3_ERR_CUDA;
  }
  return 0;
}

namespace {

// Column-major LU factorisation and solves (cuSOLVER), workspace and pivots owned by the caller.
int lu_factor_cm(cusolverDnHandle_t h, double* A, int n, DevBuf& ipiv)
{
  int lwork = 0;
  if (cusolverDnZgetrf_bufferSize(h, n, n, (cuDoubleComplex*)A, n, &lwork) != CUSOLVER_STATUS_SUCCESS) return BEM3_ERR_SOLVE;
  DevBuf work, info;
  if (work.alloc(sizeof(cuDoubleComplex) * (size_t)(lwork > 0 ? lwork : 1)) || ipiv.alloc(sizeof(int) * (size_t)n) ||
      info.alloc(sizeof(int)))
    return BEM3_ERR_CUDA;
  if (cusolverDnZgetrf(h, n, n, (cuDoubleComplex*)A, n, work.as<cuDoubleComplex>(), ipiv.as<int>(), info.as<int>()) !=
      CUSOLVER_STATUS_SUCCESS)
    return BEM3_ERR_SOLVE;
  int hinfo = 0;
  if (cudaMemcpy(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return BEM3_ERR_CUDA;
  return hinfo == 0 ? 0 : BEM3_ERR_SOLVE;
}

int lu_solve_cm(cusolverDnHandle_t h, const double* A, int n, DevBuf& ipiv, double* B, int nrhs)
{
  DevBuf info;
  if (info.alloc(sizeof(int))) return BEM3_ERR_CUDA;
  if (cusolverDnZgetrs(h, CUBLAS_OP_N, n, nrhs, (const cuDoubleComplex*)A, n, ipiv.as<int>(), (cuDoubleComplex*)B, n,
                       info.as<int>()) != CUSOLVER_STATUS_SUCCESS)
    return BEM3_ERR_SOLVE;
  int hinfo = 0;
  if (cudaMemcpy(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return BEM3_ERR_CUDA;
  return hinfo == 0 ? 0 : BEM3_ERR_SOLVE;
}

int zgemm_nn(cublasHandle_t hb, int m, int n, int k, const double* A, int lda, const double* B, int ldb, double beta,
             double* C, int ldc)
{
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), bt = make_cuDoubleComplex(beta, 0.0);
  return cublasZgemm(hb, CUBLAS_OP_N, CUBLAS_OP_N, m, n, k, &one, (const cuDoubleComplex*)A, lda,
                     (const cuDoubleComplex*)B, ldb, &bt, (cuDoubleComplex*)C, ldc) == CUBLAS_STATUS_SUCCESS
             ? 0
             : BEM3_ERR_SOLVE;
}

unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// Two-colouring of the domain graph (an edge per element between its two domains); the class of
// domain 0 is eliminated.  Returns false when the graph is not bipartite.
bool colour_domains(bem3_ctx c, std::vector<int>& elim)
{
  const int MN = c->MN;
  std::vector<std::vector<int>> adj(MN + 1);
  for (int e = 1; e <= c->Ne; e++) {
    adj[c->md_h[e]].push_back(c->sd_h[e]);
    adj[c->sd_h[e]].push_back(c->md_h[e]);
  }
  std::vector<int> col(MN + 1, -1);
  for (int s = 0; s <= MN; s++) {
    if (col[s] >= 0) continue;
    col[s] = 0;
    std::vector<int> st{s};
    while (!st.empty()) {
      int u = st.back();
      st.pop_back();
      for (int v : adj[u]) {
        if (v == u) return false;
        if (col[v] < 0) { col[v] = 1 - col[u]; st.push_back(v); }
        else if (col[v] == col[u]) return false;
      }
    }
  }
  elim.assign(MN + 1, 0);
  for (int d = 0; d <= MN; d++) elim[d] = (col[d] == col[0]);
  return true;
}

// cuSOLVER / cuBLAS handles, created once per host thread and device and kept (creating them
// costs milliseconds, more than a small problem's whole solve stage).
struct Handles {
  cusolverDnHandle_t s = nullptr;
  cublasHandle_t b = nullptr;
  int init()
  {
    // the libraries' own default is the legacy stream, which would serialise with every thread
    if (!s && cusolverDnCreate(&s) != CUSOLVER_STATUS_SUCCESS) { s = nullptr; return BEM3_ERR_CUDA; }
    if (!b && cublasCreate(&b) != CUBLAS_STATUS_SUCCESS) { b = nullptr; return BEM3_ERR_CUDA; }
    if (cusolverDnSetStream(s, cudaStreamPerThread) != CUSOLVER_STATUS_SUCCESS ||
        cublasSetStream(b, cudaStreamPerThread) != CUBLAS_STATUS_SUCCESS)
      return BEM3_ERR_CUDA;
    return 0;
  }
};

// One set per device, released when the thread ends (the main thread's before the runtime's
// own teardown at exit).
struct ThreadHandles {
  Handles h[64];
  ~ThreadHandles()
  {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return;
    for (int d = 0; d < 64; d++) {
      if (!h[d].s && !h[d].b) continue;
      if (cudaSetDevice(d) != cudaSuccess) continue;
      if (h[d].b) cublasDestroy(h[d].b);
      if (h[d].s) cusolverDnDestroy(h[d].s);
    }
    cudaSetDevice(cur);
  }
};

Handles& thread_handles(int dev)
{
  static thread_local ThreadHandles t;
  return t.h[(dev >= 0 && dev < 64) ? dev : 0];
}

DtnArgs dtn_view(bem3_ctx c, const SolveState& T, const SolveDev& S)
{
  DtnArgs A;
  A.node = T.nodes.p ? (const DtnNode*)T.nodes.p : nullptr;
  A.geo = S.geo; A.md = S.md; A.sd = S.sd; A.kn = S.kn; A.NN = c->NN;
  return A;
}

SolveDev solve_view_with(bem3_ctx c, SolveState& T)
{
  SolveDev S = solve_view(c);
  for (int d = 0; d <= c->MN; d++) {
    S.G[d] = T.G[d].as<double>(); S.H[d] = T.H[d].as<double>();
    S.dG[d] = T.dG[d].as<double>(); S.dH[d] = T.dH[d].as<double>(); S.dF[d] = T.dF[d].as<double>();
  }
  return S;
}

// Phase 1a: the buffers of every domain's coefficient matrices and the node tables.
int phase_alloc(bem3_ctx c, SolveState& T)
{
  const int MN = c->MN;
  int rc;
  for (int d = 0; d <= MN; d++) {
    const int ne = (int)c->sid[d].size();
    const size_t N = (size_t)4 * ne;
    if (T.G[d].alloc(N * N * 16) || T.H[d].alloc(N * N * 16) || T.dG[d].alloc(2 * N * N * 16) ||
        T.dH[d].alloc(2 * N * N * 16) || T.dF[d].alloc(N * 3 * 8))
      return BEM3_ERR_CUDA;
    T.bytes += N * N * 16 * 6 + N * 24;
    std::vector<int> gn, cm;
    for (int t = 0; t < ne; t++) {
      const int a = abs(c->sid[d][t]);
      for (int tn = 0; tn < c->nv[a]; tn++) {
        gn.push_back(c->eni_h[4 * a + tn]);
        cm.push_back(4 * t + tn);
      }
    }
    T.n[d] = (int)gn.size();
    if ((rc = upload(T.gnode[d], gn.data(), gn.size())) || (rc = upload(T.cmap[d], cm.data(), cm.size()))) return rc;
  }
  return 0;
}

// Phase 1b: the coefficient matrices of every domain (create_cmatrix, d3qd2_solve_bieq.c:156-163).
int phase_assemble(bem3_ctx c, SolveState& T)
{
  int rc = phase_alloc(c, T);
  if (rc) return rc;
  for (int d = 0; d <= c->MN; d++) {
    const int periodic = (d == 0 && c->ps == 1) ? 1 : 0;
    rc = bem3_assemble_domain_dev(c->geo.as<double>(), c->Ne, c->dsid[d].as<int>(), (int)c->sid[d].size(), d,
                                  periodic, &c->qd, c->kn[2 * d], c->kn[2 * d + 1], T.G[d].as<double>(),
                                  T.H[d].as<double>(), T.dG[d].as<double>(), T.dH[d].as<double>(),
                                  T.dF[d].as<double>(), nullptr);
    if (rc) return rc;
  }
  return 0;
}

// Phase 2: factorisations.  Every domain's compacted G (for the dE, dH systems and the maps),
// then the system of the potentials in the reduced form when the domain graph allows it.
int phase_factor(bem3_ctx c, SolveState& T, const SolveDev& S, Handles& hd)
{
  const int MN = c->MN, NN = c->NN;
  int rc;
  bool reduced = (c->solver != 1) && colour_domains(c, T.elim);
  std::vector<DtnNode> nodes;
  if (reduced) {
    nodes.assign((size_t)NN, DtnNode{});
    std::vector<int> seen((size_t)NN, 0);
    for (int d = 0; d <= MN; d++) {
      int j = 0;
      for (int t = 0; t < (int)c->sid[d].size(); t++) {
        const int a = abs(c->sid[d][t]);
        for (int tn = 0; tn < c->nv[a]; tn++, j++) {
          const int g = c->eni_h[4 * a + tn];
          if (g < 0 || g >= NN) return BEM3_ERR_ARG;
          DtnNode& q = nodes[g];
          q.elem = a; q.l = tn;
          if (T.elim[d]) { q.de = d; q.le = j; seen[g] |= 1; }
          else { q.dn = d; q.ln = j; seen[g] |= 2; }
        }
      }
    }
    for (int g = 0; g < NN; g++)
      if (seen[g] != 3) reduced = false;
  }
  if (!reduced && c->solver == 2) return BEM3_ERR_ARG;  // reduced form asked for but not applicable
  // compacted G of every domain; the reduced form needs the eliminated domains' K_d first (from
  // the factorised G_d) and the kept domains' G_e unfactorised for their rows
  for (int d = 0; d <= MN; d++) {
    const int n = T.n[d], N = 4 * (int)c->sid[d].size();
    if (T.Gc[d].alloc((size_t)n * n * 16)) return BEM3_ERR_CUDA;
    T.bytes += (size_t)n * n * 16;
    k_compact_cm<<<nblk((long long)n * n, 256), 256>>>(S.G[d], N, T.cmap[d].as<int>(), n, T.Gc[d].as<double>());
  }
  KPtrs KP;
  memset(&KP, 0, sizeof KP);
  if (reduced) {
    if ((rc = upload(T.nodes, nodes.data(), nodes.size()))) return rc;
    for (int d = 0; d <= MN; d++) {
      if (!T.elim[d]) continue;
      const int n = T.n[d], N = 4 * (int)c->sid[d].size();
      if ((rc = lu_factor_cm(hd.s, T.Gc[d].as<double>(), n, T.Gpiv[d]))) return rc;
      if (T.K[d].alloc((size_t)n * n * 16)) return BEM3_ERR_CUDA;
      T.bytes += (size_t)n * n * 16;
      k_compact_cm<<<nblk((long long)n * n, 256), 256>>>(S.H[d], N, T.cmap[d].as<int>(), n, T.K[d].as<double>());
      if ((rc = lu_solve_cm(hd.s, T.Gc[d].as<double>(), n, T.Gpiv[d], T.K[d].as<double>(), n))) return rc;
      KP.K[d] = T.K[d].as<double>(); KP.n[d] = n;
    }
    const DtnArgs A = dtn_view(c, T, S);
    const long long na = 4LL * NN;
    if (T.A.alloc((size_t)na * na * 16)) return BEM3_ERR_CUDA;
    T.bytes += (size_t)na * na * 16;
    long long row0 = 0;
    for (int e = 0; e <= MN; e++) {
      if (T.elim[e]) continue;
      const int n = T.n[e], N = 4 * (int)c->sid[e].size();
      DevBuf Hc, Kh, P, Q;
      if (Hc.alloc((size_t)n * n * 16) || Kh.alloc((size_t)n * NN * 16) || P.alloc((size_t)n * NN * 16) ||
          Q.alloc((size_t)n * NN * 16))
        return BEM3_ERR_CUDA;
      k_compact_cm<<<nblk((long long)n * n, 256), 256>>>(S.H[e], N, T.cmap[e].as<int>(), n, Hc.as<double>());
      k_dtn_khat<<<nblk((long long)n * NN, 256), 256>>>(A, KP, T.gnode[e].as<int>(), n, e, 0, Kh.as<double>());
      if ((rc = zgemm_nn(hd.b, n, NN, n, T.Gc[e].as<double>(), n, Kh.as<double>(), n, 0.0, P.as<double>(), n))) return rc;
      k_dtn_khat<<<nblk((long long)n * NN, 256), 256>>>(A, KP, T.gnode[e].as<int>(), n, e, 1, Kh.as<double>());
      if ((rc = zgemm_nn(hd.b, n, NN, n, T.Gc[e].as<double>(), n, Kh.as<double>(), n, 0.0, Q.as<double>(), n))) return rc;
      k_dtn_rows<<<nblk(4LL * n * na, 256), 256>>>(A, e, T.gnode[e].as<int>(), n, Hc.as<double>(), T.Gc[e].as<double>(),
                                                   P.as<double>(), Q.as<double>(), T.A.as<double>(), na, row0);
      if ((rc = lu_factor_cm(hd.s, T.Gc[e].as<double>(), n, T.Gpiv[e]))) return rc;
      row0 += 4LL * n;
    }
    if (row0 != na) return BEM3_ERR_ARG;
    if ((rc = lu_factor_cm(hd.s, T.A.as<double>(), (int)na, T.Apiv))) return rc;
    T.method = 2;
    return 0;
  }
  for (int d = 0; d <= MN; d++)
    if ((rc = lu_factor_cm(hd.s, T.Gc[d].as<double>(), T.n[d], T.Gpiv[d]))) return rc;
  // the reference's system, rows in create_tmatrix_csr order, stored row-major (solved transposed)
  const long long na = 8LL * NN;
  std::vector<int4> rowmap;
  rowmap.reserve((size_t)na);
  for (int d = 0; d <= MN; d++)
    for (int cid = 0; cid < 4; cid++)
      for (int t = 0; t < (int)c->sid[d].size(); t++) {
        const int nv = c->nv[abs(c->sid[d][t])];
        for (int tn = 0; tn < nv; tn++) rowmap.push_back(make_int4(d, cid, t, tn));
      }
  if ((long long)rowmap.size() != na) return BEM3_ERR_ARG;
  DevBuf drow, scratchB;
  if ((rc = upload(drow, rowmap.data(), rowmap.size()))) return rc;
  if (T.A.alloc((size_t)na * na * 16) || scratchB.alloc((size_t)na * 16)) return BEM3_ERR_CUDA;
  T.bytes += (size_t)na * na * 16;
  cudaMemset(T.A.p, 0, (size_t)na * na * 16);
  k_build_rows<<<(unsigned)na, 256>>>(S, drow.as<int4>(), T.A.as<double>(), scratchB.as<double>(), na);
  if (cudaGetLastError() != cudaSuccess) return BEM3_ERR_CUDA;
  // row-major A is A^T column-major: factorising that and solving with the transpose gives A x = b
  if ((rc = lu_factor_cm(hd.s, T.A.as<double>(), (int)na, T.Apiv))) return rc;
  T.method = 1;
  return 0;
}

int lu_solve_cm_t(cusolverDnHandle_t h, const double* A, int n, DevBuf& ipiv, double* B, int nrhs)
{
  DevBuf info;
  if (info.alloc(sizeof(int))) return BEM3_ERR_CUDA;
  if (cusolverDnZgetrs(h, CUBLAS_OP_T, n, nrhs, (const cuDoubleComplex*)A, n, ipiv.as<int>(), (cuDoubleComplex*)B, n,
                       info.as<int>()) != CUSOLVER_STATUS_SUCCESS)
    return BEM3_ERR_SOLVE;
  int hinfo = 0;
  if (cudaMemcpy(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return BEM3_ERR_CUDA;
  return hinfo == 0 ? 0 : BEM3_ERR_SOLVE;
}

// Phase 3: the incident field's right-hand sides, the potentials, then E, H and dE, dH.
int phase_rhs(bem3_ctx c, SolveState& T, const SolveDev& S, Handles& hd)
{
  const int MN = c->MN, NN = c->NN;
  int rc;
  const long long nx = 8LL * NN;
  DevBuf X, B[BEM3_MAXDOM];
  if (X.alloc((size_t)nx * 16)) return BEM3_ERR_CUDA;
  for (int d = 0; d <= MN; d++) {
    if (B[d].alloc((size_t)T.n[d] * 4 * 16)) return BEM3_ERR_CUDA;
    k_dtn_rhs<<<dim3(T.n[d], 4), 256>>>(S, d, T.cmap[d].as<int>(), T.n[d], B[d].as<double>());
  }
  if (T.method == 2) {
    const DtnArgs A = dtn_view(c, T, S);
    KPtrs GP;
    memset(&GP, 0, sizeof GP);
    for (int d = 0; d <= MN; d++) {  // g^d = G_d^-1 b^d (in place)
      if (!T.elim[d]) continue;
      if ((rc = lu_solve_cm(hd.s, T.Gc[d].as<double>(), T.n[d], T.Gpiv[d], B[d].as<double>(), 4))) return rc;
      GP.K[d] = B[d].as<double>(); GP.n[d] = T.n[d];
    }
    const long long na = 4LL * NN;
    DevBuf rhs;
    if (rhs.alloc((size_t)na * 16)) return BEM3_ERR_CUDA;
    long long row0 = 0;
    for (int e = 0; e <= MN; e++) {
      if (T.elim[e]) continue;
      const int n = T.n[e], N = 4 * (int)c->sid[e].size();
      DevBuf Gh;
      if (Gh.alloc((size_t)n * 4 * 16)) return BEM3_ERR_CUDA;
      k_dtn_ghat<<<nblk(4LL * n, 256), 256>>>(A, GP, T.gnode[e].as<int>(), n, e, Gh.as<double>());
      k_compact_matvec4<<<n, 256>>>(S.G[e], N, T.cmap[e].as<int>(), n, Gh.as<double>(), B[e].as<double>());
      if (cudaMemcpy(rhs.as<double>() + 2 * row0, B[e].p, (size_t)n * 4 * 16, cudaMemcpyDeviceToDevice) != cudaSuccess)
        return BEM3_ERR_CUDA;
      row0 += 4LL * n;
    }
    if ((rc = lu_solve_cm(hd.s, T.A.as<double>(), (int)na, T.Apiv, rhs.as<double>(), 1))) return rc;
    for (int d = 0; d <= MN; d++) {
      if (!T.elim[d]) continue;
      const int n = T.n[d];
      DevBuf Ud, KU;
      if (Ud.alloc((size_t)n * 4 * 16) || KU.alloc((size_t)n * 4 * 16)) return BEM3_ERR_CUDA;
      k_dtn_gather_u<<<nblk(4LL * n, 256), 256>>>(T.gnode[d].as<int>(), n, NN, rhs.as<double>(), Ud.as<double>());
      if ((rc = zgemm_nn(hd.b, n, 4, n, T.K[d].as<double>(), n, Ud.as<double>(), n, 0.0, KU.as<double>(), n))) return rc;
      k_dtn_du<<<nblk(n, 128), 128>>>(A, d, T.gnode[d].as<int>(), n, KU.as<double>(), B[d].as<double>(),
                                      rhs.as<double>(), X.as<double>());
    }
  } else if (T.method == 1) {
    // right-hand side of the full system in its row order: domain by domain, component-major
    long long off = 0;
    for (int d = 0; d <= MN; d++) {
      if (cudaMemcpy(X.as<double>() + 2 * off, B[d].p, (size_t)T.n[d] * 4 * 16, cudaMemcpyDeviceToDevice) !=
          cudaSuccess)
        return BEM3_ERR_CUDA;
      off += 4LL * T.n[d];
    }
    if ((rc = lu_solve_cm_t(hd.s, T.A.as<double>(), (int)nx, T.Apiv, X.as<double>(), 1))) return rc;
  } else {
    return BEM3_ERR_ARG;
  }
  for (int d = 0; d <= MN; d++) k_store_bv<<<(4 * S.ne[d] + 127) / 128, 128>>>(S, d, X.as<double>());
  // boundary fields E, H (interior domains, and the open-region side of their nodes)
  for (int d = 1; d <= MN; d++) k_eh_interior<<<(4 * S.ne[d] * 32 + 255) / 256, 256>>>(S, d);
  // normal derivatives: G_d [dE dH] = H_d [E H] with the factorised compacted G_d
  for (int d = 0; d <= MN; d++) {
    const int nn = T.n[d];
    DevBuf dBd;
    if (dBd.alloc((size_t)nn * 6 * 16)) return BEM3_ERR_CUDA;
    k_deh_system<<<nn, 256>>>(S, d, T.cmap[d].as<int>(), nn, nullptr, dBd.as<double>());
    if ((rc = lu_solve_cm(hd.s, T.Gc[d].as<double>(), nn, T.Gpiv[d], dBd.as<double>(), 6))) return rc;
    k_deh_store<<<(nn + 127) / 128, 128>>>(S, d, T.cmap[d].as<int>(), nn, dBd.as<double>());
  }
  if (cudaStreamSynchronize(cudaStreamPerThread) != cudaSuccess) return BEM3_ERR_CUDA;
  return 0;
}

}  // namespace

extern "C" int bem3_ctx_set_solver(bem3_ctx c, int method)
{
  if (!c || method < 0 || method > 2) return BEM3_ERR_ARG;
  c->solver = method;
  return 0;
}

namespace {
// CUDA events around the solve's phases on the calling thread's stream (the one all its work goes to).
struct PhaseClock {
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  bool ok = true;
  PhaseClock()
  {
    for (auto& e : ev)
      if (cudaEventCreate(&e) != cudaSuccess) { e = nullptr; ok = false; }
  }
  ~PhaseClock()
  {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  }
  void mark(int i) { if (ok) cudaEventRecord(ev[i], cudaStreamPerThread); }
  // elapsed ms between marks lo..hi into out[], after waiting for the last mark
  void read(int lo, int hi, double* out)
  {
    if (!ok || cudaEventSynchronize(ev[hi]) != cudaSuccess) return;
    for (int i = lo; i < hi; i++) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ev[i], ev[i + 1]) == cudaSuccess) out[i - lo] = ms;
    }
  }
};
}  // namespace

extern "C" int bem3_ctx_solve(bem3_ctx c)
{
  if (!c) return BEM3_ERR_ARG;
  DeviceGuard g(c->dev);
  delete c->st;
  c->st = new SolveState();
  SolveState& T = *c->st;
  PhaseClock clk;
  clk.mark(0);
  int rc = phase_assemble(c, T);
  if (rc) { delete c->st; c->st = nullptr; return rc; }
  clk.mark(1);
  SolveDev S = solve_view_with(c, T);
  Handles& hd = thread_handles(c->dev);
  if ((rc = hd.init()) || (rc = phase_factor(c, T, S, hd))) {
    delete c->st;
    c->st = nullptr;
    return rc;
  }
  clk.mark(2);
  if ((rc = phase_rhs(c, T, S, hd))) {
    delete c->st;
    c->st = nullptr;
    return rc;
  }
  clk.mark(3);
  c->phase_ms[0] = c->phase_ms[1] = c->phase_ms[2] = 0.0;
  clk.read(0, 3, c->phase_ms);
  return 0;
}

extern "C" int bem3_ctx_prepare(bem3_ctx c, bem3_batch_domain* doms)
{
  if (!c || !doms) return BEM3_ERR_ARG;
  DeviceGuard g(c->dev);
  delete c->st;
  c->st = new SolveState();
  int rc = phase_alloc(c, *c->st);
  if (rc) { delete c->st; c->st = nullptr; return rc; }
  for (int d = 0; d <= c->MN; d++) {
    bem3_batch_domain& b = doms[d];
    SolveState& T = *c->st;
    b.geo = c->geo.as<double>(); b.Ne = c->Ne;
    b.sid = c->dsid[d].as<int>(); b.Ne_d = (int)c->sid[d].size(); b.did = d;
    b.periodic = (d == 0 && c->ps == 1) ? 1 : 0;
    b.qd = c->qd; b.kre = c->kn[2 * d]; b.kim = c->kn[2 * d + 1];
    b.G = T.G[d].as<double>(); b.H = T.H[d].as<double>(); b.dG = T.dG[d].as<double>(); b.dH = T.dH[d].as<double>();
    b.dF = T.dF[d].as<double>();
  }
  return 0;
}

extern "C" int bem3_ctx_solve_prepared(bem3_ctx c)
{
  if (!c || !c->st || c->st->method) return BEM3_ERR_ARG;
  DeviceGuard g(c->dev);
  SolveState& T = *c->st;
  PhaseClock clk;
  clk.mark(1);
  SolveDev S = solve_view_with(c, T);
  Handles& hd = thread_handles(c->dev);
  int rc;
  if ((rc = hd.init()) || (rc = phase_factor(c, T, S, hd))) {
    delete c->st;
    c->st = nullptr;
    return rc;
  }
  clk.mark(2);
  if ((rc = phase_rhs(c, T, S, hd))) {
    delete c->st;
    c->st = nullptr;
    return rc;
  }
  clk.mark(3);
  c->phase_ms[0] = c->phase_ms[1] = c->phase_ms[2] = 0.0;
  clk.read(1, 3, c->phase_ms + 1);
  return 0;
}

extern "C" int bem3_ctx_phase_times(bem3_ctx c, double* ms)
{
  if (!c || !ms) return BEM3_ERR_ARG;
  for (int i = 0; i < 3; i++) ms[i] = c->phase_ms[i];
  return 0;
}

extern "C" int bem3_ctx_set_incident(bem3_ctx c, int nwaves, const bem3_wave* waves, const double* Ui,
                                     const double* dUi, const double* dEiz, const double* dEie)
{
  if (!c || nwaves < 0 || (nwaves > 0 && !waves) || !Ui || !dUi || !dEiz || !dEie) return BEM3_ERR_ARG;
  DeviceGuard g(c->dev);
  const size_t Ne1 = (size_t)c->Ne + 1;
  if (cudaMemcpy(c->Ui.p, Ui, Ne1 * 32 * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->dUi.p, dUi, Ne1 * 32 * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->dEiz.p, dEiz, Ne1 * 24 * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->dEie.p, dEie, Ne1 * 24 * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
    return BEM3_ERR_CUDA;
  if (nwaves > 0) {
    DevBuf w;
    int rc = upload(w, waves, (size_t)nwaves);
    if (rc) return rc;
    std::swap(c->waves.p, w.p);
  }
  c->nwaves = nwaves;
  return 0;
}

extern "C" int bem3_ctx_resolve(bem3_ctx c)
{
  if (!c) return BEM3_ERR_ARG;
  if (!c->st || !c->st->method) return bem3_ctx_solve(c);
  DeviceGuard g(c->dev);
  SolveState& T = *c->st;
  SolveDev S = solve_view_with(c, T);
  Handles& hd = thread_handles(c->dev);
  int rc = hd.init();
  PhaseClock clk;
  clk.mark(2);
  if (!rc) rc = phase_rhs(c, T, S, hd);
  clk.mark(3);
  if (!rc) {
    c->phase_ms[0] = c->phase_ms[1] = c->phase_ms[2] = 0.0;
    clk.read(2, 3, c->phase_ms + 2);
  }
  return rc;
}

extern "C" int bem3_ctx_release(bem3_ctx c)
{
  if (!c) return BEM3_ERR_ARG;
  DeviceGuard g(c->dev);
  delete c->st;
  c->st = nullptr;
  return 0;
}

extern "C" size_t bem3_ctx_device_bytes(bem3_ctx c) { return (c && c->st) ? c->st->bytes : 0; }

namespace {

FieldArgs field_view(bem3_ctx c)
{
  FieldArgs A;
  memset(&A, 0, sizeof A);
  A.geo = c->geo.as<double>(); A.rn = c->rn.as<double>(); A.ed = c->ed.as<int>();
  A.MN = c->MN; A.ps = c->ps;
  A.dlist = c->dlist.as<int>(); A.dsd = c->dsd.as<int>();
  for (int d = 0; d <= c->MN + 1; d++) A.doff[d] = c->doff[d];
  for (int d = 0; d <= c->MN; d++) {
    A.ne[d] = (int)c->sid[d].size();
    A.sid[d] = c->dsid[d].as<int>();
    A.E[d] = c->E[d].as<double>(); A.dE[d] = c->dE[d].as<double>();
    A.H[d] = c->H[d].as<double>(); A.dH[d] = c->dH[d].as<double>();
    A.U[d] = c->U[d].as<double>(); A.dU[d] = c->dU[d].as<double>();
    A.kn[2 * d] = c->kn[2 * d]; A.kn[2 * d + 1] = c->kn[2 * d + 1];
  }
  A.vk0 = c->qd.vk[0]; A.vk1 = c->qd.vk[1];
  A.d1x = c->qd.vd1[0]; A.d1y = c->qd.vd1[1]; A.d2x = c->qd.vd2[0]; A.d2y = c->qd.vd2[1];
  const double det = A.d1x * A.d2y - A.d2x * A.d1y;
  A.i_detd = det != 0.0 ? 1.0 / det : 0.0;
  A.waves = c->waves.as<bem3_wave>(); A.nwaves = c->nwaves;
  return A;
}

int run_domain_id(bem3_ctx c, const FieldArgs& A, int n, const double* r, DevBuf& dr, DevBuf& ddid, DevBuf& dcell)
{
  int rc;
  if ((rc = upload(dr, r, (size_t)3 * n))) return rc;
  if (ddid.alloc(sizeof(int) * (size_t)n) || dcell.alloc(sizeof(int2) * (size_t)n)) return BEM3_ERR_CUDA;
  k_domain_id<<<(unsigned)(((size_t)n * 32 + 255) / 256), 256>>>(A, n, dr.as<double>(), ddid.as<int>(),
                                                                  dcell.as<int2>());
  return cudaGetLastError() == cudaSuccess ? 0 : BEM3_ERR_CUDA;
}

}  // namespace

extern "C" int bem3_ctx_domain_id(bem3_ctx c, int n, const double* r, int* did)
{
  if (!c || n < 0 || (n > 0 && (!r || !did))) return BEM3_ERR_ARG;
  if (n == 0) return 0;
  DeviceGuard g(c->dev);
  FieldArgs A = field_view(c);
  DevBuf dr, ddid, dcell;
  int rc = run_domain_id(c, A, n, r, dr, ddid, dcell);
  if (rc) return rc;
  return cudaMemcpy(did, ddid.p, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : BEM3_ERR_CUDA;
}

// E, H (pot false) or U (pot true) at n points; mode 0 scattered / interior, 1 total, 2 incident.
static int ctx_field_run(bem3_ctx c, int n, const double* r, int type, int mode, bool pot, double* E, double* H,
                         int* did)
{
  if (!c || n < 0 || (n > 0 && (!r || !E || (!pot && !H))) || type < 0 || type > 3 || mode < 0 || mode > 2)
    return BEM3_ERR_ARG;
  if (n == 0) return 0;
  DeviceGuard g(c->dev);
  if (type >= 2 && ensure_tables() != 0) return BEM3_ERR_CUDA;  // Gauss-Legendre tables
  FieldArgs A = field_view(c);
  DevBuf dr, ddid, dcell, dE, dH;
  int rc = run_domain_id(c, A, n, r, dr, ddid, dcell);
  if (rc) return rc;
  const size_t eo = (size_t)n * (pot ? 8 : 6) * sizeof(double);
  if (dE.alloc(eo) || (!pot && dH.alloc((size_t)n * 6 * sizeof(double)))) return BEM3_ERR_CUDA;
  cudaMemset(c->status.p, 0, sizeof(int));
  if (pot)
    k_field_t<true><<<(unsigned)n, FIELD_THREADS>>>(A, c->L, n, dr.as<double>(), ddid.as<int>(), dcell.as<int2>(), type,
                                                    mode, dE.as<double>(), nullptr, c->status.as<int>());
  else
    k_field_t<false><<<(unsigned)n, FIELD_THREADS>>>(A, c->L, n, dr.as<double>(), ddid.as<int>(), dcell.as<int2>(), type,
                                                     mode, dE.as<double>(), dH.as<double>(), c->status.as<int>());
  if (cudaGetLastError() != cudaSuccess) return BEM3_ERR_CUDA;
  int hs = 0;
  if (cudaMemcpy(&hs, c->status.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(E, dE.p, eo, cudaMemcpyDeviceToHost) != cudaSuccess ||
      (!pot && cudaMemcpy(H, dH.p, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ||
      (did && cudaMemcpy(did, ddid.p, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess))
    return BEM3_ERR_CUDA;
  return hs;
}

extern "C" int bem3_ctx_field(bem3_ctx c, int n, const double* r, int type, int total, double* E, double* H, int* did)
{
  return ctx_field_run(c, n, r, type, total, false, E, H, did);
}

extern "C" int bem3_ctx_potential(bem3_ctx c, int n, const double* r, int type, int total, double* U, int* did)
{
  return ctx_field_run(c, n, r, type, total, true, U, nullptr, did);
}

extern "C" int bem3_ctx_field_memp(bem3_ctx c, int n, const double* r, int type, int total, double* E, double* H,
                                   int* did)
{
  if (!c || n < 0 || (n > 0 && (!r || !E || !H)) || type < 0 || type > 3 || total < 0 || total > 2) return BEM3_ERR_ARG;
  if (n == 0) return 0;
  DeviceGuard g(c->dev);
  if (type >= 2 && ensure_tables() != 0) return BEM3_ERR_CUDA;
  FieldArgs A = field_view(c);
  DevBuf dr, ddid, dcell, dE, dH;
  int rc = run_domain_id(c, A, n, r, dr, ddid, dcell);
  if (rc) return rc;
  if (dE.alloc((size_t)n * 6 * sizeof(double)) || dH.alloc((size_t)n * 6 * sizeof(double))) return BEM3_ERR_CUDA;
  cudaMemset(c->status.p, 0, sizeof(int));
  k_eh_memp<<<(unsigned)n, FIELD_THREADS>>>(A, c->L, n, dr.as<double>(), ddid.as<int>(), dcell.as<int2>(), type, total,
                                            c->lambda0, dE.as<double>(), dH.as<double>(), c->status.as<int>());
  if (cudaGetLastError() != cudaSuccess) return BEM3_ERR_CUDA;
  int hs = 0;
  if (cudaMemcpy(&hs, c->status.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(E, dE.p, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(H, dH.p, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
      (did && cudaMemcpy(did, ddid.p, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess))
    return BEM3_ERR_CUDA;
  return hs;
}

extern "C" int bem3_ctx_force(bem3_ctx c, const double* rc, int type, double* F, double* N)
{
  if (!c || !rc || !F || !N || (type != 0 && type != 1)) return BEM3_ERR_ARG;
  DeviceGuard g(c->dev);
  const int ne = (int)c->sid[0].size();
  // the boundary field at points other than nodes needs the periodic self rule
  bool needs_bd = (type == 1);
  for (int s : c->sid[0]) needs_bd = needs_bd || (c->nv[abs(s)] == 3);
  if (needs_bd && c->ps != 1) return BEM3_ERR_ARG;
  if (ensure_tables() != 0) return BEM3_ERR_CUDA;
  ForceArgs A;
  memset(&A, 0, sizeof A);
  A.geo = c->geo.as<double>(); A.ne = ne; A.sid = c->dsid[0].as<int>();
  A.E = c->E[0].as<double>(); A.dE = c->dE[0].as<double>(); A.H = c->H[0].as<double>(); A.dH = c->dH[0].as<double>();
  A.k0re = c->kn[0]; A.k0im = c->kn[1];
  const double n0 = c->kn[0] * c->lambda0 / (2.0 * QP_PI);  // kn[0] = 2 pi n0 / lambda0
  A.epd = n0 * n0;
  for (int l = 0; l < 3; l++) A.rc[l] = rc[l];
  A.type = type;
  A.waves = c->waves.as<bem3_wave>(); A.nwaves = c->nwaves;
  const int npt = ne * FORCE_MAXPTS;
  DevBuf part, res;
  if (part.alloc((size_t)npt * 6 * sizeof(double)) || res.alloc(6 * sizeof(double))) return BEM3_ERR_CUDA;
  cudaMemset(c->status.p, 0, sizeof(int));
  k_force_points<<<npt, FORCE_THREADS>>>(A, c->L, part.as<double>(), c->status.as<int>());
  k_force_sum<<<1, FORCE_THREADS>>>(part.as<double>(), npt, res.as<double>());
  if (cudaGetLastError() != cudaSuccess) return BEM3_ERR_CUDA;
  double h[6];
  int hs = 0;
  if (cudaMemcpy(h, res.p, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&hs, c->status.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return BEM3_ERR_CUDA;
  for (int l = 0; l < 3; l++) { F[l] = h[l]; N[l] = h[3 + l]; }
  return hs;
}

extern "C" int bem3_ctx_field_bd(bem3_ctx c, int did, int n, const int* t, const double* zeta_eta, int type,
                                 int total, double* E, double* H)
{
  if (!c || n < 0 || (n > 0 && (!t || !zeta_eta || !E || !H)) || type < 0 || type > 3 || total < 0 || total > 1)
    return BEM3_ERR_ARG;
  // the open region of a quasi-periodic problem only: the element's own integral uses the periodic
  // self rule (interior domains would need the free-space rule of coef_bd at arbitrary points)
  if (did != 0 || c->ps != 1) return BEM3_ERR_ARG;
  if (n == 0) return 0;
  const int ne = (int)c->sid[0].size();
  std::vector<int> tl((size_t)n);
  for (int i = 0; i < n; i++) {
    if (t[i] < 1 || t[i] > ne) return BEM3_ERR_ARG;
    tl[(size_t)i] = t[i] - 1;
  }
  DeviceGuard g(c->dev);
  if (ensure_tables() != 0) return BEM3_ERR_CUDA;
  ForceArgs A;
  memset(&A, 0, sizeof A);
  A.geo = c->geo.as<double>(); A.ne = ne; A.sid = c->dsid[0].as<int>();
  A.E = c->E[0].as<double>(); A.dE = c->dE[0].as<double>(); A.H = c->H[0].as<double>(); A.dH = c->dH[0].as<double>();
  A.k0re = c->kn[0]; A.k0im = c->kn[1];
  A.waves = c->waves.as<bem3_wave>(); A.nwaves = c->nwaves;
  DevBuf dt, dze, dE, dH;
  int rc;
  if ((rc = upload(dt, tl.data(), (size_t)n)) || (rc = upload(dze, zeta_eta, (size_t)2 * n))) return rc;
  if (dE.alloc((size_t)n * 6 * sizeof(double)) || dH.alloc((size_t)n * 6 * sizeof(double))) return BEM3_ERR_CUDA;
  cudaMemset(c->status.p, 0, sizeof(int));
  k_field_bd<<<(unsigned)n, FORCE_THREADS>>>(A, c->L, n, dt.as<int>(), dze.as<double>(), type, total, dE.as<double>(),
                                             dH.as<double>(), c->status.as<int>());
  if (cudaGetLastError() != cudaSuccess) return BEM3_ERR_CUDA;
  int hs = 0;
  if (cudaMemcpy(&hs, c->status.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(E, dE.p, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(H, dH.p, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return BEM3_ERR_CUDA;
  return hs;
}

extern "C" int bem3_solve_bieq_arrays(const bem3_problem* P, bem3_bv* out)
{
  if (!out) return BEM3_ERR_ARG;
  bem3_ctx c = nullptr;
  int rc = bem3_ctx_create(P, &c);
  if (rc) return rc;
  rc = bem3_ctx_solve(c);
  if (!rc) rc = bem3_ctx_get_bv(c, out);
  bem3_ctx_destroy(c);
  return rc;
}

// capi.cu -- extern "C" entry points (include/bem3_qd2_b200.h) and the per-device resources
// they share: scratch for the assembly, a status word written by the kernels.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "elem.cuh"
#include "bem3_internal.h"

#define MAX_DEV 64

namespace {

struct DevRes {
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  int* status = nullptr;  // device int
  unsigned long long* terms = nullptr;  // device counter (profiling only)
  QPProp* prop = nullptr;               // propagating orders of the lattice being assembled
};

// One set per host thread and device: concurrent assemblies from different threads (each on its
// own stream) never share scratch.  A thread's scratch is kept until the process exits.
thread_local DevRes t_res[MAX_DEV];
thread_local bem3_stats t_last_stats;
thread_local int t_profiling = 0;

int cur_dev()
{
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

// Grows the device scratch of the current device to at least `bytes`.
int ensure_scratch(size_t bytes, DevRes** out)
{
  int d = cur_dev();
  if (d < 0 || d >= MAX_DEV) return BEM3_ERR_ARG;
  DevRes& r = t_res[d];
  if (!r.status) {
    if (cudaMalloc(&r.status, sizeof(int)) != cudaSuccess) return BEM3_ERR_CUDA;
  }
  if (r.scratch_bytes < bytes) {
    if (r.scratch) cudaFree(r.scratch);
    r.scratch = nullptr;
    r.scratch_bytes = 0;
    if (cudaMalloc(&r.scratch, bytes) != cudaSuccess) return BEM3_ERR_CUDA;
    r.scratch_bytes = bytes;
  }
  *out = &r;
  return 0;
}

// The lattice's propagating orders into device memory `dst` (QP_PROP_CAP entries) on `st`, for
// the hoisted spectral sums of the assembly kernels.
int attach_prop_list(QPLattice* L, QPProp* dst, cudaStream_t st)
{
  static thread_local QPProp host[QP_PROP_CAP];
  const int n = qp_prop_list(*L, host, QP_PROP_CAP);
  if (n < 0) return BEM3_ERR_LATTICE;  // more propagating orders than the list holds
  L->prop = dst;
  L->nprop = n;
  if (n > 0 && cudaMemcpyAsync(dst, host, sizeof(QPProp) * (size_t)n, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return BEM3_ERR_CUDA;
  return 0;
}

int lattice_from(const bem3_qpd2* qd, QPLattice* L)
{
  if (!qd) return BEM3_ERR_ARG;
  if (qp_lattice_init(*L, qd->k, qd->vk[0], qd->vk[1], qd->vd1[0], qd->vd1[1], qd->vd2[0], qd->vd2[1]) != 0)
    return BEM3_ERR_LATTICE;
  return 0;
}

}  // namespace

// ------------------------------------------------------------------------------------------
__global__ void k_qpgf_points(const __grid_constant__ QPLattice L, int n, const double* __restrict__ r, double* __restrict__ out,
                              int* __restrict__ ret, int mode)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double p[3] = {r[3 * i], r[3 * i + 1], r[3 * i + 2]};
  QPVal v;
  int e = (mode == 0) ? qpgf_eval<QP_V1>(L, p, v) : qpgf_eval<QP_BOTH>(L, p, v);
  ret[i] = e;
  double* o = out + 8 * (size_t)i;
  o[0] = v.G.re; o[1] = v.G.im;
  for (int c = 0; c < 3; c++) { o[2 + 2 * c] = v.dG[c].re; o[3 + 2 * c] = v.dG[c].im; }
}

extern "C" int bem3_qpgf_dev(const bem3_qpd2* qd, int n, const double* r_dev, double* out_dev, int* ret_dev, int mode,
                             void* stream)
{
  if (n < 0 || (n > 0 && (!r_dev || !out_dev || !ret_dev))) return BEM3_ERR_ARG;
  QPLattice L;
  int e = lattice_from(qd, &L);
  if (e) return e;
  if (n == 0) return 0;
  k_qpgf_points<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(L, n, r_dev, out_dev, ret_dev, mode);
  return cudaGetLastError() == cudaSuccess ? 0 : BEM3_ERR_CUDA;
}

extern "C" int bem3_qpgf(const bem3_qpd2* qd, int n, const double* r, double* out, int* ret, int mode)
{
  if (n < 0 || (n > 0 && (!r || !out || !ret))) return BEM3_ERR_ARG;
  if (n == 0) return 0;
  double *dr = nullptr, *dout = nullptr;
  int* dret = nullptr;
  int rc = BEM3_ERR_CUDA;
  if (cudaMalloc(&dr, 3 * sizeof(double) * n) != cudaSuccess) goto done;
  if (cudaMalloc(&dout, 8 * sizeof(double) * n) != cudaSuccess) goto done;
  if (cudaMalloc(&dret, sizeof(int) * n) != cudaSuccess) goto done;
  if (cudaMemcpy(dr, r, 3 * sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess) goto done;
  rc = bem3_qpgf_dev(qd, n, dr, dout, dret, mode, nullptr);
  if (rc) goto done;
  if (cudaMemcpy(out, dout, 8 * sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess) { rc = BEM3_ERR_CUDA; goto done; }
  if (cudaMemcpy(ret, dret, sizeof(int) * n, cudaMemcpyDeviceToHost) != cudaSuccess) { rc = BEM3_ERR_CUDA; goto done; }
  rc = 0;
done:
  cudaFree(dr);
  cudaFree(dout);
  cudaFree(dret);
  return rc;
}

// ------------------------------------------------------------------------------------------
extern "C" int bem3_geo_stride(void) { return GEO_STRIDE; }

extern "C" int bem3_pack_geometry(const bem3_mesh* m, double* geo)
{
  if (!m || !geo || m->Ne <= 0 || !m->cr || !m->cw || !m->ren || !m->wen || !m->nv) return BEM3_ERR_ARG;
  for (int i = 0; i <= m->Ne; i++) {
    double* g = geo + (size_t)i * GEO_STRIDE;
    memset(g, 0, sizeof(double) * GEO_STRIDE);
    if (i == 0) continue;
    memcpy(g + GEO_CR, m->cr + (size_t)i * 12, 12 * sizeof(double));
    memcpy(g + GEO_CW, m->cw + (size_t)i * 9, 9 * sizeof(double));
    memcpy(g + GEO_REN, m->ren + (size_t)i * 12, 12 * sizeof(double));
    memcpy(g + GEO_WEN, m->wen + (size_t)i * 12, 12 * sizeof(double));
    int nv = m->nv[i];
    if (nv != 3 && nv != 4) return BEM3_ERR_ARG;
    g[GEO_NN] = (double)nv;
  }
  return 0;
}

extern "C" unsigned long long bem3_last_gh_pairs(void) { return t_last_stats.gh_pairs; }

extern "C" void bem3_set_profiling(int on) { t_profiling = on ? 1 : 0; }

extern "C" int bem3_last_stats(bem3_stats* out)
{
  if (!out) return BEM3_ERR_ARG;
  *out = t_last_stats;
  return 0;
}

// Rows per chunk so that the per-pair scratch stays near 384 MB.
static int default_rows_per_chunk(int ne)
{
  long long rows = (16LL << 20) / (ne > 0 ? ne : 1);
  if (rows < 4) rows = 4;
  if (rows > 4LL * ne) rows = 4LL * ne;
  return (int)rows;
}

// One domain's assembly in flight on a stream: its per-thread resources and counters.
struct DomainRun {
  DevRes* R = nullptr;
  AssembleStats S;
  bool profiling = false;
};

// Enqueues the assembly of one domain on `st` (device inputs and outputs) without waiting for it;
// `hook` (optional) sees every row chunk as its kernels are enqueued.
static int enqueue_domain(const double* geo_dev, int Ne, const int* sid_dev, int Ne_d, int did, int periodic,
                          const bem3_qpd2* qd, double kre, double kim, double* G_dev, double* H_dev, double* dG_dev,
                          double* dH_dev, double* dF_dev, cudaStream_t st, int rows, const ChunkHook* hook,
                          DomainRun& run)
{
  if (!geo_dev || !sid_dev || Ne <= 0 || Ne_d <= 0 || Ne_d > 2 * Ne || !G_dev || !H_dev) return BEM3_ERR_ARG;
  QPLattice L;
  memset(&L, 0, sizeof L);
  if (periodic) {
    int e = lattice_from(qd, &L);
    if (e) return e;
  }
  size_t need = bem3_scratch_bytes(Ne_d, rows);
  DevRes* R = nullptr;
  int e = ensure_scratch(need, &R);
  if (e) return e;
  AssembleArgs A;
  A.geo = geo_dev; A.sid = sid_dev; A.ne = Ne_d; A.did = did; A.periodic = periodic ? 1 : 0;
  A.kre = kre; A.kim = kim;
  A.G = G_dev; A.H = H_dev; A.dG = dG_dev; A.dH = dH_dev; A.dF = dF_dev;
  if (periodic) {
    if (!R->prop && cudaMalloc(&R->prop, sizeof(QPProp) * QP_PROP_CAP) != cudaSuccess) return BEM3_ERR_CUDA;
    if ((e = attach_prop_list(&L, R->prop, st))) return e;
  }
  if (cudaMemsetAsync(R->status, 0, sizeof(int), st) != cudaSuccess) return BEM3_ERR_CUDA;
  A.terms = nullptr;
  run.profiling = t_profiling != 0;
  if (run.profiling) {
    if (!R->terms && cudaMalloc(&R->terms, sizeof(unsigned long long)) != cudaSuccess) return BEM3_ERR_CUDA;
    A.terms = R->terms;
    cudaMemsetAsync(R->terms, 0, sizeof(unsigned long long), st);
  }
  memset(&run.S, 0, sizeof run.S);
  run.S.time_kernels = t_profiling;
  run.R = R;
  return bem3_assemble_run(A, &L, R->scratch, R->scratch_bytes, rows, R->status, st, &run.S, hook);
}

// Waits for `st` and returns the kernels' status; fills this thread's counters.
static int finish_domain(cudaStream_t st, const DomainRun& run)
{
  int hs = 0;
  unsigned long long terms = 0, gh = 0;
  if (cudaMemcpyAsync(&hs, run.R->status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return BEM3_ERR_CUDA;
  if (run.profiling && cudaMemcpyAsync(&terms, run.R->terms, sizeof terms, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return BEM3_ERR_CUDA;
  if (cudaMemcpyAsync(&gh, run.S.d_gh_total, sizeof gh, cudaMemcpyDeviceToHost, st) != cudaSuccess) return BEM3_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return BEM3_ERR_CUDA;
  memset(&t_last_stats, 0, sizeof t_last_stats);
  t_last_stats.gh_pairs = gh;
  t_last_stats.qpgf_terms = terms;
  t_last_stats.launches = run.S.launches;
  t_last_stats.reg_periodic_launches = run.S.reg_periodic_launches;
  t_last_stats.reg_periodic_ms = run.S.reg_periodic_ms;
  for (int i = 0; i < 4; i++) t_last_stats.class_ms[i] = run.S.class_ms[i];
  return hs;
}

extern "C" int bem3_assemble_domain_dev(const double* geo_dev, int Ne, const int* sid_dev, int Ne_d, int did, int periodic,
                                        const bem3_qpd2* qd, double kre, double kim, double* G_dev, double* H_dev,
                                        double* dG_dev, double* dH_dev, double* dF_dev, void* stream)
{
  cudaStream_t st = (cudaStream_t)stream;
  DomainRun run;
  int e = enqueue_domain(geo_dev, Ne, sid_dev, Ne_d, did, periodic, qd, kre, kim, G_dev, H_dev, dG_dev, dH_dev, dF_dev,
                         st, default_rows_per_chunk(Ne_d), nullptr, run);
  if (e) return e;
  return finish_domain(st, run);
}

namespace {
// Row chunks finished on the device, copied to the caller's host matrices on a copy stream as soon
// as each chunk's kernels have run: the transfer of chunk c overlaps the computation of the chunks
// after it.  (To page-locked host memory the copies are asynchronous; to pageable memory each copy
// call returns once done, while the GPU keeps computing the chunks already enqueued.)
struct RowCopies {
  size_t N = 0;
  std::vector<cudaEvent_t> ev;
  std::vector<int> r0, nr;
  bool failed = false;
  static void hook(void* user, int r0, int nr, cudaStream_t st)
  {
    RowCopies& c = *(RowCopies*)user;
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess || cudaEventRecord(e, st) != cudaSuccess) {
      c.failed = true;
      if (e) cudaEventDestroy(e);
      return;
    }
    c.ev.push_back(e);
    c.r0.push_back(r0);
    c.nr.push_back(nr);
  }
  ~RowCopies()
  {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
  }
};
}  // namespace

extern "C" int bem3_assemble_domain(const bem3_mesh* mesh, const int* sid, int Ne_d, int did, int periodic,
                                    const bem3_qpd2* qd, double kre, double kim, double* G, double* H, double* dG,
                                    double* dH, double* dF)
{
  if (!mesh || !sid || Ne_d <= 0 || !G || !H) return BEM3_ERR_ARG;
  for (int i = 0; i < Ne_d; i++)
    if (sid[i] == 0 || sid[i] > mesh->Ne || -sid[i] > mesh->Ne) return BEM3_ERR_ARG;
  const int Ne = mesh->Ne;
  std::vector<double> geo((size_t)(Ne + 1) * GEO_STRIDE);
  int e = bem3_pack_geometry(mesh, geo.data());
  if (e) return e;
  const size_t N = (size_t)4 * Ne_d;
  double *dgeo = nullptr, *dG_ = nullptr, *dH_ = nullptr, *ddG = nullptr, *ddH = nullptr, *ddF = nullptr;
  int* dsid = nullptr;
  cudaStream_t cs = nullptr;
  int rc = BEM3_ERR_CUDA;
  RowCopies rcp;
  rcp.N = N;
  const ChunkHook hook = {RowCopies::hook, &rcp};
  // about 8 row chunks per domain (at least 64 rows each), so that copies overlap the kernels
  int rows = (int)((N + 7) / 8);
  rows = rows < 64 ? 64 : rows;
  rows = rows > default_rows_per_chunk(Ne_d) ? default_rows_per_chunk(Ne_d) : rows;
  DomainRun run;
  if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) { cs = nullptr; goto done; }
  if (cudaMalloc(&dgeo, geo.size() * sizeof(double)) != cudaSuccess) goto done;
  if (cudaMalloc(&dsid, Ne_d * sizeof(int)) != cudaSuccess) goto done;
  if (cudaMalloc(&dG_, N * N * 16) != cudaSuccess) goto done;
  if (cudaMalloc(&dH_, N * N * 16) != cudaSuccess) goto done;
  if (dG && cudaMalloc(&ddG, 2 * N * N * 16) != cudaSuccess) goto done;
  if (dH && cudaMalloc(&ddH, 2 * N * N * 16) != cudaSuccess) goto done;
  if (dF && cudaMalloc(&ddF, 3 * N * sizeof(double)) != cudaSuccess) goto done;
  if (cudaMemcpy(dgeo, geo.data(), geo.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) goto done;
  if (cudaMemcpy(dsid, sid, Ne_d * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) goto done;
  rc = enqueue_domain(dgeo, Ne, dsid, Ne_d, did, periodic, qd, kre, kim, dG_, dH_, ddG, ddH, ddF, nullptr, rows, &hook,
                      run);
  if (rc) goto done;
  rc = BEM3_ERR_CUDA;
  if (rcp.failed) goto done;
  for (size_t c = 0; c < rcp.ev.size(); c++) {
    const size_t a = (size_t)rcp.r0[c], n = (size_t)rcp.nr[c];
    if (cudaStreamWaitEvent(cs, rcp.ev[c], 0) != cudaSuccess) goto done;
    if (cudaMemcpyAsync(G + 2 * a * N, dG_ + 2 * a * N, n * N * 16, cudaMemcpyDeviceToHost, cs) != cudaSuccess) goto done;
    if (cudaMemcpyAsync(H + 2 * a * N, dH_ + 2 * a * N, n * N * 16, cudaMemcpyDeviceToHost, cs) != cudaSuccess) goto done;
    if (dG && cudaMemcpyAsync(dG + 4 * a * N, ddG + 4 * a * N, 2 * n * N * 16, cudaMemcpyDeviceToHost, cs) != cudaSuccess)
      goto done;
    if (dH && cudaMemcpyAsync(dH + 4 * a * N, ddH + 4 * a * N, 2 * n * N * 16, cudaMemcpyDeviceToHost, cs) != cudaSuccess)
      goto done;
    if (dF && cudaMemcpyAsync(dF + 3 * a, ddF + 3 * a, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, cs) != cudaSuccess)
      goto done;
  }
  if (cudaStreamSynchronize(cs) != cudaSuccess) goto done;
  rc = finish_domain(nullptr, run);
done:
  if (cs) { cudaStreamSynchronize(cs); cudaStreamDestroy(cs); }
  cudaDeviceSynchronize();  // nothing of this call may still use the buffers freed below
  cudaFree(dgeo); cudaFree(dsid); cudaFree(dG_); cudaFree(dH_); cudaFree(ddG); cudaFree(ddH); cudaFree(ddF);
  return rc;
}

// Every domain of a problem through host pointers: the reference's create_cmatrix, the loop of
// create_cmatrix_domain over did = 0..MN (d3qd2_solve_bieq.c:155-163).  The domains' kernels run back
// to back on this thread's stream, the interior domains first: their matrices are large and quick to
// compute, and the open region's long lattice sums then hide their copies.  Every finished row chunk
// of every domain is copied on one copy stream while the later chunks compute, so only the open
// region's last chunk is copied after the kernels end.  All domains' device matrices are held at once.
extern "C" int bem3_assemble_domains(const bem3_mesh* mesh, int MN, const int* const* sid, const int* Ne_d, int periodic,
                                     const bem3_qpd2* qd, const double* kn, double* const* G, double* const* H,
                                     double* const* dG, double* const* dH, double* const* dF)
{
  if (!mesh || MN < 0 || !sid || !Ne_d || !kn || !G || !H) return BEM3_ERR_ARG;
  const int Ne = mesh->Ne, nd = MN + 1;
  for (int d = 0; d < nd; d++) {
    if (!sid[d] || Ne_d[d] <= 0 || !G[d] || !H[d]) return BEM3_ERR_ARG;
    for (int i = 0; i < Ne_d[d]; i++)
      if (sid[d][i] == 0 || sid[d][i] > Ne || -sid[d][i] > Ne) return BEM3_ERR_ARG;
  }
  auto opt = [](double* const* a, int d) { return a ? a[d] : nullptr; };
  std::vector<double> geo((size_t)(Ne + 1) * GEO_STRIDE);
  int e = bem3_pack_geometry(mesh, geo.data());
  if (e) return e;
  std::vector<int> order;  // interior domains first, the open region (did 0) last
  for (int d = 1; d < nd; d++) order.push_back(d);
  order.push_back(0);
  std::vector<size_t> N(nd);
  std::vector<int> rows(nd);
  size_t need = 0;
  for (int d = 0; d < nd; d++) {
    N[d] = (size_t)4 * Ne_d[d];
    int r = (int)((N[d] + 7) / 8);  // about 8 row chunks per domain, as bem3_assemble_domain
    r = r < 64 ? 64 : r;
    r = r > default_rows_per_chunk(Ne_d[d]) ? default_rows_per_chunk(Ne_d[d]) : r;
    rows[d] = r;
    const size_t b = bem3_scratch_bytes(Ne_d[d], r);
    need = b > need ? b : need;
  }
  double* dgeo = nullptr;
  int* dstat = nullptr;
  unsigned long long* dgh = nullptr;
  std::vector<int*> dsid(nd, nullptr);
  std::vector<double*> dG_(nd, nullptr), dH_(nd, nullptr), ddG(nd, nullptr), ddH(nd, nullptr), ddF(nd, nullptr);
  std::vector<RowCopies> rcp(nd);
  std::vector<DomainRun> run(nd);
  std::vector<int> hs(nd, 0);
  std::vector<unsigned long long> hgh(nd, 0);
  cudaStream_t cs = nullptr;
  const cudaStream_t st = cudaStreamPerThread;
  int rc = BEM3_ERR_CUDA;
  DevRes* R = nullptr;
  // the scratch at its largest before the first launch: no domain may reallocate it under another's kernels
  if ((rc = ensure_scratch(need, &R))) goto done;
  rc = BEM3_ERR_CUDA;
  if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) { cs = nullptr; goto done; }
  if (cudaMalloc(&dgeo, geo.size() * sizeof(double)) != cudaSuccess) goto done;
  if (cudaMalloc(&dstat, nd * sizeof(int)) != cudaSuccess) goto done;
  if (cudaMalloc(&dgh, nd * sizeof(unsigned long long)) != cudaSuccess) goto done;
  for (int d = 0; d < nd; d++) {
    const size_t n2 = N[d] * N[d] * 16;
    if (cudaMalloc(&dsid[d], Ne_d[d] * sizeof(int)) != cudaSuccess) goto done;
    if (cudaMalloc(&dG_[d], n2) != cudaSuccess || cudaMalloc(&dH_[d], n2) != cudaSuccess) goto done;
    if (opt(dG, d) && cudaMalloc(&ddG[d], 2 * n2) != cudaSuccess) goto done;
    if (opt(dH, d) && cudaMalloc(&ddH[d], 2 * n2) != cudaSuccess) goto done;
    if (opt(dF, d) && cudaMalloc(&ddF[d], 3 * N[d] * sizeof(double)) != cudaSuccess) goto done;
    if (cudaMemcpy(dsid[d], sid[d], Ne_d[d] * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) goto done;
    rcp[d].N = N[d];
  }
  if (cudaMemcpy(dgeo, geo.data(), geo.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) goto done;
  for (int d : order) {
    const ChunkHook hook = {RowCopies::hook, &rcp[d]};
    rc = enqueue_domain(dgeo, Ne, dsid[d], Ne_d[d], d, (periodic && d == 0) ? 1 : 0, qd, kn[2 * d], kn[2 * d + 1],
                        dG_[d], dH_[d], ddG[d], ddH[d], ddF[d], st, rows[d], &hook, run[d]);
    if (rc) goto done;
    rc = BEM3_ERR_CUDA;
    if (rcp[d].failed) goto done;
    // the domain's status word and near-singular count, kept before the next domain resets them
    if (cudaMemcpyAsync(dstat + d, run[d].R->status, sizeof(int), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(dgh + d, run[d].S.d_gh_total, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, st) !=
            cudaSuccess)
      goto done;
    const size_t n = N[d];
    for (size_t c = 0; c < rcp[d].ev.size(); c++) {
      const size_t a = (size_t)rcp[d].r0[c], m = (size_t)rcp[d].nr[c];
      if (cudaStreamWaitEvent(cs, rcp[d].ev[c], 0) != cudaSuccess) goto done;
      if (cudaMemcpyAsync(G[d] + 2 * a * n, dG_[d] + 2 * a * n, m * n * 16, cudaMemcpyDeviceToHost, cs) != cudaSuccess)
        goto done;
      if (cudaMemcpyAsync(H[d] + 2 * a * n, dH_[d] + 2 * a * n, m * n * 16, cudaMemcpyDeviceToHost, cs) != cudaSuccess)
        goto done;
      if (ddG[d] &&
          cudaMemcpyAsync(dG[d] + 4 * a * n, ddG[d] + 4 * a * n, 2 * m * n * 16, cudaMemcpyDeviceToHost, cs) != cudaSuccess)
        goto done;
      if (ddH[d] &&
          cudaMemcpyAsync(dH[d] + 4 * a * n, ddH[d] + 4 * a * n, 2 * m * n * 16, cudaMemcpyDeviceToHost, cs) != cudaSuccess)
        goto done;
      if (ddF[d] &&
          cudaMemcpyAsync(dF[d] + 3 * a, ddF[d] + 3 * a, 3 * m * sizeof(double), cudaMemcpyDeviceToHost, cs) != cudaSuccess)
        goto done;
    }
  }
  if (cudaStreamSynchronize(cs) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) goto done;
  if (cudaMemcpy(hs.data(), dstat, nd * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(hgh.data(), dgh, nd * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess)
    goto done;
  memset(&t_last_stats, 0, sizeof t_last_stats);
  for (int d = 0; d < nd; d++) {
    t_last_stats.gh_pairs += hgh[d];
    t_last_stats.launches += run[d].S.launches;
    t_last_stats.reg_periodic_launches += run[d].S.reg_periodic_launches;
  }
  rc = 0;
  for (int d = 0; d < nd; d++)
    if (hs[d]) { rc = hs[d]; break; }
done:
  if (cs) { cudaStreamSynchronize(cs); cudaStreamDestroy(cs); }
  cudaDeviceSynchronize();  // nothing of this call may still use the buffers freed below
  cudaFree(dgeo); cudaFree(dstat); cudaFree(dgh);
  for (int d = 0; d < nd; d++) {
    cudaFree(dsid[d]); cudaFree(dG_[d]); cudaFree(dH_[d]); cudaFree(ddG[d]); cudaFree(ddH[d]); cudaFree(ddF[d]);
  }
  return rc;
}

// ------------------------------------------------------------------------------------------
// FP64 peak probe: independent DFMA chains, 8 per thread, sized so the launch runs ~100 ms.
__global__ void __launch_bounds__(256) k_dfma_probe(double* out, int iters, double a, double b)
{
  double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-9, x2 = x0 + 2e-9, x3 = x0 + 3e-9;
  double x4 = x0 + 4e-9, x5 = x0 + 5e-9, x6 = x0 + 6e-9, x7 = x0 + 7e-9;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 16; u++) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 12345.6789) out[blockIdx.x] = s;  // keeps the chains live; never true in practice
}

extern "C" double bem3_fp64_peak_tflops(void)
{
  int dev = cur_dev(), sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double* d = nullptr;
  if (cudaMalloc(&d, sizeof(double) * sms * 8) != cudaSuccess) return -1.0;
  const int blocks = sms * 8, iters = 4096;
  k_dfma_probe<<<blocks, 256>>>(d, 16, 0.999999, 1e-7);  // warm-up
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  k_dfma_probe<<<blocks, 256>>>(d, iters, 0.999999, 1e-7);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  double flops = 2.0 * 8 * 16 * (double)iters * blocks * 256;
  return ms > 0 ? flops / (ms * 1e-3) / 1e12 : -1.0;
}

extern "C" const char* bem3_version(void) { return "bem3_emf_qd2_b200 0.1 (sm_100a, FP64)"; }

// ------------------------------------------------------------------------------------------
// Assembly without device allocation.
//
// Some callers cannot call cudaMalloc: a serving process that hands every byte of HBM out of
// its own pool under a fixed budget (allocations outside the pool are forbidden), or a
// pipeline that must not hit the implicit device-wide synchronisation cudaMalloc/cudaFree can
// cause.  For them the per-call scratch of the assembly (the chunk's F row-sum terms, the
// near-singular work list, the status word) lives in this file-scope device array instead of
// the cudaMalloc'd pool used by bem3_assemble_domain_dev.  Every GPU that loads the library
// holds the array (BEM3_NOALLOC_SCRATCH_BYTES) until the process exits.
#define BEM3_NOALLOC_SCRATCH_BYTES (32u << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[BEM3_NOALLOC_SCRATCH_BYTES];
static void* g_noalloc_addr[MAX_DEV];  // device address of g_noalloc_scratch, per device
static std::mutex g_noalloc_mu;

extern "C" int bem3_assemble_domain_dev_noalloc(const double* geo_dev, int Ne, const int* sid_dev, int Ne_d, int did,
                                                int periodic, const bem3_qpd2* qd, double kre, double kim,
                                                double* G_dev, double* H_dev, double* dG_dev, double* dH_dev,
                                                double* dF_dev, void* stream)
{
  if (!geo_dev || !sid_dev || Ne <= 0 || Ne_d <= 0 || Ne_d > 2 * Ne || !G_dev || !H_dev) return BEM3_ERR_ARG;
  QPLattice L;
  memset(&L, 0, sizeof L);
  if (periodic) {
    int e = lattice_from(qd, &L);
    if (e) return e;
  }
  // The array's device address: host code may not use the symbol itself (that is a host-side
  // stand-in, not a device pointer), so resolve it once per device with that device current.
  const int dev = cur_dev();
  if (dev < 0 || dev >= MAX_DEV) return BEM3_ERR_ARG;
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return BEM3_ERR_CUDA;
      g_noalloc_addr[dev] = p;
    }
    base = g_noalloc_addr[dev];
  }
  // [0, 256): status word; then the lattice's propagating orders; then the assembly scratch,
  // chunked to fit
  int* status = (int*)base;
  QPProp* prop = (QPProp*)((char*)base + 256);
  const size_t head = 256 + sizeof(QPProp) * QP_PROP_CAP;
  void* scratch = (char*)base + head;
  const size_t avail = BEM3_NOALLOC_SCRATCH_BYTES - head;
  int rows = default_rows_per_chunk(Ne_d);
  while (rows > 4 && bem3_scratch_bytes(Ne_d, rows) > avail) rows = rows / 2 > 4 ? rows / 2 : 4;
  if (bem3_scratch_bytes(Ne_d, rows) > avail) return BEM3_ERR_SCRATCH;  // domain too large for the array
  cudaStream_t st = (cudaStream_t)stream;
  AssembleArgs A;
  A.geo = geo_dev; A.sid = sid_dev; A.ne = Ne_d; A.did = did; A.periodic = periodic ? 1 : 0;
  A.kre = kre; A.kim = kim;
  A.G = G_dev; A.H = H_dev; A.dG = dG_dev; A.dH = dH_dev; A.dF = dF_dev;
  A.terms = nullptr;
  if (periodic) {
    int e2 = attach_prop_list(&L, prop, st);
    if (e2) return e2;
  }
  // the array keeps the previous call's contents: the status word must start at zero (the
  // run itself clears its row-sum slots and work-list counter before use)
  if (cudaMemsetAsync(status, 0, sizeof(int), st) != cudaSuccess) return BEM3_ERR_CUDA;
  AssembleStats S;
  memset(&S, 0, sizeof S);
  int e = bem3_assemble_run(A, &L, scratch, avail, rows, status, st, &S);
  if (e) return e;
  int hs = 0;
  unsigned long long gh = 0;
  if (cudaMemcpyAsync(&hs, status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return BEM3_ERR_CUDA;
  if (cudaMemcpyAsync(&gh, S.d_gh_total, sizeof gh, cudaMemcpyDeviceToHost, st) != cudaSuccess) return BEM3_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return BEM3_ERR_CUDA;
  // this thread's counters, as the allocating entry fills them (no term counter or kernel timing:
  // bem3_set_profiling does not apply to this entry point)
  memset(&t_last_stats, 0, sizeof t_last_stats);
  t_last_stats.gh_pairs = gh;
  t_last_stats.launches = S.launches;
  return hs;
}

// batch.cu -- the coefficient matrices of many domains of many instances (meshes, wavelengths,
// incidence angles, lattices) assembled together: one launch per pair class for the whole batch,
// fed from device work lists, replayed as one CUDA graph.
//
// The reference assembles one domain at a time (create_cmatrix_domain,
// d3qd2_src/d3qd2_solve_bieq.c:165-256), and so does bem3_assemble_domain_dev.  A batch of
// instances of uneven size run that way leaves the GPU partly idle at the end of every launch
// and launches (self, regular, near-singular, row sums) per domain.  Here:
//
//   descriptor table  BatchDomain[nd] in device memory: the domain's AssembleArgs, its own
//                     QPLattice (Bloch wave vector, Ewald split parameter veps0, propagating
//                     orders) and its scratch (per-pair F terms, near-singular work list,
//                     status word);
//   work segments     per pair class, the cumulative work of the domains of that class
//                     (rows, pairs or pair units); a launch maps its global work index to
//                     (domain, local index) by binary search over them;
//   persistent kernel k_batch_reg_periodic, the dominant class: every warp takes `grab` units of
//                     REGP_PAIRS pairs at a time from one device counter until the batch's
//                     regular periodic pairs are exhausted, whatever domain they belong to;
//   graph             reset, zero, then two branches -- periodic (self, regular, near-singular)
//                     and interior (self, regular, near-singular) -- joined before the row sums.
//
// Every pair is computed by the same device functions, in the same order of operations, as in
// the one-domain kernels (assemble.cu), so a domain's matrices do not depend on what else is in
// the batch.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "bem3_internal.h"

struct BatchDomain {
  AssembleArgs A;
  QPLattice L;         // periodic domains only; L.prop points into the batch's list buffer
  double3* Fp;         // [4 ne * ne] per-pair F terms (the domain is one chunk)
  double3* Fself;      // [4 ne]
  unsigned* gh_list;   // [gh_cap] near-singular pairs (pair index within the domain)
  unsigned* gh_count;  // entries appended (may exceed gh_cap: then status -900)
  unsigned gh_cap;
  int* status;         // the domain's status word (first error code)
};

// Cumulative work of the domains of one class: base[0] = 0, base[n] = total, domain dom[i]
// holds work [base[i], base[i + 1]).
struct BatchSeg {
  const long long* base;
  const int* dom;
  int n;
};

__device__ __forceinline__ int seg_find(const BatchSeg& S, long long x)
{
  int lo = 0, hi = S.n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (S.base[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Counters of a run: [0] regular periodic units taken.  Status words and work-list counters of
// every domain are cleared too.
__global__ void k_batch_reset(BatchDomain* D, int nd, unsigned long long* next)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) next[0] = 0ull;
  if (i < nd) {
    *D[i].gh_count = 0u;
    *D[i].status = 0;
  }
}

// Zeroes every output of domain blockIdx.y (rows of triangles with tn = 3 stay zero, as in the
// reference) and its self-pair F slots.
__global__ void k_batch_zero(const BatchDomain* __restrict__ D)
{
  const BatchDomain& d = D[blockIdx.y];
  const size_t N = (size_t)4 * d.A.ne;
  const size_t nn = N * N;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t i0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const double2 z = make_double2(0.0, 0.0);
  double2* G = (double2*)d.A.G;
  double2* H = (double2*)d.A.H;
  double2* dG = (double2*)d.A.dG;
  double2* dH = (double2*)d.A.dH;
  for (size_t i = i0; i < nn; i += stride) { G[i] = z; H[i] = z; }
  if (dG) for (size_t i = i0; i < 2 * nn; i += stride) dG[i] = z;
  if (dH) for (size_t i = i0; i < 2 * nn; i += stride) dH[i] = z;
  if (d.A.dF) for (size_t i = i0; i < 3 * N; i += stride) d.A.dF[i] = 0.0;
  for (size_t i = i0; i < N; i += stride) d.Fself[i] = make_double3(0.0, 0.0, 0.0);
}

__global__ void __launch_bounds__(SELF_THREADS, 2) k_batch_self_periodic(const BatchDomain* __restrict__ D, BatchSeg S)
{
  __shared__ double red[SELF_THREADS / 32][24];
  __shared__ int serr[SELF_THREADS / 32];
  const long long g = blockIdx.x;
  const int i = seg_find(S, g);
  const BatchDomain& d = D[S.dom[i]];
  self_periodic_row(d.A, d.L, (int)(g - S.base[i]), d.Fself, d.status, red, serr);
}

__global__ void __launch_bounds__(SI_THREADS) k_batch_self_interior(const BatchDomain* __restrict__ D, BatchSeg S)
{
  __shared__ double red[SI_NW * SELF_NV];
  __shared__ double res[4][SELF_NV];
  const long long g = blockIdx.x;
  const int i = seg_find(S, g);
  const BatchDomain& d = D[S.dom[i]];
  self_interior_row(d.A, (int)(g - S.base[i]), d.Fself, red, res);
}

// Persistent: gridDim.x CTAs of 8 warps; a warp takes `grab` units (REGP_PAIRS pairs each) per
// atomic on next[0] and runs them, until the units of all periodic domains are taken.
__global__ void __launch_bounds__(256, REGP_MIN_BLOCKS) k_batch_reg_periodic(const BatchDomain* __restrict__ D, BatchSeg S,
                                                                             int grab, unsigned long long* next)
{
  extern __shared__ __align__(16) unsigned char regp_smem[];  // REGP_SMEM_BYTES
  RegWarp(*sw)[REGP_PAIRS] = reinterpret_cast<RegWarp(*)[REGP_PAIRS]>(regp_smem);
  AccP(*sacc)[256] = reinterpret_cast<AccP(*)[256]>(regp_smem + sizeof(RegWarp) * 8 * REGP_PAIRS);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const long long total = S.base[S.n];
  for (;;) {
    unsigned long long u0 = 0ull;
    if (lane == 0) u0 = atomicAdd(next, (unsigned long long)grab);
    u0 = __shfl_sync(0xffffffffu, u0, 0);
    if ((long long)u0 >= total) break;
    const long long uend = min(total, (long long)u0 + grab);
    for (long long u = (long long)u0; u < uend; u++) {
      const int i = seg_find(S, u);
      const BatchDomain& d = D[S.dom[i]];
      const long long np = 4LL * d.A.ne * d.A.ne;
      reg_periodic_unit(d.A, d.L, 0, np, (u - S.base[i]) * REGP_PAIRS, d.Fp, d.gh_list, d.gh_count, d.gh_cap, d.status,
                        sw[wib], sacc, lane);
    }
  }
}

__global__ void __launch_bounds__(128) k_batch_reg_interior(const BatchDomain* __restrict__ D, BatchSeg S)
{
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= S.base[S.n]) return;
  const int i = seg_find(S, g);
  const BatchDomain& d = D[S.dom[i]];
  reg_interior_pair(d.A, 0, g - S.base[i], d.Fp, d.gh_list, d.gh_count, d.gh_cap, d.status);
}

// Near-singular pairs: the domains' lists in turn, CTAs (periodic) or warps (interior) striding
// over each.
__global__ void __launch_bounds__(256, 2) k_batch_gh_periodic(const BatchDomain* __restrict__ D, const int* __restrict__ dom, int n)
{
  __shared__ double red[8][19];
  __shared__ int serr[8];
  for (int i = 0; i < n; i++) {
    const BatchDomain& d = D[dom[i]];
    const unsigned cnt = min(*d.gh_count, d.gh_cap);
    for (unsigned it = blockIdx.x; it < cnt; it += gridDim.x) gh_periodic_pair(d.A, d.L, 0, d.gh_list[it], d.Fp, d.status, red, serr);
  }
}

__global__ void __launch_bounds__(256) k_batch_gh_interior(const BatchDomain* __restrict__ D, const int* __restrict__ dom, int n)
{
  const int lane = threadIdx.x & 31;
  const unsigned wglob = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = 0; i < n; i++) {
    const BatchDomain& d = D[dom[i]];
    const unsigned cnt = min(*d.gh_count, d.gh_cap);
    for (unsigned it = wglob; it < cnt; it += nw) gh_interior_pair(d.A, 0, d.gh_list[it], d.Fp, lane);
  }
}

// Row sums of every domain: one warp per row.
__global__ void k_batch_rowsum(const BatchDomain* __restrict__ D, BatchSeg S)
{
  const long long g = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (g >= S.base[S.n]) return;
  const int i = seg_find(S, g);
  const BatchDomain& d = D[S.dom[i]];
  const int row = (int)(g - S.base[i]);
  rowsum_row(d.A, row, d.Fp + (size_t)row * d.A.ne, d.Fself, threadIdx.x & 31);
}

// ------------------------------------------------------------------------------------------
// Host side
struct bem3_batch_s {
  int dev = 0;
  int nd = 0;
  void* mem = nullptr;  // one device allocation: table, segments, lists, scratch
  size_t bytes = 0;
  BatchDomain* dD = nullptr;
  int* dstatus = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int launches = 0;
};

namespace {

struct SegHost {
  std::vector<long long> base{0};
  std::vector<int> dom;
  void add(int d, long long work)
  {
    if (work <= 0) return;
    dom.push_back(d);
    base.push_back(base.back() + work);
  }
  long long total() const { return base.back(); }
  int n() const { return (int)dom.size(); }
};

// Bump allocator over the batch's single device allocation (256-byte aligned pieces).
struct Layout {
  size_t off = 0;
  size_t take(size_t bytes)
  {
    const size_t at = off;
    off += (bytes + 255) & ~(size_t)255;
    return at;
  }
};

void batch_free(bem3_batch b)
{
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->mem) cudaFree(b->mem);
  delete b;
}

}  // namespace

extern "C" size_t bem3_batch_scratch_bytes(const bem3_batch_domain* doms, int n)
{
  if (!doms || n <= 0) return 0;
  size_t total = 0;
  for (int i = 0; i < n; i++) {
    const size_t ne = (size_t)(doms[i].Ne_d > 0 ? doms[i].Ne_d : 0);
    const size_t np = 4 * ne * ne;
    total += ((np * sizeof(double3) + 255) & ~(size_t)255) + ((4 * ne * sizeof(double3) + 255) & ~(size_t)255) +
             (((np / 8 + 4096) * sizeof(unsigned) + 255) & ~(size_t)255) + 256;
    if (doms[i].periodic) total += (sizeof(QPProp) * QP_PROP_CAP + 255) & ~(size_t)255;
  }
  // table, status words and segments
  total += (((sizeof(BatchDomain) + 2 * sizeof(long long) + 5 * sizeof(int)) * (size_t)n + 8 * sizeof(long long)) * 5 +
            255) & ~(size_t)255;
  return total + 4096;
}

extern "C" int bem3_batch_create(const bem3_batch_domain* doms, int n, const bem3_batch_tuning* tune, bem3_batch* out)
{
  if (!out) return BEM3_ERR_ARG;
  *out = nullptr;
  if (!doms || n <= 0 || n > 65535) return BEM3_ERR_ARG;  // the zero kernel's grid has one row per domain
  bem3_batch_tuning T = {8, REGP_MIN_BLOCKS, 4};
  if (tune) T = *tune;
  if (T.grab_units < 1 || T.grab_units > 4096 || T.regp_blocks_per_sm < 1 || T.regp_blocks_per_sm > REGP_MIN_BLOCKS ||
      T.gh_blocks_per_sm < 1 || T.gh_blocks_per_sm > 16)
    return BEM3_ERR_ARG;
  for (int i = 0; i < n; i++) {
    const bem3_batch_domain& d = doms[i];
    if (!d.geo || !d.sid || d.Ne <= 0 || d.Ne_d <= 0 || d.Ne_d > 2 * d.Ne || !d.G || !d.H) return BEM3_ERR_ARG;
    // pair indices of a domain's work list are 32-bit
    if (4.0 * d.Ne_d * (double)d.Ne_d >= 4294967295.0) return BEM3_ERR_ARG;
  }
  if (ensure_tables() != 0) return BEM3_ERR_CUDA;
  if (cudaFuncSetAttribute(k_batch_reg_periodic, cudaFuncAttributePreferredSharedMemoryCarveout,
                           (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess ||
      cudaFuncSetAttribute(k_batch_reg_periodic, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)REGP_SMEM_BYTES) !=
          cudaSuccess)
    return BEM3_ERR_CUDA;

  bem3_batch b = new bem3_batch_s;
  cudaGetDevice(&b->dev);
  b->nd = n;

  // host descriptors, lattices and propagating orders
  std::vector<BatchDomain> hD((size_t)n);
  std::vector<std::vector<QPProp>> props((size_t)n);
  SegHost selfP, selfI, regP, regI, rows;
  std::vector<int> pdom, idom;
  for (int i = 0; i < n; i++) {
    const bem3_batch_domain& d = doms[i];
    BatchDomain& B = hD[(size_t)i];
    memset(&B, 0, sizeof B);
    AssembleArgs& A = B.A;
    A.geo = d.geo; A.sid = d.sid; A.ne = d.Ne_d; A.did = d.did; A.periodic = d.periodic ? 1 : 0;
    A.kre = d.kre; A.kim = d.kim;
    A.G = d.G; A.H = d.H; A.dG = d.dG; A.dH = d.dH; A.dF = d.dF;
    A.terms = nullptr;
    const long long ne = d.Ne_d;
    if (A.periodic) {
      int e = lattice_from(&d.qd, &B.L);
      if (e) { batch_free(b); return e; }
      props[(size_t)i].resize(QP_PROP_CAP);
      const int np = qp_prop_list(B.L, props[(size_t)i].data(), QP_PROP_CAP);
      if (np < 0) { batch_free(b); return BEM3_ERR_LATTICE; }
      props[(size_t)i].resize((size_t)np);
      B.L.nprop = np;
      selfP.add(i, 4 * ne);
      regP.add(i, (4 * ne * ne + REGP_PAIRS - 1) / REGP_PAIRS);
      pdom.push_back(i);
    } else {
      selfI.add(i, 4 * ne);
      regI.add(i, 4 * ne * ne);
      idom.push_back(i);
    }
    rows.add(i, 4 * ne);
  }

  // one allocation
  Layout Lay;
  const size_t oD = Lay.take(sizeof(BatchDomain) * (size_t)n);
  const size_t oStatus = Lay.take(sizeof(int) * (size_t)n);
  const size_t oNext = Lay.take(sizeof(unsigned long long) * 4);
  SegHost* segs[5] = {&selfP, &selfI, &regP, &regI, &rows};
  size_t oBase[5], oDom[5];
  for (int k = 0; k < 5; k++) {
    oBase[k] = Lay.take(sizeof(long long) * segs[k]->base.size());
    oDom[k] = Lay.take(sizeof(int) * (segs[k]->dom.size() + 1));
  }
  const size_t oPdom = Lay.take(sizeof(int) * (pdom.size() + 1));
  const size_t oIdom = Lay.take(sizeof(int) * (idom.size() + 1));
  std::vector<size_t> oFp((size_t)n), oFself((size_t)n), oList((size_t)n), oCount((size_t)n), oProp((size_t)n, 0);
  for (int i = 0; i < n; i++) {
    const size_t ne = (size_t)doms[i].Ne_d, np = 4 * ne * ne;
    oFp[(size_t)i] = Lay.take(np * sizeof(double3));
    oFself[(size_t)i] = Lay.take(4 * ne * sizeof(double3));
    hD[(size_t)i].gh_cap = (unsigned)(np / 8 + 4096);
    oList[(size_t)i] = Lay.take((size_t)hD[(size_t)i].gh_cap * sizeof(unsigned));
    oCount[(size_t)i] = Lay.take(sizeof(unsigned));
    if (doms[i].periodic && !props[(size_t)i].empty()) oProp[(size_t)i] = Lay.take(sizeof(QPProp) * props[(size_t)i].size());
  }
  b->bytes = Lay.off;
  if (cudaMalloc(&b->mem, b->bytes) != cudaSuccess) { b->mem = nullptr; batch_free(b); return BEM3_ERR_CUDA; }
  char* m = (char*)b->mem;
  b->dD = (BatchDomain*)(m + oD);
  b->dstatus = (int*)(m + oStatus);
  unsigned long long* next = (unsigned long long*)(m + oNext);
  for (int i = 0; i < n; i++) {
    BatchDomain& B = hD[(size_t)i];
    B.Fp = (double3*)(m + oFp[(size_t)i]);
    B.Fself = (double3*)(m + oFself[(size_t)i]);
    B.gh_list = (unsigned*)(m + oList[(size_t)i]);
    B.gh_count = (unsigned*)(m + oCount[(size_t)i]);
    B.status = b->dstatus + i;
    if (doms[i].periodic) B.L.prop = props[(size_t)i].empty() ? nullptr : (QPProp*)(m + oProp[(size_t)i]);
  }
  // uploads (synchronous: creation is outside the timed path)
  bool ok = cudaMemcpy(b->dD, hD.data(), sizeof(BatchDomain) * (size_t)n, cudaMemcpyHostToDevice) == cudaSuccess;
  BatchSeg S[5];
  for (int k = 0; k < 5 && ok; k++) {
    ok = cudaMemcpy(m + oBase[k], segs[k]->base.data(), sizeof(long long) * segs[k]->base.size(), cudaMemcpyHostToDevice) ==
         cudaSuccess;
    if (ok && !segs[k]->dom.empty())
      ok = cudaMemcpy(m + oDom[k], segs[k]->dom.data(), sizeof(int) * segs[k]->dom.size(), cudaMemcpyHostToDevice) ==
           cudaSuccess;
    S[k].base = (const long long*)(m + oBase[k]);
    S[k].dom = (const int*)(m + oDom[k]);
    S[k].n = segs[k]->n();
  }
  if (ok && !pdom.empty())
    ok = cudaMemcpy(m + oPdom, pdom.data(), sizeof(int) * pdom.size(), cudaMemcpyHostToDevice) == cudaSuccess;
  if (ok && !idom.empty())
    ok = cudaMemcpy(m + oIdom, idom.data(), sizeof(int) * idom.size(), cudaMemcpyHostToDevice) == cudaSuccess;
  for (int i = 0; i < n && ok; i++)
    if (oProp[(size_t)i])
      ok = cudaMemcpy(m + oProp[(size_t)i], props[(size_t)i].data(), sizeof(QPProp) * props[(size_t)i].size(),
                      cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) { batch_free(b); return BEM3_ERR_CUDA; }

  // the launch sequence, captured once
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->dev);
  cudaStream_t s0 = nullptr, s1 = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  if (cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s1, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&join, cudaEventDisableTiming) != cudaSuccess) {
    ok = false;
  }
  int launches = 0;
  if (ok && cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) ok = false;
  if (ok) {
    k_batch_reset<<<(n + 255) / 256, 256, 0, s0>>>(b->dD, n, next);
    k_batch_zero<<<dim3(2 * sms, (unsigned)n), 256, 0, s0>>>(b->dD);
    launches += 2;
    cudaEventRecord(fork, s0);
    cudaStreamWaitEvent(s1, fork, 0);
    // periodic branch
    if (selfP.total() > 0) { k_batch_self_periodic<<<(unsigned)selfP.total(), SELF_THREADS, 0, s0>>>(b->dD, S[0]); launches++; }
    if (regP.total() > 0) {
      const long long want = (regP.total() * 32 + 255) / 256;  // CTAs that would give every warp one unit
      const unsigned ctas = (unsigned)std::min<long long>((long long)sms * T.regp_blocks_per_sm, std::max(want, 1LL));
      k_batch_reg_periodic<<<ctas, 256, REGP_SMEM_BYTES, s0>>>(b->dD, S[2], T.grab_units, next);
      k_batch_gh_periodic<<<(unsigned)(sms * T.gh_blocks_per_sm), 256, 0, s0>>>(b->dD, (const int*)(m + oPdom),
                                                                             (int)pdom.size());
      launches += 2;
    }
    // interior branch
    if (selfI.total() > 0) { k_batch_self_interior<<<(unsigned)selfI.total(), SI_THREADS, 0, s1>>>(b->dD, S[1]); launches++; }
    if (regI.total() > 0) {
      k_batch_reg_interior<<<(unsigned)((regI.total() + 127) / 128), 128, 0, s1>>>(b->dD, S[3]);
      k_batch_gh_interior<<<(unsigned)(sms * T.gh_blocks_per_sm), 256, 0, s1>>>(b->dD, (const int*)(m + oIdom),
                                                                             (int)idom.size());
      launches += 2;
    }
    cudaEventRecord(join, s1);
    cudaStreamWaitEvent(s0, join, 0);
    k_batch_rowsum<<<(unsigned)((rows.total() * 32 + 255) / 256), 256, 0, s0>>>(b->dD, S[4]);
    launches++;
    if (cudaGetLastError() != cudaSuccess) ok = false;
    cudaGraph_t g = nullptr;
    if (cudaStreamEndCapture(s0, &g) != cudaSuccess || !g) ok = false;
    b->graph = g;
    if (ok && cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) { b->exec = nullptr; ok = false; }
  }
  if (fork) cudaEventDestroy(fork);
  if (join) cudaEventDestroy(join);
  if (s0) cudaStreamDestroy(s0);
  if (s1) cudaStreamDestroy(s1);
  if (!ok) { batch_free(b); return BEM3_ERR_CUDA; }
  b->launches = launches;
  *out = b;
  return 0;
}

extern "C" int bem3_batch_run(bem3_batch b, void* stream)
{
  if (!b || !b->exec) return BEM3_ERR_ARG;
  return cudaGraphLaunch(b->exec, (cudaStream_t)stream) == cudaSuccess ? 0 : BEM3_ERR_CUDA;
}

extern "C" int bem3_batch_wait(bem3_batch b, void* stream, int* per_domain)
{
  if (!b) return BEM3_ERR_ARG;
  std::vector<int> st((size_t)b->nd, 0);
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(st.data(), b->dstatus, sizeof(int) * (size_t)b->nd, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return BEM3_ERR_CUDA;
  int first = 0;
  for (int i = 0; i < b->nd; i++) {
    if (per_domain) per_domain[i] = st[(size_t)i];
    if (!first && st[(size_t)i]) first = st[(size_t)i];
  }
  return first;
}

extern "C" int bem3_batch_info(bem3_batch b, int* launches, size_t* device_bytes)
{
  if (!b) return BEM3_ERR_ARG;
  if (launches) *launches = b->launches;
  if (device_bytes) *device_bytes = b->bytes;
  return 0;
}

extern "C" int bem3_batch_destroy(bem3_batch b)
{
  if (!b) return BEM3_ERR_ARG;
  int cur = 0;
  cudaGetDevice(&cur);
  const int dev = b->dev;
  if (cur != dev) cudaSetDevice(dev);
  batch_free(b);
  if (cur != dev) cudaSetDevice(cur);
  return 0;
}

/*
 * bem3_qd2_b200.h -- C ABI of the B200 (sm_100a) implementation of bem3_emf_qd2's
 * boundary-integral hot path: the quasi-periodic Green's function (QPGF) and the
 * element-quadrature assembly of the coefficient matrices.
 *
 * Every entry point takes plain pointers and sizes; no CUDA or framework types appear in the
 * signatures (a stream is passed as `void *`, NULL = the default stream).  Return values are
 * 0 on success or one of the negative BEM3_ERR_* codes below.  Arrays follow the reference's
 * in-memory conventions (1-based element ids with slot 0 unused, row-major complex doubles
 * stored as interleaved re/im pairs) so that a caller holding a DQD2 (d3qd2_src/d3qd2_elem.h:49-60)
 * can pass its arrays after flattening.
 */
#ifndef BEM3_QD2_B200_H_
#define BEM3_QD2_B200_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BEM3_OK 0
#define BEM3_ERR_ARG -1      /* invalid argument */
#define BEM3_ERR_CUDA -2     /* CUDA failure (device memory, launch, copy) */
#define BEM3_ERR_SCRATCH -3  /* scratch smaller than required */
#define BEM3_ERR_LATTICE -4  /* degenerate lattice (det[d1 d2] == 0) or more than 2048 propagating orders */
#define BEM3_ERR_SOLVE -5    /* singular system */
/* Kernel status codes (returned as is): -11..-14 and -21..-24 are the QPGF failures of
 * d3hm_qpgf_d2_v1 (qgf2_src/d3_qpgf_d2.h:112-123); -900 near-singular work-list overflow. */

/* Quasi-periodic data, same field order and meaning as QPD2 (qgf2_src/d3_qpgf_d2.h:32-36). */
typedef struct {
  double k;        /* wave number of the open (periodic) region */
  double vk[3];    /* incident wave vector; vk[0], vk[1] give the Bloch phase */
  double vd1[2];   /* lattice vector d1 (z = 0) */
  double vd2[2];   /* lattice vector d2 (z = 0) */
} bem3_qpd2;

/* Surface mesh in the reference's element-constant form (BOUD, d3qd2_src/d3qd2_elem.h:22-47),
 * flattened, element ids 1..Ne with slot 0 unused:
 *   cr  [(Ne+1)][3][4]  bilinear/linear map coefficients  (init_elem_const, d3qd2_setup.c:1139)
 *   cw  [(Ne+1)][3][3]  normal-vector (Jacobian) coefficients
 *   ren [(Ne+1)][4][3]  collocation node positions        (init_boundary_data, d3qd2_setup.c:1309)
 *   wen [(Ne+1)][4][3]  normal vectors at the nodes
 *   nv  [(Ne+1)]        vertices per element: 3 (triangle) or 4 (bilinear quad)            */
typedef struct {
  int Ne;
  const double *cr;
  const double *cw;
  const double *ren;
  const double *wen;
  const int *nv;
} bem3_mesh;

/* ---------------------------------------------------------------------------------------------
 * Green's function.
 * Replaces d3hm_qpgf_d2_v1 (qgf2_src/d3_qpgf_d2.h:112, d3_qpgf_d2.c:124) for n points at once.
 * r: [n][3] host array; out: [n][4] complex (qG, dqG/dx, dqG/dy, dqG/dz); ret: [n] codes as the
 * reference (> 0 number of lattice terms, < 0 failure).  mode 0: the reference's v1 stop rules;
 * mode 1: stop only when the rules of both d3hm_qpgf_d2_qG and d3hm_qpgf_d2_dqG
 * (d3_qpgf_d2.h:125-126) are met.  Runs on the current CUDA device. */
int bem3_qpgf(const bem3_qpd2 *qd, int n, const double *r, double *out, int *ret, int mode);

/* Same with device-resident r / out / ret (pointers into device memory) on `stream`. */
int bem3_qpgf_dev(const bem3_qpd2 *qd, int n, const double *r_dev, double *out_dev, int *ret_dev, int mode,
                  void *stream);

/* ---------------------------------------------------------------------------------------------
 * Coefficient matrices of one domain.
 * Replaces create_cmatrix_domain (d3qd2_src/d3qd2_solve_bieq.c:165-256): for every collocation
 * node (t, tn) of the domain and every source element s it evaluates what the reference gets
 * from q0_dcoef_bd_node_t2_cc (did 0, periodic; d3qd2_elem.c:830) or dcoef_bd_node_t2 (interior
 * domains; d3qd2_elem.c:515) with PREC_DEF_BE = 2, and writes the matrices that the reference
 * writes to its tmpG/tmpH/tmpdG/tmpdH/tmpdF files, in the same layout (N = 4 Ne_d):
 *   G, H   [N][N] complex,  dG, dH [2N][N] complex,  dF [N][3] double.
 * sid: [Ne_d] signed element ids of the domain (sb[did].sid[1..Ne_d]).  periodic: 1 when
 * did == 0 and the problem is periodic (bd.ps == 1).  kre/kim: domain wave number kn[did].
 * dG, dH or dF may be NULL to skip them.  Host pointers; the call is synchronous. */
int bem3_assemble_domain(const bem3_mesh *mesh, const int *sid, int Ne_d, int did, int periodic,
                         const bem3_qpd2 *qd, double kre, double kim, double *G, double *H, double *dG,
                         double *dH, double *dF);

/* Every domain of a problem in one call: the reference's create_cmatrix, the loop of
 * create_cmatrix_domain over did = 0..MN (d3qd2_solve_bieq.c:155-163).  Domain d has sid[d]
 * (Ne_d[d] signed ids), wave number kn[2 d] + i kn[2 d + 1] and host outputs G[d], H[d], dG[d],
 * dH[d], dF[d] as bem3_assemble_domain's (dG, dH, dF: NULL arrays, or NULL entries, skip them);
 * domain 0 is the quasi-periodic open region when periodic != 0.  The domains' kernels run back to
 * back, the interior domains first, and the row chunks of every domain are copied to the host
 * while later chunks compute; the device holds every domain's matrices at once.  Host pointers;
 * synchronous.  Returns the first failing domain's status.  Fills bem3_last_gh_pairs and the
 * gh_pairs / launches of bem3_last_stats, summed over the domains (no term counter or kernel times). */
int bem3_assemble_domains(const bem3_mesh *mesh, int MN, const int *const *sid, const int *Ne_d, int periodic,
                          const bem3_qpd2 *qd, const double *kn, double *const *G, double *const *H,
                          double *const *dG, double *const *dH, double *const *dF);

/* Device-resident variant.  geo_dev: packed geometry from bem3_pack_geometry (uploaded by the
 * caller); sid_dev: [Ne_d] ints; outputs in device memory.  The library allocates its scratch
 * with cudaMalloc on a calling thread's first use and keeps it, per host thread and device, for
 * that thread's later calls; calls from different threads may run concurrently. */
int bem3_assemble_domain_dev(const double *geo_dev, int Ne, const int *sid_dev, int Ne_d, int did, int periodic,
                             const bem3_qpd2 *qd, double kre, double kim, double *G_dev, double *H_dev,
                             double *dG_dev, double *dH_dev, double *dF_dev, void *stream);

/* Same as bem3_assemble_domain_dev, for callers that cannot allocate device memory (a serving
 * process whose pool owns all of HBM under a fixed budget, a pipeline that must avoid the implicit
 * synchronisation of cudaMalloc/cudaFree).  No counterpart in the reference, whose assembly runs
 * on the host.  The call allocates nothing: its scratch is a 32 MiB file-scope device array that
 * every GPU loading the library holds until exit, and regular pairs are processed in row chunks
 * that fit it.  A domain whose four rows of one element do not fit (about 170,000 elements per
 * domain) is rejected with BEM3_ERR_SCRATCH.  All calls share the array: calls that overlap on the
 * GPU (other streams, other threads on the same device) race and must be serialised by the caller.
 * The first call on a device resolves the array's device address (cudaGetSymbolAddress); make that
 * first call before any stream capture.  The address is kept for the life of the process, so the
 * library must not be used on a device after cudaDeviceReset.  Synchronous on `stream`.  Fills
 * bem3_last_gh_pairs and the gh_pairs / launches of bem3_last_stats; bem3_set_profiling (term
 * counter, kernel timing) does not apply to it. */
int bem3_assemble_domain_dev_noalloc(const double *geo_dev, int Ne, const int *sid_dev, int Ne_d, int did, int periodic,
                                     const bem3_qpd2 *qd, double kre, double kim, double *G_dev, double *H_dev,
                                     double *dG_dev, double *dH_dev, double *dF_dev, void *stream);

/* Packs a bem3_mesh into the device geometry layout: (Ne+1) * bem3_geo_stride() doubles. */
int bem3_geo_stride(void);
int bem3_pack_geometry(const bem3_mesh *mesh, double *geo);

/* The same geometry records computed on the device from the mesh itself: the element constants of
 * init_elem_const (d3qd2_setup.c:1139-1186) and the collocation nodes and normals of
 * init_boundary_data (d3qd2_setup.c:1309-1349), bit-identical to bem3_pack_geometry of the
 * host set-up's constants.  rn_dev: [Nn + 1][3] node coordinates (row 0 unused, after any rotation
 * and translation; read_mesh_data's dqd2.bd.rn); ed_dev: [Ne + 1][4] vertex node ids (1..Nn; the
 * fourth 0 for a triangle; dqd2.bd.ed); geo_dev: [(Ne + 1) * bem3_geo_stride()] out.  Device
 * pointers; synchronous on `stream`.  BEM3_ERR_ARG if an element names a node outside 1..Nn. */
int bem3_mesh_pack_dev(int Ne, int Nn, const double *rn_dev, const int *ed_dev, double *geo_dev, void *stream);

/* Counters of the last assembly on this thread: near-singular (64x64 rule) pairs. */
unsigned long long bem3_last_gh_pairs(void);

/* Profiling counters of the last assembly on this thread.  Filled only after
 * bem3_set_profiling(1) (which adds a per-warp term counter and CUDA-event timing of every
 * kernel, synchronising after each); otherwise only gh_pairs and launches are set. */
typedef struct {
  unsigned long long gh_pairs;     /* pairs recomputed with the 64x64 near-singular rule */
  unsigned long long qpgf_terms;   /* lattice-sum terms summed by the regular periodic kernel */
  int launches;                    /* kernels launched by the call */
  int reg_periodic_launches;       /* launches of the regular periodic kernel */
  double reg_periodic_ms;          /* their summed duration (CUDA events) */
  double class_ms[4];              /* kernel time by pair class: self (t == s), regular,
                                      near-singular (64x64 rule), row sums of F */
} bem3_stats;
void bem3_set_profiling(int on);
int bem3_last_stats(bem3_stats *out);

/* Measures the FP64 FMA throughput of the current device (TFLOP/s), the denominator of the
 * FP64 roofline.  Runs a ~100 ms kernel. */
double bem3_fp64_peak_tflops(void);

/* One incident plane wave after set-up: the derived data IpwD and the translation of Ipw
 * (d3qd2_src/ipw.h:19-37, filled by setup_ipw ipw.c:121-145).  Fields at x:
 * E = E0 e exp(i ki k.(x - f)), H = E0 h exp(i ki k.(x - f)), k = (sin_t cos_p, sin_t sin_p, cos_t). */
typedef struct {
  double E0, ki;
  double cos_t, sin_t, cos_p, sin_p;
  double f[3];
  double e[6]; /* ex, ey, ez complex */
  double h[6]; /* hx, hy, hz complex */
} bem3_wave;

/* ---------------------------------------------------------------------------------------------
 * Boundary-integral equation solve.
 * Replaces solve_bieq (d3qd2_src/d3qd2_solve_bieq.c:36-84) on arrays: assembles every domain
 * (create_cmatrix, :156-256), builds the global system of 8 NN unknowns (create_matrix_csr_dac,
 * :284-421), solves it with a dense device LU (in place of PARDISO, d3qd2_mkl_solver.c:18),
 * stores U, dU (tmatrix_bd_store, :456-544), computes E, H on the boundary (q1_solve_eh_bv,
 * :931-1030) and dE, dH (solve_deh_bv, :662-791).  Everything runs on the current CUDA device;
 * the dense system needs (8 NN)^2 * 16 bytes of device memory.
 * Layouts follow DQD2 (d3qd2_src/d3qd2_elem.h:13-60), flattened, element ids 1..Ne (slot 0 unused). */
typedef struct {
  int MN;                   /* media 1..MN; domain 0 is the open region */
  int Ne, NN;               /* elements; element nodes (3 per triangle, 4 per quad) */
  int ps;                   /* 1: quasi-periodic open region */
  bem3_mesh mesh;
  const int *md, *sd;       /* [(Ne+1)] main / sub domain of each element */
  const int *eni;           /* [(Ne+1)][4] element node ids (-1 for the 4th node of triangles) */
  const int *Ne_d;          /* [MN+1] elements per domain */
  const int *const *sid;    /* [MN+1] -> [Ne_d] signed element ids (sb[d].sid[1..Ne_d]) */
  const double *kn;         /* [MN+1] complex wave numbers */
  bem3_qpd2 qd;
  double lambda0;
  const double *Ui, *dUi;   /* [(Ne+1)][4][4] complex incident potential and normal derivative */
  const double *dEiz, *dEie;/* [(Ne+1)][4][3] complex tangential derivatives of the incident E */
  int Nn;                   /* mesh nodes (ids 1..Nn) */
  const double *rn;         /* [(Nn+1)][3] node coordinates (BOUD.rn) */
  const int *ed;            /* [(Ne+1)][4] element vertex node ids (BOUD.ed; ed[e][3] = 0 for triangles) */
  int nwaves;
  const bem3_wave *waves;   /* [nwaves] incident plane waves (MIPW) */
} bem3_problem;

/* Boundary values of one domain, same layout as SUBD (d3qd2_elem.h:13-20), slot 0 unused:
 * U, dU [(Ne_d+1)][4][4], E, dE, H, dH [(Ne_d+1)][4][3] complex.  NULL members are skipped. */
typedef struct {
  double *U, *dU, *E, *dE, *H, *dH;
} bem3_bv;

int bem3_solve_bieq_arrays(const bem3_problem *P, bem3_bv *out /* [MN+1] */);

/* ---------------------------------------------------------------------------------------------
 * Device-resident problem.  A context holds one problem's geometry, media, incident waves and
 * boundary values on the current CUDA device, so that a solve and any number of field
 * evaluations share one upload.  Contexts are independent of each other: each call's work goes
 * to the calling host thread's default stream, so contexts driven from different threads run
 * concurrently on the GPU.  One context must not be used from two threads at once. */
typedef struct bem3_ctx_s *bem3_ctx;

/* Copies the problem to the device.  The caller's arrays may be freed afterwards. */
int bem3_ctx_create(const bem3_problem *P, bem3_ctx *out);
void bem3_ctx_destroy(bem3_ctx c);

/* solve_bieq on the device; the boundary values stay in the context. */
int bem3_ctx_solve(bem3_ctx c);

/* How bem3_ctx_solve solves the system of the potentials.  0 (default): eliminate dU through the
 * Dirichlet-to-Neumann maps of one class of domains and solve the remaining 4 NN equations when the
 * domains allow it (every element separates the two classes), else method 1.  1: the reference's
 * system of 8 NN unknowns (create_tmatrix_csr, d3qd2_solve_bieq.c:258-282) as one dense LU.
 * 2: the reduced system only (BEM3_ERR_ARG when not applicable).  No counterpart in the reference,
 * which always solves the 8 NN system with PARDISO. */
int bem3_ctx_set_solver(bem3_ctx c, int method);

/* A solve leaves the matrices and factorisations on the device (bem3_ctx_device_bytes says how
 * much).  A new incident field with the same wavelength and direction (another polarisation, a
 * different amplitude or phase; the matrices depend on the wavelength and on k||) then needs
 * only its right-hand sides: bem3_ctx_set_incident replaces the incident data of bem3_problem
 * (same layouts), bem3_ctx_resolve recomputes the boundary values.  bem3_ctx_release frees the
 * matrices and factorisations and keeps the boundary values.  No counterpart in the reference,
 * which assembles and factorises for every run. */
/* Device time (ms, CUDA events) of the last bem3_ctx_solve's phases, the three that the reference's
 * solve_bieq reports (d3qd2_solve_bieq.c:48-83): ms[0] the coefficient matrices of every domain
 * (create_cmatrix), ms[1] the factorisations (every domain's compacted G and the system of the
 * potentials: create_tmatrix_csr + solve_tmatrix_csr's factorisation), ms[2] the right-hand sides,
 * the boundary values, E, H and dE, dH on the boundary (tmatrix_bd_store, q1_solve_eh_bv,
 * solve_deh_bv).  After bem3_ctx_resolve, ms[0] = ms[1] = 0 and ms[2] is the re-solve. */
int bem3_ctx_phase_times(bem3_ctx c, double *ms /* [3] */);

int bem3_ctx_set_incident(bem3_ctx c, int nwaves, const bem3_wave *waves, const double *Ui, const double *dUi,
                          const double *dEiz, const double *dEie);
int bem3_ctx_resolve(bem3_ctx c);
int bem3_ctx_release(bem3_ctx c);
size_t bem3_ctx_device_bytes(bem3_ctx c);

/* Boundary values to host arrays (layout of bem3_bv), or from host arrays (for example the
 * values a reference result file holds, read by dat_read d3qd2_setup.c:300). */
int bem3_ctx_get_bv(bem3_ctx c, bem3_bv *out /* [MN+1] */);
int bem3_ctx_set_bv(bem3_ctx c, const bem3_bv *bv /* [MN+1] */);

/* Domain of each point (q0_domain_id / domain_id, d3qd2_setup.c:157-238): did[n]. */
int bem3_ctx_domain_id(bem3_ctx c, int n, const double *r, int *did);

/* Electromagnetic field at n points (EH_s / EH_t / EH_i, d3qd2_src/d3qd2_field.c:203-300).
 * r: [n][3]; E, H: [n][3] complex; did: [n] domain of each point (may be NULL).
 * type 0: nodal 4-point rules, type 1: 9-point (quads) / 7-point (triangles) rules, types 2 and
 * 3: 12 x 12 and 64 x 64 Gauss-Legendre rules (three sub-quads on triangles), for points near the
 * boundary.  (The reference's type 4, double-exponential integration, is not provided.)
 * total 0: scattered / internal field (EH_s); 1: plus the incident field in the open region
 * (EH_t); 2: the incident field alone, at every point (EH_i).
 * Points outside every domain get did = -1 and zero fields (except with total 2). */
int bem3_ctx_field(bem3_ctx c, int n, const double *r, int type, int total, double *E, double *H, int *did);

/* Modified electromagnetic potentials at n points (mEMP_s / mEMP_t / mEMP_i,
 * d3qd2_src/d3qd2_field.c:10-87): U [n][4] complex = (vector potential x, y, z, scalar
 * potential).  type, total and did as bem3_ctx_field; total 1 adds the incident electric field
 * to the vector potential in the open region, total 2 gives U = (E_inc, 0). */
int bem3_ctx_potential(bem3_ctx c, int n, const double *r, int type, int total, double *U, int *did);

/* Electromagnetic field at n points from the derivatives of the potentials (EH_mEMP_s / _t / _i,
 * d3qd2_src/d3qd2_field.c:89-201): E = A - grad phi, H = lambda0 / (2 pi i) curl A, with the
 * coefficient-gradient rules (q0_dcoef_rt_grad / dcoef_rt_grad, d3qd2_elem.c:316, 650) and the
 * Green's function's second derivatives (d3hm_qpgf_d2_v2).  More accurate than bem3_ctx_field in
 * the far field, slower.  type and total as bem3_ctx_field.  A point too close to the boundary
 * for these rules (|dF/dr| > 10, CBD_CDF) gets zero fields and did = -did (-99 in the open
 * region), as the reference returns. */
int bem3_ctx_field_memp(bem3_ctx c, int n, const double *r, int type, int total, double *E, double *H, int *did);

/* Electromagnetic field on the boundary of the open region at n points on its elements (EH_s_bd /
 * EH_t_bd, d3qd2_src/d3qd2_field.c:299-385): t[i] the element's 1-based position in domain did's list
 * (the reference's t), zeta_eta [n][2] the point's parameters on it (main-domain side).  Every other
 * element by the rule `type` (0-3), the element itself by the singular rule around the point, divided
 * by 1 + F.  total 0: scattered field (EH_s_bd), 1: plus the incident field (EH_t_bd).  E, H: [n][3]
 * complex.  did must be 0 and the problem quasi-periodic (BEM3_ERR_ARG otherwise: interior domains
 * would need the free-space rule of coef_bd at arbitrary points, not provided). */
int bem3_ctx_field_bd(bem3_ctx c, int did, int n, const int *t, const double *zeta_eta, int type, int total,
                      double *E, double *H);

/* Radiation force F[3] and torque N[3] about rc[3] on the objects, from the Maxwell stress tensor
 * of the total field on the open region's boundary (force_FN, d3qd2_src/d3qd2_force.c:10-54).
 * type 0: element nodes (plus the centroid on triangles); type 1: 9-point (quads) / 7-point
 * (triangles) rules, with the boundary field EH_t_bd (d3qd2_field.c:343-385) at the points.
 * Points other than nodes need the quasi-periodic open region (BEM3_ERR_ARG otherwise). */
int bem3_ctx_force(bem3_ctx c, const double *rc, int type, double *F, double *N);

/* ---------------------------------------------------------------------------------------------
 * Batched assembly: the coefficient matrices of many domains of many instances (each its own
 * mesh, wavelength, incidence and lattice) in one launch per pair class, replayed as one CUDA
 * graph.  No counterpart in the reference (one domain per create_cmatrix_domain call,
 * d3qd2_solve_bieq.c:165); each domain's results are those of bem3_assemble_domain_dev on the
 * same inputs.
 *
 * One entry per (instance, domain), all pointers device memory on the current device:
 * geo/Ne and sid/Ne_d/did/periodic as bem3_assemble_domain_dev; qd the instance's lattice and
 * Bloch wave vector (periodic domains); outputs G, H, dG, dH, dF in the reference layout (dG, dH,
 * dF may be NULL). */
typedef struct {
  const double *geo;
  int Ne;
  const int *sid;
  int Ne_d;
  int did;
  int periodic;
  bem3_qpd2 qd;
  double kre, kim;
  double *G, *H, *dG, *dH, *dF;
} bem3_batch_domain;

/* Launch shape of a batch (bem3_batch_create with NULL takes {8, 2, 4}).
 *   grab_units          work units (2 regular periodic pairs each) a warp takes per atomic
 *                       on the batch's work counter, 1..4096
 *   regp_blocks_per_sm  resident CTAs per SM of the persistent regular periodic kernel, 1..2
 *   gh_blocks_per_sm    CTAs per SM of the near-singular kernels, 1..16 */
typedef struct {
  int grab_units;
  int regp_blocks_per_sm;
  int gh_blocks_per_sm;
} bem3_batch_tuning;

typedef struct bem3_batch_s *bem3_batch;

/* Device bytes bem3_batch_create allocates for these domains (an upper bound): per domain
 * 96 Ne_d^2 bytes of per-pair F terms, its near-singular work list and self-pair terms, plus the
 * descriptor table.  The outputs are the caller's. */
size_t bem3_batch_scratch_bytes(const bem3_batch_domain *doms, int n);

/* Builds a batch over n <= 65535 domains: descriptor table, work segments, scratch (one
 * cudaMalloc) and the captured graph.  Synchronous.  Must not be called during a stream capture. */
int bem3_batch_create(const bem3_batch_domain *doms, int n, const bem3_batch_tuning *tune, bem3_batch *out);

/* Enqueues one assembly of every domain of the batch on `stream` (one graph launch).  Runs of
 * the same batch must not overlap: they share its scratch. */
int bem3_batch_run(bem3_batch b, void *stream);

/* Waits for `stream` and returns 0 or the first failing domain's status code (kernel codes as
 * for bem3_assemble_domain_dev); per_domain (optional, n entries) receives every domain's. */
int bem3_batch_wait(bem3_batch b, void *stream, int *per_domain);

/* Kernels one run launches, and the device bytes the batch holds. */
int bem3_batch_info(bem3_batch b, int *launches, size_t *device_bytes);

int bem3_batch_destroy(bem3_batch b);

/* A solve in two halves, so that the coefficient matrices of several contexts can be assembled
 * together by one batch: bem3_ctx_prepare allocates the context's matrices (what bem3_ctx_solve
 * holds) and describes every domain in doms[MN+1] (device pointers into the context; give them to
 * bem3_batch_create, with other contexts' entries); once a batch run has filled them (after its
 * bem3_batch_wait), bem3_ctx_solve_prepared does the rest of bem3_ctx_solve (factorisations,
 * right-hand sides, boundary values and fields).  No counterpart in the reference (one solve_bieq per problem). */
int bem3_ctx_prepare(bem3_ctx c, bem3_batch_domain *doms /* [MN+1] */);
int bem3_ctx_solve_prepared(bem3_ctx c);

/* Gauss-Legendre nodes and weights on [-1, 1] (the reference's gauleg, com_src/gauleg.c:3). */
void bem3_gauss_legendre(int n, double *x, double *w);

/* Library version string. */
const char *bem3_version(void);

#ifdef __cplusplus
}
#endif

#endif /* BEM3_QD2_B200_H_ */

// bem3_internal.h -- declarations shared by the CUDA translation units of the library.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "qpgf.cuh"

#include "bem3_qd2_b200.h"

struct AssembleArgs {
  const double* geo;  // [(Ne+1) * GEO_STRIDE] element geometry, id 0 unused
  const int* sid;     // [ne] signed element ids of the domain (0-based positions)
  int ne;             // elements seen by the domain
  int did;            // domain id (0 = open, periodic region)
  int periodic;       // 1: quasi-periodic Green's function (did 0 with ps == 1)
  double kre, kim;    // wave number of the domain
  double* G;          // [N][N] complex (N = 4 ne)
  double* H;          // [N][N] complex
  double* dG;         // [2N][N] complex
  double* dH;         // [2N][N] complex
  double* dF;         // [N][3]
  unsigned long long* terms;  // optional device counter: lattice-sum terms of the regular periodic pairs
};

struct AssembleStats {
  unsigned long long gh_pairs;   // near-singular pairs recomputed with the 64x64 rule
  int launches;                  // kernels launched
  int time_kernels;              // in: 1 = time every kernel with CUDA events (synchronising)
  double reg_periodic_ms;        // out: summed duration of k_reg_periodic launches
  int reg_periodic_launches;     // out: number of k_reg_periodic launches
  double class_ms[4];            // out: self, regular, near-singular, row-sum kernels (any domain)
  unsigned long long* d_gh_total;  // out: device counter of near-singular pairs (read it after the stream syncs)
};

// Called after each row chunk's kernels are enqueued on `st` (rows r0 .. r0 + nr - 1 are final
// once they have run): lets a caller copy finished rows out while later chunks compute.
struct ChunkHook {
  void (*fn)(void* user, int r0, int nr, cudaStream_t st);
  void* user;
};

size_t bem3_scratch_bytes(int ne, int rows);
int bem3_assemble_run(const AssembleArgs& A, const QPLattice* L, void* scratch, size_t scratch_bytes, int rows_per_chunk,
                      int* d_status, cudaStream_t st, AssembleStats* stats, const ChunkHook* hook = nullptr);
void bem3_launch_self_interior(const AssembleArgs& A, double3* Fself, int* d_status, cudaStream_t st);

// bem3_solve.h -- device-side views used by the solve stage (solve.cu).
#pragma once

#define BEM3_MAXDOM 16

// All pointers are device memory.  Per-domain arrays are indexed by domain id 0..MN.
struct SolveDev {
  int MN;                       // number of media (domains 1..MN), domain 0 = open region
  int NN;                       // total element nodes (3 per triangle, 4 per quad)
  int Ne;                       // elements
  const double* geo;            // packed geometry [(Ne+1) * GEO_STRIDE]
  const int* md;                // [(Ne+1)] main domain of each element
  const int* sd;                // [(Ne+1)] sub domain of each element
  const int* eni;               // [(Ne+1)][4] element node ids (-1 for the 4th node of triangles)
  const double* kn;             // [(MN+1)] complex wave numbers
  const double* Ui;             // [(Ne+1)][4][4] complex incident potential at the nodes
  const double* dUi;            // [(Ne+1)][4][4] complex normal derivative
  const double* dEiz;           // [(Ne+1)][4][3] complex dE_inc / dt_zeta at the nodes
  const double* dEie;           // [(Ne+1)][4][3] complex dE_inc / dt_eta
  double ch_re, ch_im;          // lambda0 / (2 pi i)
  int ne[BEM3_MAXDOM];          // elements per domain
  const int* sid_h[BEM3_MAXDOM];     // [ne] signed ids per domain
  const double* G[BEM3_MAXDOM];      // [4ne][4ne] complex
  const double* H[BEM3_MAXDOM];
  const double* dG[BEM3_MAXDOM];     // [8ne][4ne] complex
  const double* dH[BEM3_MAXDOM];
  const double* dF[BEM3_MAXDOM];     // [4ne][3]
  double* U[BEM3_MAXDOM];            // [(ne+1)][4][4] complex (slot 0 unused)
  double* dU[BEM3_MAXDOM];
  double* E[BEM3_MAXDOM];            // [(ne+1)][4][3] complex
  double* H_[BEM3_MAXDOM];
  double* dE[BEM3_MAXDOM];
  double* dH_[BEM3_MAXDOM];
  const int* pos0;              // [(Ne+1)] position (0-based) of each element in sb[0].sid, -1 if absent
};

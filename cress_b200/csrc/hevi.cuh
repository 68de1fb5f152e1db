// HE-VI substep kernel interface (internal to the library).
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"
#include "status.h"

namespace cress {

// 1-D base-state / metric columns of a horizontally uniform base state,
// stored as col[field*(nk+1) + k], k = 1..nk.
enum ColField {
  C_JCB = 0, C_JCB8U, C_JCB8V, C_JCB8W, C_RBR, C_PTBR, C_RST, C_RST8U, C_RST8V, C_RST8W, C_RCSQ,
  C_PBR, C_QVBR, C_UBR, C_VBR, C_ZPH8S, C_NFIELDS
};

struct HeviArgs {
  Grid g;
  const float* u_old; const float* v_old; const float* w_old; const float* p_old;
  float* u_new; float* v_new; float* w_new; float* p_new;
  const float* ufrc; const float* vfrc; const float* wfrc; const float* pfrc;
  const float* col;       // 1-D base columns
  const float* thom_rr;   // [k] sub-diagonal a_k of the w system (float, as formed by stepwi)
  const double* thom_aa;  // [k] 1/(b_k - a_k c'_{k-1})
  const double* thom_cp;  // [k] c'_k
  float dts, dxiv, dyiv, dziv, divch, divcv, weicoe, dtdzw, dtw, g05, g05n;
  int divopt, buyopt, sthopt, bbc;
};

// tile: 0 = 32x4 (default), 1 = 32x2, 2 = 32x8, 3 = 16x8
int launch_hevi_substep(const HeviArgs& a, int tile, cudaStream_t st);

}  // namespace cress

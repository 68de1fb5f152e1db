// Open (radiation) west and east boundaries for sm_100a (internal): the
// boundary columns of the small step, of the leapfrog scalars, and the
// phase speeds that drive both.  See openbc.cu.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace cress {

// Variables with phase speeds (the C-ABI field order).
enum RadVar { RAD_U = 0, RAD_V, RAD_W, RAD_P, RAD_PT, RAD_QV, RAD_N = RAD_QV + 9 };

// Phase speed c(var, side, j, k) at cp[((var*2 + side)*(nk+1) + k)*(nj+2) + j];
// side 0 west, 1 east (ucpx(1:nj,1:nk,1:2) and its siblings).
__host__ __device__ inline long long rad_at(const Grid& g, int var, int side, int j, int k) {
  return (((long long)var * 2 + side) * (g.nk + 1) + k) * (g.nj + 2) + j;
}
inline size_t rad_floats(const Grid& g) { return (size_t)RAD_N * 2 * (g.nk + 1) * (g.nj + 2); }

// One small step's boundary columns: new values from the substep's old
// arrays (the same pointers the HE-VI launch reads and writes).
struct RbcSmallArgs {
  Grid g;
  const float* cp;
  const float* col;   // column fields, col[f*(nk+1) + k]
  const float *u_old, *v_old, *w_old, *p_old;
  float *u_new, *v_new, *w_new, *p_new;
  int sthopt, bbc;
};

// The leapfrog scalars' boundary columns (theta' and the moist species).
struct RbcLeapArgs {
  Grid g;
  const float* cp;
  int n;
  const float* s[10];    // present level
  const float* sp[10];   // past level
  float* sf[10];         // future level (boundary columns written)
  int var[10];           // RadVar
  int kind[10];          // 0 theta', 1 qv and 2 mixing ratios (clipped at zero), 3 number concentrations
};

// The phase speeds of every variable from the present (filtered), past and
// future levels.
struct PhaseArgs {
  Grid g;
  float* cp;
  int n;
  const float* s[14];
  const float* sp[14];
  const float* sf[14];
  int var[14];
  int obc;               // 4, 5 or 7
  float gwave, dxiv, dtb, dts;
};

int launch_rbc_small(const RbcSmallArgs& a, cudaStream_t st);
int launch_rbc_leapfrog(const RbcLeapArgs& a, cudaStream_t st);
int launch_phase(const PhaseArgs& a, cudaStream_t st);

}  // namespace cress

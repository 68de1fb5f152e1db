// TKE equation of the 1.5-order closure (tubopt=2): forcing and leapfrog
// step in one kernel (tke.cu) (internal).
#pragma once
#include <cuda.h>
#include "common.cuh"
#include "forcing.cuh"

namespace cress {

// TMA box rows of the TKE kernel's staged fields for a 32 x kScalarTY tile:
// the TKE at t and t-dt with two rows of y halo (from j0-2), u and w on
// the tile rows (from j0), v from one row south to two rows north and the
// eddy viscosity with one row each side (both from j0-1).
struct TkeRows {
  static constexpr int s = kScalarTY + 4, u = kScalarTY, v = kScalarTY + 3, w = kScalarTY, r = kScalarTY + 2;
};

struct TkeArgs {
  Grid g;
  const float* lvl;                      // level table (nk+1) x kLevelStride for this dtb
  // per point from k_turb_visc: 1/Pr*rkv/jcb, N^2 at w level k, shear
  // production and dissipation
  const float *rks, *nsq, *shr, *dsp;
  float* tkef;                           // TKE at t+dt (output)
  float dxiv, dyiv, dziv, smhcoe, smvcoe;
  int smtopt, vspopt, sthopt, ksp0, advopt;
  int vsp_tke;                           // vspvar(10:10) == 'o'
  int* err;                              // device error word (a bounded wait gave up)
};

struct TkeMaps {
  CUtensorMap s, sp, u, v, w, rkv;       // TKE at t, t-dt; present winds; eddy viscosity
};

int launch_tke(const TkeArgs& a, const TkeMaps& maps, cudaStream_t st);

}  // namespace cress

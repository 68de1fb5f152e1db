// Shared definitions for the cress_b200 CUDA kernels.
//
// Device layout of one 3-D field: the reference's explicit-shape array
//   real :: a(0:ni+1, 0:nj+1, 1:nk)
// stored x-fastest with the x pitch padded to a multiple of 32 floats so
// that every row starts on a 128-byte boundary:
//   a(i,j,k) -> base[i + px*(j + py*(k-1))],  px >= ni+2, py = nj+2.
// Host <-> device syncs are pitched copies, so the host mirror keeps the
// reference's exact layout.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cress {

struct Grid {
  int ni, nj, nk;   // reference dims (ni = nx+3, nj = ny+3, nk = nz+3)
  int px, py;       // x pitch (floats) and y extent of one plane
  long long plane;  // px*py
  int openx;        // 1: open (radiation) west and east boundaries, 0: periodic x
  int slaby;        // 1: one y slab of a decomposed domain (y ghosts come from the neighbours), 0: periodic y
  __host__ __device__ inline long long at(int i, int j, int k) const {
    return (long long)i + (long long)px * ((long long)j + (long long)py * (long long)(k - 1));
  }
  __host__ __device__ inline long long count() const { return plane * (long long)nk; }
};

inline Grid make_grid(int ni, int nj, int nk) {
  Grid g;
  g.ni = ni; g.nj = nj; g.nk = nk;
  g.px = ((ni + 2) + 31) / 32 * 32;
  g.py = nj + 2;
  g.plane = (long long)g.px * g.py;
  g.openx = 0;
  g.slaby = 0;
  return g;
}

// Columns of the pointwise large-step work (microphysics, filters,
// saturation adjustment): the interior, and with open x also the boundary
// columns i = 1 and ni-1, which the reference's loops over i = 1..ni-1
// update (with periodic x those are ghosts the wrap refills).
__host__ __device__ inline int col_lo(const Grid& g) { return g.openx ? 1 : 2; }
__host__ __device__ inline int col_hi(const Grid& g) { return g.openx ? g.ni - 1 : g.ni - 2; }
__host__ __device__ inline int ncols(const Grid& g) { return col_hi(g) - col_lo(g) + 1; }

// Staggering of a field for the periodic wrap of SrcOrig/bcycle.f90: which
// interior index feeds which ghost.  S = scalar/w point, U = x face, V = y face.
enum Stag { STAG_S = 0, STAG_U = 1, STAG_V = 2 };

// Periodic images of interior point (i,j) under s_bcycle (bcycle.f90:159-225)
// as the steppers call it (stepuv.f90:390-393, stepwi.f90:517, steppi.f90:293):
//   scalar/w/p : (2,1,ni-2,ni-1, 2,1,nj-2,nj-1)
//   u          : (3,1,ni-2,ni,   2,1,nj-2,nj-1)
//   v          : (2,1,ni-2,ni-1, 3,1,nj-2,nj)
// Writes `val` at (i,j,k) and at every ghost position the wrap copies it to.
__device__ __forceinline__ void store_periodic(float* __restrict__ f, const Grid& g, int stag,
                                               int i, int j, int k, float val) {
  int xs[2], ys[2];
  int nx = 1, ny = 1;
  xs[0] = i; ys[0] = j;
  if (g.openx) {   // open x: no x ghosts (the radiation boundaries set i = 1, ni-1 / ni)
  } else if (i == g.ni - 2) {
    xs[nx++] = 1;
  } else if (stag == STAG_U ? (i == 3) : (i == 2)) {
    xs[nx++] = (stag == STAG_U) ? g.ni : g.ni - 1;
  }
  if (g.slaby) {   // a y slab: the neighbours' rows fill the y ghosts (slab.h)
  } else if (j == g.nj - 2) {
    ys[ny++] = 1;
  } else if (stag == STAG_V ? (j == 3) : (j == 2)) {
    ys[ny++] = (stag == STAG_V) ? g.nj : g.nj - 1;
  }
  for (int b = 0; b < ny; ++b)
    for (int a = 0; a < nx; ++a) f[g.at(xs[a], ys[b], k)] = val;
}

}  // namespace cress

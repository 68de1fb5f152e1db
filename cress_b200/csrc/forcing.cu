// Large-step kernels for sm_100a: the Asselin filter and the periodic
// ghost planes (the forcing is in force.cu, the moist scalars in
// scalars.cu).
#include <cuda_runtime.h>
#include "common.cuh"
#include "forcing.cuh"
#include "hevi.cuh"

namespace cress {
namespace {

// s_timeflt, SrcOrig/timeflt.f90:335-404 on the interior (ghosts are
// refilled by k_halo afterwards); with open x also on the boundary
// columns (u: i = 1 and ni, the rest i = 1 and ni-1), which the
// reference's loops over i = 1..ni-1 (u: 1..ni) include.
__global__ void __launch_bounds__(256) k_timeflt(const FilterArgs a) {
  const Grid g = a.g;
  const int i = col_lo(g) + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > col_hi(g) + 1 || j > g.nj - 1 || k > g.nk) return;
  const long long id = g.at(i, j, k);
  const float fc = a.filcoe, m1fc2 = 1.f - 2.f * a.filcoe;
  const bool si = i <= col_hi(g), sj = j <= g.nj - 2;
  const bool lk = k <= g.nk - 1;
  // every load before the first store (the compiler cannot tell the fields
  // apart), so a thread's loads are all in flight at once
  const bool du = lk && sj, dv = lk && si, ds = lk && si && sj, dw = si && sj, dt = ds && a.tke;
  float u0 = 0.f, u1 = 0.f, u2 = 0.f, v0 = 0.f, v1 = 0.f, v2 = 0.f, p0 = 0.f, p1 = 0.f, p2 = 0.f;
  float t0 = 0.f, t1 = 0.f, t2 = 0.f, w0 = 0.f, w1 = 0.f, w2 = 0.f, e0 = 0.f, e1 = 0.f, e2 = 0.f;
  if (du) { u0 = a.u[id]; u1 = a.uf[id]; u2 = a.up[id]; }
  if (dv) { v0 = a.v[id]; v1 = a.vf[id]; v2 = a.vp[id]; }
  if (ds) { p0 = a.pp[id]; p1 = a.ppf[id]; p2 = a.ppp[id]; t0 = a.ptp[id]; t1 = a.ptpf[id]; t2 = a.ptpp[id]; }
  if (dt) { e0 = a.tke[id]; e1 = a.tkef[id]; e2 = a.tkep[id]; }
  if (dw) { w0 = a.w[id]; w1 = a.wf[id]; w2 = a.wp[id]; }
  if (du) a.u[id] = m1fc2 * u0 + fc * (u1 + u2);
  if (dv) a.v[id] = m1fc2 * v0 + fc * (v1 + v2);
  if (ds) {
    a.pp[id] = m1fc2 * p0 + fc * (p1 + p2);
    a.ptp[id] = m1fc2 * t0 + fc * (t1 + t2);
  }
  if (dt)   // timeflt.f90:866-884: twice the coefficient for the TKE
    a.tke[id] = (1.f - 4.f * a.filcoe) * e0 + (2.f * a.filcoe) * (e1 + e2);
  if (dw) a.w[id] = m1fc2 * w0 + fc * (w1 + w2);
}

// Both periodic ghost layers (bcycle.f90:159-225 with the stepper and the
// shift2nd.f90:4274-4300 arguments): ghost index g maps to the interior
// point 2 + ((g-2) mod P), P = n-3, for i in {0,1,ni-1,ni} (scalars) or
// {0,1,ni,ni+1} (u), and likewise in y.
__device__ __forceinline__ int wrap(int x, int n) {
  const int P = n - 3;
  int r = (x - 2) % P;
  if (r < 0) r += P;
  return 2 + r;
}

// Threads run over the frame of possible ghost points only: the rows
// j in {0, 1, nj-1, nj, nj+1} (all i) and the columns i in {0, 1, ni-1, ni,
// ni+1} (j = 2..nj-2), one level per blockIdx.y and one field per
// blockIdx.z (every copy its own thread, so none waits behind another's
// store); the field's staggering decides which points are ghosts.
// Sources are never ghosts, so the order of the copies does not matter.
__global__ void __launch_bounds__(128) k_halo(const HaloArgs a) {
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = 1 + blockIdx.y;
  const int rows = 5 * (ni + 2);
  int i, j;
  if (b < rows) {
    const int r = b / (ni + 2);
    i = b % (ni + 2);
    j = r < 2 ? r : nj - 1 + (r - 2);
  } else {
    const int c = b - rows;
    if (c >= 5 * (nj - 3)) return;
    const int q = c / (nj - 3);
    j = 2 + c % (nj - 3);
    i = q < 2 ? q : ni - 1 + (q - 2);
  }
  const int n = blockIdx.z;
  const int st = a.stag[n];
  // open x: only the y wrap (over every column, boundary columns included)
  const bool gx = !g.openx && ((st == STAG_U) ? (i <= 1 || i >= ni) : (i <= 1 || (i >= ni - 1 && i <= ni)));
  // a y slab: the neighbours' rows fill the y ghosts (slab.h)
  const bool gy = !g.slaby && ((st == STAG_V) ? (j <= 1 || j >= nj) : (j <= 1 || (j >= nj - 1 && j <= nj)));
  const bool inx = (st == STAG_U) ? (i <= ni + 1) : (i <= ni);
  const bool iny = (st == STAG_V) ? (j <= nj + 1) : (j <= nj);
  if (!(gx || gy) || !inx || !iny) return;
  const int si = gx ? wrap(i, ni) : i;
  const int sj = gy ? wrap(j, nj) : j;
  float* f = a.f[n];
  f[g.at(i, j, k)] = f[g.at(si, sj, k)];
}

// One thread per element, 4 elements per thread along x; rows in blockIdx.y
// (grid-strided).
__global__ void __launch_bounds__(256) k_repitch(const float* __restrict__ src, int sp, float* __restrict__ dst,
                                                 int dp, int w, long long rows) {
  for (long long r = blockIdx.y; r < rows; r += gridDim.y) {
    const float* s = src + r * sp;
    float* d = dst + r * dp;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < w; x += gridDim.x * blockDim.x) d[x] = __ldg(s + x);
  }
}

}  // namespace

int launch_repitch(const float* src, int src_pitch, float* dst, int dst_pitch, int w, long long rows,
                   cudaStream_t st) {
  dim3 gr((w + 255) / 256, (unsigned)(rows < 65535 ? rows : 65535), 1);
  k_repitch<<<gr, 256, 0, st>>>(src, src_pitch, dst, dst_pitch, w, rows);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

int launch_timeflt(const FilterArgs& a, cudaStream_t st) {
  dim3 b(32, 8, 1);
  dim3 gr((ncols(a.g) + 1 + 31) / 32, (a.g.nj - 2 + 7) / 8, a.g.nk);
  k_timeflt<<<gr, b, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

int launch_halo(const HaloArgs& a, cudaStream_t st) {
  const int frame = 5 * (a.g.ni + 2) + 5 * (a.g.nj - 3);
  if (a.n < 1) return CRESS_OK;
  dim3 gr((frame + 127) / 128, a.g.nk, a.n);
  k_halo<<<gr, 128, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace cress

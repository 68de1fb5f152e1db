// Domain diagnostics of one time level for sm_100a: FP64 sums of the water
// and mass budgets, wind and theta' maxima, and a count of non-finite
// values.  The reference has no such sums (its run-time monitor is the
// max/min printout of s_mxndrv, SrcOrig/mxndrv.f90); they are the
// conservation check of the GPU path and its blow-up detector.
//
//   water  = sum rst(k) (qv+qc+qr+qi+qs+qg) dx dy dz          [kg]
//   precip = sum (prc+prr+pri+prs+prg accumulated) rhow dx dy [kg]
//   mass   = sum rst(k) (1 + p'/rcsq(k)) dx dy dz             [kg]
// (rst = rho_bar J, rcsq = rho_bar c^2, so rst p'/rcsq = J p'/c^2 is the
// acoustic density perturbation), over the physical cells i = 2..ni-2,
// j = 2..nj-2, k = 2..nk-2.  Every cell adds in double; each warp reduces
// with shuffles and adds once per quantity to the accumulators.
#include <cuda_runtime.h>
#include <cstdint>
#include "common.cuh"
#include "diag.cuh"
#include "hevi.cuh"

namespace cress {
namespace {

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned warp_max(unsigned v) {
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// |x| as ordered bits (non-negative floats order like their bit patterns)
__device__ __forceinline__ unsigned abs_bits(float x) { return __float_as_uint(fabsf(x)); }

__global__ void __launch_bounds__(256) k_diag(const DiagArgs a) {
  const Grid g = a.g;
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 2 + blockIdx.z;
  const bool in = i <= g.ni - 2 && j <= g.nj - 2 && k <= g.nk - 2;
  double water = 0.0, precip = 0.0, mass = 0.0;
  unsigned mu = 0, mv = 0, mw = 0, mt = 0, bad = 0;
  if (in) {
    const long long id = g.at(i, j, k);
    const int nc = g.nk + 1;
    const double rst = __ldg(a.col + C_RST * nc + k);
    const float u = __ldg(a.u + id), v = __ldg(a.v + id), w = __ldg(a.w + id);
    const float pp = __ldg(a.pp + id), ptp = __ldg(a.ptp + id);
    bad += !isfinite(u) + !isfinite(v) + !isfinite(w) + !isfinite(pp) + !isfinite(ptp);
    mu = abs_bits(u); mv = abs_bits(v); mw = abs_bits(w); mt = abs_bits(ptp);
    mass = rst * (1.0 + (double)pp / (double)__ldg(a.col + C_RCSQ * nc + k)) * a.dv;
    if (a.q[0]) {
      double qsum = 0.0;
      for (int n = 0; n < 6; ++n) {
        const float q = __ldg(a.q[n] + id);
        bad += !isfinite(q);
        qsum += (double)q;
      }
      for (int n = 0; n < 3; ++n) bad += !isfinite(__ldg(a.n[n] + id));
      water = rst * qsum * a.dv;
    }
    if (k == 2 && a.prec) {
      const long long pp2 = (long long)g.px * g.py, pid = (long long)j * g.px + i;
      double acc = 0.0;
      for (int s = 0; s < 5; ++s) acc += (double)__ldg(a.prec + (2 * s + 1) * pp2 + pid);
      precip = acc * 1.e3 * a.dxdy;   // rhow = 1e3 kg/m3 (comphy.f90)
    }
  }
  water = warp_sum(water); precip = warp_sum(precip); mass = warp_sum(mass);
  mu = warp_max(mu); mv = warp_max(mv); mw = warp_max(mw); mt = warp_max(mt);
  for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, o);
  if ((threadIdx.x & 31) == 0) {
    DiagAcc* d = a.acc;
    if (water != 0.0) atomicAdd(&d->sum[0], water);
    if (precip != 0.0) atomicAdd(&d->sum[1], precip);
    atomicAdd(&d->sum[2], mass);
    atomicMax(&d->maxbits[0], mu); atomicMax(&d->maxbits[1], mv);
    atomicMax(&d->maxbits[2], mw); atomicMax(&d->maxbits[3], mt);
    if (bad) atomicAdd(&d->nonfinite, (unsigned long long)bad);
  }
}

}  // namespace

int launch_diag(const DiagArgs& a, cudaStream_t st) {
  dim3 b(32, 8, 1);
  dim3 gr((a.g.ni - 3 + 31) / 32, (a.g.nj - 3 + 7) / 8, a.g.nk - 3);
  k_diag<<<gr, b, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace cress

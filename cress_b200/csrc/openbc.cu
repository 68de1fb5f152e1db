// Open (radiation) west and east boundaries for sm_100a: wbc = ebc in
// {4, 5, 7}, periodic y, advopt=2, no lateral damping (lbcvar 'x', so the
// reference's lbnews / lbnorm terms vanish), no GPV nudging.
//
//   k_rbc_small     per acoustic substep, after the HE-VI launch: s_rbcu,
//                   s_rbcv (stepuv.f90:266-280, rbcu.f90:228-300,
//                   rbcv.f90:324-400), s_rbcw (rbcw.f90:401-483), s_rbcss
//                   (rbcss.f90:392-472) on the boundary columns, then the
//                   vertical rules of vbcu/vbcv/vbcw/vbcp and the y wrap of
//                   those columns (bcycle.f90:182-199)
//   k_rbc_leapfrog  per large step, before the microphysics: s_rbcpt,
//                   s_rbcqv, s_rbcq, s_rbcs in leapfrog form (steps.f90:
//                   1024-1260; rbcpt.f90:626-760 and siblings), then vbcs
//                   (vbcs.f90:116-132)
//   k_phase         at the end of the large step: s_phasev (phvuvw.f90,
//                   phvs.f90) for every variable
//
// Every kernel works on the 2 x nj boundary columns only: a thread per
// (column, variable) walks k, so the few kilobytes per level they touch
// are negligible next to the interior kernels.  The interior kernels stay
// untouched except that with open x they write no x ghosts and narrow
// their 4th-order stencils at the boundary columns.
#include <cuda_runtime.h>
#include "hevi.cuh"
#include "openbc.cuh"

namespace cress {
namespace {

// Store v at (i, j, k) and at the y ghost the periodic wrap copies it to
// (scalar and u rows: j = nj-2 -> 1, j = 2 -> nj-1; v rows: j = nj-2 -> 1,
// j = 3 -> nj).
__device__ __forceinline__ void store_y(float* f, const Grid& g, bool vrow, int i, int j, int k, float v) {
  f[g.at(i, j, k)] = v;
  if (j == g.nj - 2) f[g.at(i, 1, k)] = v;
  if (vrow ? j == 3 : j == 2) f[g.at(i, vrow ? g.nj : g.nj - 1, k)] = v;
}

// blockIdx.y: side (0 west, 1 east); threads over j = 2..nj-1.
__global__ void __launch_bounds__(128) k_rbc_small(const RbcSmallArgs a) {
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const int side = blockIdx.y;
  const int j = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  if (j > nj - 1) return;
  auto C = [&](int var, int k) { return __ldg(a.cp + rad_at(g, var, side, j, k)); };
  // radiation step toward the neighbour column: west s - c*(s2 - s), east s + c*(s2 - s)
  auto rad = [&](float s, float s2, float c) { return side == 0 ? s - c * (s2 - s) : s + c * (s2 - s); };
  {  // v: i = 1 / ni-1, rows 2..nj-1 (rbcv.f90:324-400), vbcv, level nk carried over
    const int ib = side == 0 ? 1 : ni - 1, in = side == 0 ? 2 : ni - 2;
    float v2 = 0.f, vt = 0.f;
    for (int k = 2; k <= nk - 2; ++k) {
      const float v = rad(a.v_old[g.at(ib, j, k)], a.v_old[g.at(in, j, k)], C(RAD_V, k));
      store_y(a.v_new, g, true, ib, j, k, v);
      if (k == 2) v2 = v;
      vt = v;
    }
    store_y(a.v_new, g, true, ib, j, 1, v2);
    store_y(a.v_new, g, true, ib, j, nk - 1, vt);
    store_y(a.v_new, g, true, ib, j, nk, a.v_old[g.at(ib, j, nk)]);
  }
  if (j > nj - 2) return;
  {  // u: i = 1 / ni (rbcu.f90:228-300), vbcu, level nk carried over
    const int ib = side == 0 ? 1 : ni, in = side == 0 ? 2 : ni - 1;
    float u2 = 0.f, ut = 0.f;
    for (int k = 2; k <= nk - 2; ++k) {
      const float u = rad(a.u_old[g.at(ib, j, k)], a.u_old[g.at(in, j, k)], C(RAD_U, k));
      store_y(a.u_new, g, false, ib, j, k, u);
      if (k == 2) u2 = u;
      ut = u;
    }
    store_y(a.u_new, g, false, ib, j, 1, u2);
    store_y(a.u_new, g, false, ib, j, nk - 1, ut);
    store_y(a.u_new, g, false, ib, j, nk, a.u_old[g.at(ib, j, nk)]);
  }
  const int ib = side == 0 ? 1 : ni - 1, in = side == 0 ? 2 : ni - 2;
  {  // w: k = 2..nk-1 (rbcw.f90:401-483), then phy2cnt + vbcw (flat terrain)
    float w3 = 0.f, wt = 0.f;
    for (int k = 3; k <= nk - 2; ++k) {
      const float w = rad(a.w_old[g.at(ib, j, k)], a.w_old[g.at(in, j, k)], C(RAD_W, k));
      store_y(a.w_new, g, false, ib, j, k, w);
      if (k == 3) w3 = w;
      wt = w;
    }
    const float j8w3 = __ldg(a.col + C_JCB8W * (nk + 1) + 3), j8wt = __ldg(a.col + C_JCB8W * (nk + 1) + nk - 2);
    const float wc3 = a.sthopt ? w3 / j8w3 : w3;       // phy2cnt.f90:219
    const float wct = a.sthopt ? wt / j8wt : wt;
    // levels 2 and nk-1 come out of rbcw and are then zeroed by vbcw (rigid
    // ground and lid, bbc = tbc = 2, the only setting the library accepts)
    store_y(a.w_new, g, false, ib, j, 1, -j8w3 * wc3 - 0.f);
    store_y(a.w_new, g, false, ib, j, 2, 0.f);
    store_y(a.w_new, g, false, ib, j, nk - 1, 0.f);
    store_y(a.w_new, g, false, ib, j, nk, -j8wt * wct - 0.f);
  }
  {  // p': k = 2..nk-2 (rbcss.f90:392-472), vbcp, level nk carried over
    float p2 = 0.f, p3 = 0.f, pt = 0.f;
    for (int k = 2; k <= nk - 2; ++k) {
      const float p = rad(a.p_old[g.at(ib, j, k)], a.p_old[g.at(in, j, k)], C(RAD_P, k));
      store_y(a.p_new, g, false, ib, j, k, p);
      if (k == 2) p2 = p;
      if (k == 3) p3 = p;
      pt = p;
    }
    store_y(a.p_new, g, false, ib, j, 1, a.bbc == 2 ? 2.f * p2 - p3 : p2);
    store_y(a.p_new, g, false, ib, j, nk - 1, pt);
    store_y(a.p_new, g, false, ib, j, nk, a.p_old[g.at(ib, j, nk)]);
  }
}

// blockIdx.y: field, blockIdx.z: side; threads over j = 2..nj-2.  The y
// ghosts follow with the end-of-step wrap.
__global__ void __launch_bounds__(128) k_rbc_leapfrog(const RbcLeapArgs a) {
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const int f = blockIdx.y, side = blockIdx.z;
  const int j = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  if (j > nj - 2 || f >= a.n) return;
  const int ib = side == 0 ? 1 : ni - 1, in = side == 0 ? 2 : ni - 2;
  const int var = a.var[f], kind = a.kind[f];
  const float* s = a.s[f];
  const float* sp = a.sp[f];
  float* sf = a.sf[f];
  float v2 = 0.f, vt = 0.f;
  for (int k = 2; k <= nk - 2; ++k) {
    const float c = __ldg(a.cp + rad_at(g, var, side, j, k));
    const float p = sp[g.at(ib, j, k)], d = s[g.at(in, j, k)] - p;
    // west gamma = 2c/(1-c), sf = sp - gamma*d; east gamma = 2c/(1+c), sf = sp + gamma*d
    const float gam = side == 0 ? 2.f * c / (1.f - c) : 2.f * c / (1.f + c);
    float v = side == 0 ? p - gam * d : p + gam * d;
    if (kind == 1 || kind == 2) v = fmaxf(v, 0.f);   // rbcqv.f90:660, rbcq.f90:655
    sf[g.at(ib, j, k)] = v;
    if (k == 2) v2 = v;
    vt = v;
  }
  sf[g.at(ib, j, 1)] = v2;        // vbcs.f90:118
  sf[g.at(ib, j, nk - 1)] = vt;   // vbcs.f90:132
}

// blockIdx.y: variable, blockIdx.z: side; threads over j = 1..jend.
__global__ void __launch_bounds__(128) k_phase(const PhaseArgs a) {
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const int f = blockIdx.y, side = blockIdx.z;
  if (f >= a.n) return;
  const int var = a.var[f];
  // per variable: east points (u: ni-1, ni-2; the rest ni-2, ni-3), rows, levels
  const int ie1 = var == RAD_U ? ni - 1 : ni - 2;
  const int jend = var == RAD_V ? nj : nj - 1;
  const int kend = var == RAD_W ? nk - 1 : nk - 2;
  const bool sml = var <= RAD_P;   // scaled to the small step (phasev.f90:464-477)
  const int j = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (j > jend) return;
  const int i1 = side == 0 ? 2 : ie1, i2 = side == 0 ? 3 : ie1 - 1;
  const float* s = a.s[f];
  const float* sp = a.sp[f];
  const float* sf = a.sf[f];
  const float eps = 1.e-20f;                          // commath.f90:177
  const float gw = a.gwave * a.dtb * a.dxiv;          // gdxdt; gdxdtn = -gdxdt
  const float dtsdb = a.dts / a.dtb;
  const float nkv = 1.f / (float)(kend - 1);          // nkm3v or nkm2v (w)
  float* out = a.cp;
  float av = 0.f;
  for (int k = 2; k <= kend; ++k) {
    float c;
    if (a.obc == 4 || a.obc == 5) {
      const float fv = sf[g.at(i1, j, k)], pv = sp[g.at(i1, j, k)], nv = s[g.at(i2, j, k)];
      float den = side == 0 ? (fv + pv) - 2.f * nv : (2.f * nv - fv) - pv;
      if (fabsf(den) < eps) den = copysignf(eps, den);
      c = (fv - pv) / den;
      c = side == 0 ? fminf(c, -gw) : fmaxf(c, gw);
    } else {
      c = side == 0 ? -gw : gw;
    }
    if (a.obc == 5) av = av + c * nkv;
    out[rad_at(g, var, side, j, k)] = c;
  }
  for (int k = 2; k <= kend; ++k) {
    float c = a.obc == 5 ? av : out[rad_at(g, var, side, j, k)];
    c = side == 0 ? fmaxf(c, -1.f) : fminf(c, 1.f);
    if (sml) c = c * dtsdb;
    out[rad_at(g, var, side, j, k)] = c;
  }
}

}  // namespace

int launch_rbc_small(const RbcSmallArgs& a, cudaStream_t st) {
  dim3 gr((a.g.nj - 2 + 127) / 128, 2, 1);
  k_rbc_small<<<gr, 128, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

int launch_rbc_leapfrog(const RbcLeapArgs& a, cudaStream_t st) {
  if (a.n < 1 || a.n > 10) return CRESS_E_ARG;
  dim3 gr((a.g.nj - 3 + 127) / 128, a.n, 2);
  k_rbc_leapfrog<<<gr, 128, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

int launch_phase(const PhaseArgs& a, cudaStream_t st) {
  if (a.n < 1 || a.n > 14) return CRESS_E_ARG;
  dim3 gr((a.g.nj + 127) / 128, a.n, 2);
  k_phase<<<gr, 128, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace cress

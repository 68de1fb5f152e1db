// Eddy viscosity for sm_100a (isoopt=1, trnopt=0, mfcopt=0, sfcopt=0): one
// thread per scalar point i, j = 1..n-1, k = 1..nk-1 forms
//   N^2 at the w levels k and k+1      s_bruntv, SrcOrig/bruntv.f90:212-345
//   the deformation and its square     s_defomten / s_defomssq
//                                      (defomten.f90:305-1106, defomssq.f90:130-141)
// from the past level, then either the Smagorinsky form (tubopt=1)
//   rkv = rbr min(cs^2 l^2 sqrt(max(ssq - N^2/Pr, 0)), ckmax l^2)
//                                      s_eddyvis, eddyvis.f90:213-268
// or the Deardorff form from the past TKE e (tubopt=2)
//   l = l0 in unstable air, else max(0.1 l0, min(0.76 sqrt(e/N^2), l0)),
//   1/Pr = 1 + 2 l/l0, rkv = rbr min(max(ckm l sqrt(e), ckmin l0^2 where
//   1/Pr N^2 < ssq), ckmax l0^2)   s_eddyvis, eddyvis.f90:448-481
// and writes rkv (one field).  With the TKE closure it also writes what the
// TKE equation and the scalar mixing take from this point, so no later
// kernel recomputes the deformation or N^2:
//   rks = 1/Pr * rkv/jcb               s_eddyvisj + s_eddydif
//                                      (eddyvisj.f90:121-134, eddydif.f90:265-284)
//   nsq = N^2 at w level k             (s_buoytke's nsq8w, buoytke.f90:124-134)
//   shr = jcb rkv ssq                  s_sheartke, sheartke.f90:112-120
//   dsp = (0.37/Pr - 0.18) rst e^1.5 / ((1/Pr - 1) (dx dy dz jcb/8)^(1/3) + eps)
//                                      s_disptke, disptke.f90:181-195
// The stresses, their divergence and the scalar fluxes (strsten, turbuvw,
// kh8uv, turbflx, turbs, tkeflx, turbtke) are formed where they are used,
// in k_force, k_scalars and k_tke, from these fields and the past winds.
#include <cuda_runtime.h>
#include "common.cuh"
#include "forcing.cuh"
#include "hevi.cuh"
#include "turb.cuh"

namespace cress {
namespace {

// comphy.f90:61-130 constants used by bruntv
constexpr float kRd = 287.f, kCp = 1004.f, kEpsva = .622f, kEpsav = 1.6077f, kTlow = 233.16f;
constexpr float kLv0 = 2.50078e6f, kLf0 = 3.34e5f, kT0 = 273.16f, kCwmci = 4.218e3f - 2.106e3f;

// Each thread owns one column (i, j) and marches k = 1..nk-1 upward, so the
// thermodynamics of a level (bruntv's theta, and in moist air its
// saturated and virtual forms, which cost five exp/log each) is formed
// once and serves N^2 at the w levels below and above it, and the z-x /
// z-y deformation components at the upper faces of level k are kept for
// the lower faces of level k+1.  The block first copies the level table
// into shared memory (the columns and the reciprocals defomten and bruntv
// divide by, one shared load each) and forms the per-level length scales
// (ds3 jcb)^(1/3) and (ds308 jcb)^(1/3) once per level instead of once per
// point.
constexpr int kTurbThreads = 128;

template <bool TKE>
__global__ void __launch_bounds__(kTurbThreads) k_turb_visc(const TurbArgs a) {
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  extern __shared__ __align__(16) float tsm[];
  float* tab = tsm;                                   // rows 0..nk of the level table
  float* lnk = tab + (nk + 1) * kLevelStride;         // (ds3 jcb)^(1/3) per level
  float* ldk = lnk + (nk + 1);                        // (ds308 jcb)^(1/3) per level (TKE)
  const float oned3 = 1.f / 3.f;
  {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const float4* src = reinterpret_cast<const float4*>(a.lvl);
    float4* dst = reinterpret_cast<float4*>(tab);
    const int nv = (nk + 1) * kLevelStride / 4;
    for (int v = tid; v < nv; v += kTurbThreads) dst[v] = __ldg(src + v);
    for (int kk = tid; kk <= nk; kk += kTurbThreads) {
      const float jcb = __ldg(a.lvl + kk * kLevelStride + C_JCB);
      lnk[kk] = expf(oned3 * logf(a.ds3 * jcb));
      if constexpr (TKE) ldk[kk] = expf(oned3 * logf(a.ds308 * jcb));
    }
  }
  __syncthreads();
  if (i > ni - 1 || j > nj - 1) return;
  const long long px = g.px, pl = g.plane;
  const long long id0 = g.at(i, j, 1);
  auto C = [&](int f, int kk) { return tab[kk * kLevelStride + f]; };
  const float gdzv = 9.8f * a.dziv, gdzv05 = .5f * 9.8f * a.dziv;
  const bool moist = a.qvp != nullptr;

  // bruntv's per-level quantities of level kl (1..nk-1)
  struct Lev { float pt, ptm, av, ptv, qall; };
  auto lev = [&](int kl) {
    const long long p = id0 + (long long)(kl - 1) * pl;
    Lev L{};
    L.pt = C(C_PTBR, kl) + __ldg(a.ptpp + p);
    if (moist) {
      const float pt = L.pt;
      const float qv = __ldg(a.qvp + p);
      L.ptv = pt * (1.f + kEpsav * qv) / (1.f + qv);
      const float t = pt * expf((kRd / kCp) * logf((1.f / 1.e5f) * (C(C_PBR, kl) + __ldg(a.ppp + p))));
      float av = kLv0 * expf((.167f + 3.67e-4f * t) * logf(kT0 / t));
      if (t <= kTlow) av = av + (kLf0 + kCwmci * (t - kT0));
      const float lhcpt = av / (kCp * t);
      L.ptm = pt * expf(lhcpt * qv);
      av = av * qv / (kRd * t);
      L.av = (1.f + av) / (1.f + kEpsva * lhcpt * av);
      L.qall = (((__ldg(a.qcp + p) + __ldg(a.qrp + p)) + __ldg(a.qip + p)) + __ldg(a.qsp + p)) + __ldg(a.qgp + p);
    }
    return L;
  };
  // N^2 at w level kk (2..nk-1) from levels kk-1 and kk
  auto nsqv = [&](const Lev& l0, const Lev& l1, int kk) -> float {
    const float b0 = C(C_PTBR, kk - 1), b1 = C(C_PTBR, kk);
    if (moist && l1.qall > a.thresq)
      return gdzv05 * ((l0.qall - l1.qall) + (l1.ptm - l0.ptm) * (l0.av + l1.av) / (b0 + b1)) / C(C_JCB8W, kk);
    const float d = moist ? l1.ptv - l0.ptv : l1.pt - l0.pt;
    return gdzv * d / (C(C_JCB8W, kk) * (b0 + b1));
  };

  Lev lc = lev(2);   // the upper level of the last N^2 formed
  float nq = 0.f, c31_0 = 0.f, c31_1 = 0.f, c32_0 = 0.f, c32_1 = 0.f;
  for (int k = 1; k <= nk - 1; ++k) {
    const long long id = id0 + (long long)(k - 1) * pl;
    auto U = [&](int x, int y, int z) { return __ldg(a.up + id + x + y * px + z * pl); };
    auto V = [&](int x, int y, int z) { return __ldg(a.vp + id + x + y * px + z * pl); };
    auto W = [&](int x, int y, int z) { return __ldg(a.wp + id + x + y * px + z * pl); };
    const auto D = deform_at(C, U, V, W, k, nk, a.dxiv, a.dyiv, a.dziv);
    if (k == 1) {
      c31_0 = D.s31(0, 0, 0); c31_1 = D.s31(1, 0, 0);
      c32_0 = D.s32(0, 0, 0); c32_1 = D.s32(0, 1, 0);
    }
    // N^2 at the w levels k and k+1, clamped to 2..nk-1 (level 1 takes
    // level 2's, level nk level nk-1's: bruntv.f90:337-345)
    float nk0, nk1;
    if (k == 1) {
      nq = nsqv(lev(1), lc, 2);
      nk0 = nk1 = nq;
    } else {
      nk0 = nq;
      if (k + 1 <= nk - 1) {
        const Lev l1 = lev(k + 1);
        nk1 = nsqv(lc, l1, k + 1);
        lc = l1;
      } else {
        nk1 = nk0;
      }
      nq = nk1;
    }
    const float n31_0 = D.s31(0, 0, 1), n31_1 = D.s31(1, 0, 1);
    const float n32_0 = D.s32(0, 0, 1), n32_1 = D.s32(0, 1, 1);
    const float s11 = D.s11(0, 0, 0), s22 = D.s22(0, 0, 0), s33 = D.s33(0, 0, 0);
    const float s128s = (D.s12(0, 0, 0) + D.s12(1, 1, 0)) + (D.s12(1, 0, 0) + D.s12(0, 1, 0));
    const float s318s = (c31_0 + n31_1) + (n31_0 + c31_1);
    const float s328s = (c32_0 + n32_1) + (n32_0 + c32_1);
    c31_0 = n31_0; c31_1 = n31_1; c32_0 = n32_0; c32_1 = n32_1;
    const float ssq =
        .5f * (s33 * s33 + (s11 * s11 + s22 * s22)) + .0625f * (s128s * s128s + (s318s * s318s + s328s * s328s));
    if constexpr (!TKE) {
      const float ln = lnk[k];   // (ds3 jcb)^(1/3)
      const float ln2 = ln * ln;
      float kv = (.21f * .21f) * ln2 * sqrtf(fmaxf(ssq - (nk0 + nk1) * a.cpriv, 0.f));
      kv = C(C_RBR, k) * fminf(kv, a.ckmax * ln2);
      a.rkv[id] = kv;
    } else {
      constexpr float ckm = .1f, ckmin = 1.e-6f, eps = 1.e-20f;   // comphy.f90:341-344, commath.f90:177
      const float jcb = C(C_JCB, k);
      const float ln0 = lnk[k];   // (ds3 jcb)^(1/3)
      const float ln02 = ln0 * ln0;
      const float ns = nk0 + nk1;
      const float e = __ldg(a.tkep + id);
      const float ln = ns < 0.f ? ln0 : fmaxf(.1f * ln0, fminf(.76f * sqrtf(e / (ns + eps)), ln0));
      const float priv = 1.f + 2.f * ln / ln0;
      float kv = ckm * ln * sqrtf(e);
      if (priv * ns < ssq) kv = fmaxf(kv, ckmin * ln02);
      kv = C(C_RBR, k) * fminf(kv, a.ckmax * ln02);
      a.rkv[id] = kv;
      a.rks[id] = priv * (C(C_IJCB, k) * kv);
      a.nsq[id] = nk0;
      a.shr[id] = jcb * kv * ssq;
      const float ld = (priv - 1.f) * ldk[k] + eps;   // (ds308 jcb)^(1/3)
      a.dsp[id] = (.37f * priv - .18f) * C(C_RST, k) * e * sqrtf(e) / ld;
    }
  }
}

}  // namespace

int launch_turb_visc(const TurbArgs& a, cudaStream_t st) {
  if (a.g.nk < 4 || !a.lvl) return CRESS_E_UNSUPPORTED;
  const size_t bytes = sizeof(float) * ((size_t)(a.g.nk + 1) * kLevelStride + 2 * (size_t)(a.g.nk + 1));
  if (bytes > 48 * 1024) return CRESS_E_UNSUPPORTED;
  dim3 b(32, kTurbThreads / 32, 1);
  dim3 gr((a.g.ni - 1 + 31) / 32, (a.g.nj - 1 + b.y - 1) / b.y, 1);
  if (a.tkep)
    k_turb_visc<true><<<gr, b, bytes, st>>>(a);
  else
    k_turb_visc<false><<<gr, b, bytes, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace cress

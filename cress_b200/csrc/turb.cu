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

template <bool TKE>
__global__ void __launch_bounds__(256) k_turb_visc(const TurbArgs a) {
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > ni - 1 || j > nj - 1 || k > nk - 1) return;
  const long long px = g.px, pl = g.plane;
  const long long id = g.at(i, j, k);
  const int nc = nk + 1;
  auto B = [&](int f, int kk) { return __ldg(a.col + f * nc + kk); };
  auto C = [&](int f, int kk) { return level_value(f, kk, B, 0.f); };
  auto U = [&](int x, int y, int z) { return __ldg(a.up + id + x + y * px + z * pl); };
  auto V = [&](int x, int y, int z) { return __ldg(a.vp + id + x + y * px + z * pl); };
  auto W = [&](int x, int y, int z) { return __ldg(a.wp + id + x + y * px + z * pl); };
  const auto D = deform_at(C, U, V, W, k, nk, a.dxiv, a.dyiv, a.dziv);
  const float gdzv = 9.8f * a.dziv, gdzv05 = .5f * 9.8f * a.dziv;
  const bool moist = a.qvp != nullptr;

  // N^2 at w level kk (2..nk-1); below and above, the nearest defined level
  auto nsq = [&](int kk) -> float {
    kk = max(2, min(kk, nk - 1));
    const long long p1 = id + (long long)(kk - k) * pl, p0 = p1 - pl;
    const float b0 = C(C_PTBR, kk - 1), b1 = C(C_PTBR, kk);
    const float pt0 = b0 + __ldg(a.ptpp + p0), pt1 = b1 + __ldg(a.ptpp + p1);
    if (!moist) return gdzv * (pt1 - pt0) / (C(C_JCB8W, kk) * (b0 + b1));
    struct Lev { float ptm, av, ptv, qall; };
    auto lev = [&](long long p, int kl, float pt) {
      Lev L;
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
      return L;
    };
    const Lev l0 = lev(p0, kk - 1, pt0), l1 = lev(p1, kk, pt1);
    if (l1.qall > a.thresq)
      return gdzv05 * ((l0.qall - l1.qall) + (l1.ptm - l0.ptm) * (l0.av + l1.av) / (b0 + b1)) / C(C_JCB8W, kk);
    return gdzv * (l1.ptv - l0.ptv) / (C(C_JCB8W, kk) * (b0 + b1));
  };

  const float s11 = D.s11(0, 0, 0), s22 = D.s22(0, 0, 0), s33 = D.s33(0, 0, 0);
  const float s128s = (D.s12(0, 0, 0) + D.s12(1, 1, 0)) + (D.s12(1, 0, 0) + D.s12(0, 1, 0));
  const float s318s = (D.s31(0, 0, 0) + D.s31(1, 0, 1)) + (D.s31(0, 0, 1) + D.s31(1, 0, 0));
  const float s328s = (D.s32(0, 0, 0) + D.s32(0, 1, 1)) + (D.s32(0, 0, 1) + D.s32(0, 1, 0));
  const float ssq = .5f * (s33 * s33 + (s11 * s11 + s22 * s22)) + .0625f * (s128s * s128s + (s318s * s318s + s328s * s328s));
  const float oned3 = 1.f / 3.f;
  if constexpr (!TKE) {
    const float ln = expf(oned3 * logf(a.ds3 * C(C_JCB, k)));
    const float ln2 = ln * ln;
    float kv = (.21f * .21f) * ln2 * sqrtf(fmaxf(ssq - (nsq(k) + nsq(k + 1)) * a.cpriv, 0.f));
    kv = C(C_RBR, k) * fminf(kv, a.ckmax * ln2);
    a.rkv[id] = kv;
  } else {
    constexpr float ckm = .1f, ckmin = 1.e-6f, eps = 1.e-20f;   // comphy.f90:341-344, commath.f90:177
    const float jcb = C(C_JCB, k);
    const float ln0 = expf(oned3 * logf(a.ds3 * jcb));
    const float ln02 = ln0 * ln0;
    const float nk0 = nsq(k);
    const float ns = nk0 + nsq(k + 1);
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
    const float ld = (priv - 1.f) * expf(oned3 * logf(a.ds308 * jcb)) + eps;
    a.dsp[id] = (.37f * priv - .18f) * C(C_RST, k) * e * sqrtf(e) / ld;
  }
}

}  // namespace

int launch_turb_visc(const TurbArgs& a, cudaStream_t st) {
  dim3 b(32, 8, 1);
  dim3 gr((a.g.ni - 1 + 31) / 32, (a.g.nj - 1 + 7) / 8, a.g.nk - 1);
  if (a.tkep)
    k_turb_visc<true><<<gr, b, 0, st>>>(a);
  else
    k_turb_visc<false><<<gr, b, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace cress

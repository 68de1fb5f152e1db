// Smagorinsky eddy viscosity for sm_100a (tubopt=1, isoopt=1, trnopt=0,
// mfcopt=0): one thread per scalar point i, j = 1..n-1, k = 1..nk-1 forms
//   N^2 at the w levels k and k+1      s_bruntv, SrcOrig/bruntv.f90:212-345
//   the deformation and its square     s_defomten / s_defomssq
//                                      (defomten.f90:305-1106, defomssq.f90:130-141)
//   rkv = rbr min(cs^2 l^2 sqrt(max(ssq - N^2/Pr, 0)), ckmax l^2)
//                                      s_eddyvis, eddyvis.f90:213-268
// from the past level and writes rkv (one field).  The stresses, their
// divergence and the scalar diffusivities (strsten, turbuvw, eddydif,
// kh8uv, turbflx, turbs) are formed where they are used, in k_force and
// k_moist_scalars, from this field and the past winds.
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
  const float ln = expf((1.f / 3.f) * logf(a.ds3 * C(C_JCB, k)));
  const float ln2 = ln * ln;
  float kv = (.21f * .21f) * ln2 * sqrtf(fmaxf(ssq - (nsq(k) + nsq(k + 1)) * a.cpriv, 0.f));
  kv = C(C_RBR, k) * fminf(kv, a.ckmax * ln2);
  a.rkv[id] = kv;
}

}  // namespace

int launch_turb_visc(const TurbArgs& a, cudaStream_t st) {
  dim3 b(32, 8, 1);
  dim3 gr((a.g.ni - 1 + 31) / 32, (a.g.nj - 1 + 7) / 8, a.g.nk - 1);
  k_turb_visc<<<gr, b, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace cress

// Forcing and leapfrog step of the turbulent kinetic energy for sm_100a
// (tubopt=2, isoopt=1, flat terrain, no surface flux): s_forcetke
// (SrcOrig/forcetke.f90:269-354) and the TKE part of s_steps, with the
// terms added in the reference's order
//   tkefrc = advs of the present TKE             (advs.f90:205-370)
//          + jcb rkv ssq                         (sheartke.f90:112-120)
//          + smoo4s of rbr*tkep                  (smoo4s.f90:184-296)
//          - dissipation                         (disptke.f90:181-195)
//          + div(2 K grad tkep), K = rkv/jcb     (eddyvisj.f90:121-134,
//                                                 tkeflx.f90:251-462, turbtke.f90:203-237)
//          - vsps0 of tkep when vspvar(10:10)='o' (vsps0.f90:114-124)
//          - (b(k) + b(k+1)), b(k) = jcb8w N^2(k) (r8s(k-1) + r8s(k)),
//            r8s = 0.5 jcb 1/Pr rkv/jcb         (eddydif.f90:333-359, buoytke.f90:124-151)
//   tkef   = max(0, tkep + tkefrc 2dtb/rst)      (steps.f90:999-1014), then vbcs.
// The shear and dissipation terms, N^2 and the scalar diffusivity come
// per point from k_turb_visc (rks, nsq, shr, dsp); they are read on the
// thread's own columns one level ahead of their use, N^2 and the
// diffusivity of levels k-1 .. k+1 carried in registers as the march goes
// up.
//
// Design (2.5-D), as the moist scalar kernel: a block owns a 32 x 8 tile
// of columns and marches k upward; one elected thread issues TMA boxes of
// the TKE at t and t-dt (two rows of y halo), u, v, w and the eddy
// viscosity (one row of y halo) of every level 1..nk-1 into an S-stage
// shared-memory ring guarded by bounded mbarrier waits, so every neighbour
// of the advection, smoothing and transport stencils is a shared-memory
// read.  Each thread owns a pair of x-neighbouring columns and computes
// both with packed FP32x2 arithmetic (f2.cuh).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "common.cuh"
#include "f2.cuh"
#include "forcing.cuh"
#include "hevi.cuh"
#include "stencil.cuh"
#include "tke.cuh"
#include "tma.cuh"

namespace cress {
namespace {

__host__ __device__ constexpr int r128f(int n) { return (n + 31) / 32 * 32; }  // floats -> multiple of 128 B

constexpr int kTkePairs = kHeviTX / 2;

template <int S>
struct TkeLayout {
  using R = TkeRows;
  static constexpr int BX = kHeviBoxX;
  static constexpr int oS = 0;                              // TKE at t, rows j0-2 ..
  static constexpr int oSP = oS + r128f(BX * R::s);         // TKE at t-dt, rows j0-2 ..
  static constexpr int oU = oSP + r128f(BX * R::s);         // rows j0 ..
  static constexpr int oV = oU + r128f(BX * R::u);          // rows j0-1 ..
  static constexpr int oW = oV + r128f(BX * R::v);          // rows j0 ..
  static constexpr int oR = oW + r128f(BX * R::w);          // eddy viscosity, rows j0-1 ..
  static constexpr int stage = oR + r128f(BX * R::r);       // floats per ring stage
  static constexpr uint32_t tx_bytes = 4u * BX * (2 * R::s + R::u + R::v + R::w + R::r);
  static constexpr int NF = kLevelStride;
  __host__ __device__ static size_t bytes() { return 4 * (size_t)S * stage + 8 * (size_t)S; }
};

__device__ __forceinline__ F2 ldg2(const float* p) { return F2{__ldg(reinterpret_cast<const float2*>(p))}; }

template <int S>
__global__ void __launch_bounds__(kTkePairs * kScalarTY) k_tke(const __grid_constant__ TkeMaps m, const TkeArgs a) {
  static_assert(S >= 6, "ring too shallow for the k-2..k+2 window");
  using L = TkeLayout<S>;
  constexpr int TY = kScalarTY, BX = kHeviBoxX;
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const int i0 = 2 + blockIdx.x * kHeviTX, j0 = 2 + blockIdx.y * TY;
  const int xb = i0 - 2;   // box x origin (multiple of 32)
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTkePairs + tx;
  const int i = i0 + 2 * tx, j = j0 + ty;
  // ownB implies ownA (i+1 <= ni-2 gives i <= ni-2)
  const bool ownA = (i <= ni - 2) && (j <= nj - 2), ownB = (i + 1 <= ni - 2) && (j <= nj - 2);

  extern __shared__ __align__(1024) float smem[];
  float* ring = smem;
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring + S * L::stage);
  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  // Levels 1..nk-1 are staged; level lv lives in slot (lv-1) % S.
  const int lmax = nk - 1;
  int issued = 0;   // highest level thread 0 has issued
  auto issue = [&](int lv) {
    issued = lv;
    const int s = (lv - 1) % S;
    float* st = ring + s * L::stage;
    uint64_t* bar = &bars[s];
    const int z = lv - 1;
    mbar_arrive_expect_tx(bar, L::tx_bytes);
    tma_load_3d(st + L::oS, &m.s, xb, j0 - 2, z, bar);
    tma_load_3d(st + L::oSP, &m.sp, xb, j0 - 2, z, bar);
    tma_load_3d(st + L::oU, &m.u, xb, j0, z, bar);
    tma_load_3d(st + L::oV, &m.v, xb, j0 - 1, z, bar);
    tma_load_3d(st + L::oW, &m.w, xb, j0, z, bar);
    tma_load_3d(st + L::oR, &m.rkv, xb, j0 - 1, z, bar);
  };
  if (tid == 0)
    for (int lv = 1; lv <= min(S, lmax); ++lv) issue(lv);

  bool fail = false;
  auto wait_level = [&](int lv) {
    if (!fail && lv <= lmax) fail = !mbar_wait(&bars[(lv - 1) % S], ((lv - 1) / S) & 1);
  };
  for (int lv = 1; lv <= 3; ++lv) wait_level(lv);

  const float oned24 = 1.f / 24.f, fourd3 = 4.f / 3.f;
  const float dxv24 = oned24 * a.dxiv, dyv24 = oned24 * a.dyiv;
  const float dxv05n = -.5f * a.dxiv, dyv05n = -.5f * a.dyiv, dzv05n = -.5f * a.dziv;
  const float dxv5 = .5f * a.dxiv, dyv5 = .5f * a.dyiv, dzv5 = .5f * a.dziv;          // tkeflx.f90:192-194
  const float dxiv2 = 2.f * a.dxiv, dyiv2 = 2.f * a.dyiv, dziv2 = 2.f * a.dziv;      // turbtke.f90:193-195
  const bool smooth = (a.smtopt % 10 == 2) || (a.smtopt % 10 == 3);
  const bool vsp = a.vspopt >= 1 && a.vsp_tke;
  // own pair in the boxes (x offset even, so every pair load is 8-byte
  // aligned): TKE rows from j0-2, u and w rows from j0, v and viscosity
  // rows from j0-1
  const int ox = 2 * tx + 2, oU = ty * BX + ox, oV = (ty + 1) * BX + ox;
  const int oS = (ty + 2) * BX + ox, oR = (ty + 1) * BX + ox;
  const long long plane = g.plane;
  long long id = g.at(i, j, 2);
  // per-point fields of levels k-1 .. k+1 on the own columns (registers),
  // each loaded one level ahead of its use
  F2 r8m = f2(0.f), r80 = f2(0.f), nq0 = f2(0.f);
  F2 shr_n = f2(0.f), dsp_n = f2(0.f), r8p_n = f2(0.f), nq1_n = f2(0.f);
  if (ownA) {
    r8m = ldg2(a.rks + id - plane);
    r80 = ldg2(a.rks + id);
    nq0 = ldg2(a.nsq + id);
    shr_n = ldg2(a.shr + id);
    dsp_n = ldg2(a.dsp + id);
    r8p_n = ldg2(a.rks + id + plane);
    nq1_n = ldg2(a.nsq + id + plane);
  }
  auto slot_ptr = [&](int lv) { return ring + ((lv - 1 + S) % S) * L::stage; };
  const float* stp[5] = {slot_ptr(0), slot_ptr(1), slot_ptr(2), slot_ptr(3), slot_ptr(4)};

  for (int k = 2; k <= nk - 2; ++k, id += plane) {
    wait_level(k + 2);
    // Every thread has finished level k-1, so the slot of level k-3 (last
    // read as k'-2 at k' = k-1) may be refilled with level k+S-3.
    __syncthreads();
    if (tid == 0 && !fail && k >= 4 && k + S - 3 <= lmax) {   // refill only after its copy was seen to land
      fence_proxy_async_smem();
      issue(k + S - 3);
    }
    if (ownA && !fail) {
      const float* ck = a.lvl + k * L::NF;
      auto C = [&](int f, int kk) { return __ldg(ck + (kk - k) * L::NF + f); };
      auto st = [&](int d) { return stp[d + 2]; };
      const float* st0 = st(0);
      const float* S0 = st0 + L::oS + oS;
      const float* SP0 = st0 + L::oSP + oS;
      const float* U = st0 + L::oU + oU;
      const float* V = st0 + L::oV + oV;
      const F2 shr = shr_n, dsp = dsp_n, r8p = r8p_n, nq1 = nq1_n;
      if (k + 1 <= nk - 2) {   // the next level's
        shr_n = ldg2(a.shr + id + plane);
        dsp_n = ldg2(a.dsp + id + plane);
        r8p_n = ldg2(a.rks + id + 2 * plane);
        nq1_n = ldg2(a.nsq + id + 2 * plane);
      }

      // advs.f90:205-370 with the fluxes of rstuvwc.f90:172-210
      const float r8u = C(C_RST8U, k), r8v = C(C_RST8V, k);
      const F2 fu_m1 = r8u * pair_at(U, -1), fu_0 = r8u * ld2(U);
      const F2 fu_p1 = r8u * pair_at(U, 1), fu_p2 = r8u * ld2(U + 2);
      const F2 fv_m1 = r8v * ld2(V - BX), fv_0 = r8v * ld2(V);
      const F2 fv_p1 = r8v * ld2(V + BX), fv_p2 = r8v * ld2(V + 2 * BX);
      auto WC = [&](F2 w, int kk) { return a.sthopt ? w * C(C_IJCB8W, kk) : w; };
      const F2 fw_0 = C(C_RST8W, k) * WC(ld2(st0 + L::oW + oU), k);
      const F2 fw_1 = C(C_RST8W, k + 1) * WC(ld2(st(1) + L::oW + oU), k + 1);
      const F2 s0 = ld2(S0);
      const F2 t1a = fu_0 * (s0 - pair_at(S0, -1)) * dxv05n;
      const F2 t1b = fu_p1 * (pair_at(S0, 1) - s0) * dxv05n;
      const F2 t2a = fv_0 * (s0 - ld2(S0 - BX)) * dyv05n;
      const F2 t2b = fv_p1 * (ld2(S0 + BX) - s0) * dyv05n;
      F2 f = (t1a + t1b) + (t2a + t2b);
      const F2 w1a = (fu_m1 + fu_0) * (s0 - ld2(S0 - 2)) * dxv24;
      const F2 w1b = (fu_p1 + fu_p2) * (ld2(S0 + 2) - s0) * dxv24;
      const F2 w2a = (fv_m1 + fv_0) * (s0 - ld2(S0 - 2 * BX)) * dyv24;
      const F2 w2b = (fv_p1 + fv_p2) * (ld2(S0 + 2 * BX) - s0) * dyv24;
      f = fourd3 * f + ((w1a + w1b) + (w2a + w2b));
      const F2 t3a = fw_0 * (s0 - ld2(st(-1) + L::oS + oS)) * dzv05n;
      const F2 t3b = fw_1 * (ld2(st(1) + L::oS + oS) - s0) * dzv05n;
      F2 vadv = t3a + t3b;
      if (a.advopt == 3 && k >= 3 && k <= nk - 3) {   // advs.f90:372-416: 4th order in z
        const float dzv24 = oned24 * a.dziv;
        const F2 fw_m1 = C(C_RST8W, k - 1) * WC(ld2(st(-1) + L::oW + oU), k - 1);
        const F2 fw_2 = C(C_RST8W, k + 2) * WC(ld2(st(2) + L::oW + oU), k + 2);
        const F2 t3w_m = (fw_m1 + fw_0) * (s0 - ld2(st(-2) + L::oS + oS)) * dzv24;
        const F2 t3w_p = (fw_1 + fw_2) * (ld2(st(2) + L::oS + oS) - s0) * dzv24;
        vadv = fourd3 * vadv + (t3w_m + t3w_p);
      }
      f = f + vadv;

      f = f + shr;   // sheartke

      // the TKE at t-dt at an offset (horizontal ones on level k only)
      auto SPo = [&](int dx, int dy, int dz) {
        return dz == 0 ? pair_at(SP0 + dy * BX, dx) : ld2(st(dz) + L::oSP + oS);
      };
      if (smooth) {
        auto A = [&](int dx, int dy, int dz) { return C(C_RBR, k + dz) * SPo(dx, dy, dz); };
        f = smooth_tile(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 2, A);
      }

      f = f - dsp;   // disptke

      // eddyvisj + tkeflx + turbtke: K = rkv/jcb at an offset (horizontal
      // ones on level k only), fluxes h1, h2 of jcb*tkep and h3 of tkep
      auto RK = [&](int dx, int dy, int dz) {
        const F2 r = dz == 0 ? pair_at(st0 + L::oR + oR + dy * BX, dx) : ld2(st(dz) + L::oR + oR);
        return C(C_IJCB, k + dz) * r;
      };
      const float jc = C(C_JCB, k);
      auto JT = [&](int dx, int dy) { return SPo(dx, dy, 0) * jc; };
      auto H1 = [&](int dx) { return (RK(dx - 1, 0, 0) + RK(dx, 0, 0)) * (JT(dx, 0) - JT(dx - 1, 0)) * dxv5; };
      auto H2 = [&](int dy) { return (RK(0, dy - 1, 0) + RK(0, dy, 0)) * (JT(0, dy) - JT(0, dy - 1)) * dyv5; };
      auto H3 = [&](int dz) { return (RK(0, 0, dz - 1) + RK(0, 0, dz)) * (SPo(0, 0, dz) - SPo(0, 0, dz - 1)) * dzv5; };
      const float j8u = C(C_JCB8U, k), j8v = C(C_JCB8V, k);
      f = f + ((H3(1) - H3(0)) * dziv2 + ((j8u * H1(1) - j8u * H1(0)) * dxiv2 + (j8v * H2(1) - j8v * H2(0)) * dyiv2));

      const F2 spv = ld2(SP0);
      if (vsp && k >= a.ksp0 - 1) f = f - (.5f * (C(C_RBCT, k) + C(C_RBCT, k + 1))) * C(C_RST, k) * spv;

      // buoytke with the half diffusivities 0.5 jcb rks of eddydif
      auto R8S = [&](F2 r, int kk) { return (.5f * C(C_JCB, kk)) * r; };
      const F2 b0 = (C(C_JCB8W, k) * nq0) * (R8S(r8m, k - 1) + R8S(r80, k));
      const F2 b1 = (C(C_JCB8W, k + 1) * nq1) * (R8S(r80, k) + R8S(r8p, k + 1));
      f = f - (b0 + b1);

      const F2 sf = fmax2(spv + f * C(D_DTDRST, k), 0.f);
      auto put = [&](long long at) {
        if (ownB) *reinterpret_cast<float2*>(a.tkef + at) = sf.v;
        else a.tkef[at] = sf.v.x;
      };
      put(id);
      if (k == 2) put(id - plane);        // vbcs.f90:118
      if (k == nk - 2) put(id + plane);   // vbcs.f90:132
      r8m = r80;
      r80 = r8p;
      nq0 = nq1;
    }
#pragma unroll
    for (int d = 0; d < 4; ++d) stp[d] = stp[d + 1];
    stp[4] = slot_ptr(k + 3);
  }

  if (__syncthreads_or(fail)) {
    // A bounded wait gave up: record it and let the copies still in flight
    // land (bounded again) so no TMA write outlives the block.
    if (tid == 0) {
      if (a.err) atomicExch(a.err, 1);
      for (int s = 0; s < S; ++s) {
        int kl = -1;
        for (int lv = 1; lv <= issued; ++lv)
          if ((lv - 1) % S == s) kl = lv;
        if (kl >= 0) mbar_wait(&bars[s], ((kl - 1) / S) & 1);
      }
    }
  }
}

}  // namespace

int launch_tke(const TkeArgs& a, const TkeMaps& maps, cudaStream_t st) {
  constexpr int S = 6;
  using L = TkeLayout<S>;
  const Grid& g = a.g;
  if (g.nk < 5) return CRESS_E_UNSUPPORTED;
  const size_t bytes = L::bytes();
  if (cudaFuncSetAttribute(k_tke<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
    return CRESS_E_CUDA;
  const int nx = g.ni - 3, ny = g.nj - 3;
  dim3 block(kTkePairs, kScalarTY, 1);
  dim3 grid((nx + kHeviTX - 1) / kHeviTX, (ny + kScalarTY - 1) / kScalarTY);
  k_tke<S><<<grid, block, bytes, st>>>(maps, a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace cress

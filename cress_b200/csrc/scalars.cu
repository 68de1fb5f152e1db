// Forcing and leapfrog step of the nine moist scalars for sm_100a
// (s_forceqv, s_forceq and their s_steps, cphopt=3):
//   sfrc = advs (advs.f90:205-370, 4th-order horizontal, 2nd-order vertical)
//        + smoo4qv / smoo4s of rbr*(qvp-qvbr) or rbr*sp (smoo4s.f90:184-296)
//        + turbs of sp with the eddy diffusivity (forceqv.f90:331-345,
//          forceq.f90:438-452; tubopt 1 and 2)
//        + vspqv / vsps / vsps0 (vspqv.f90:181-198, vsps.f90:181-198, vsps0.f90:114-124)
//   sf   = sp + sfrc*2dtb/rst, clipped at 0 for the mixing ratios
//          (steps.f90:590-764), then vbcs at k = 1, nk-1 (vbcs.f90:116-132).
//
// Design (2.5-D).  A block owns a 32 x 8 tile of columns of ONE species
// and marches k upward.  For every level 1..nk-1 one elected thread issues
// TMA box loads of the species at t and t-dt (two rows of y halo), u, v, w
// (and the eddy viscosity) into an S-stage shared-memory ring guarded by
// mbarriers.  A level stays in the ring while the march needs it (k-2 ..
// k+2 for the vertical smoothing), so every horizontal neighbour and every
// vertical neighbour is read from shared memory, and HBM sees each input
// once per species (the winds once per tile: the nine species of a tile
// are neighbours in the grid, so their wind boxes are served from L2).
// The terms are formed in the order of the reference expressions.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "common.cuh"
#include "forcing.cuh"
#include "hevi.cuh"
#include "f2.cuh"
#include "stencil.cuh"
#include "tma.cuh"

namespace cress {
namespace {

__host__ __device__ constexpr int r128f(int n) { return (n + 31) / 32 * 32; }  // floats -> multiple of 128 B

// Species per block: the three of a group share the staged winds (and the
// eddy viscosity) and the block's barriers.
constexpr int kScGroup = 3;
static_assert(kMoistN % kScGroup == 0, "species groups must tile the nine species");

template <int S, bool TURB>
struct ScLayout {
  using R = ScalarRows;
  static constexpr int BX = kHeviBoxX;
  static constexpr int sbox = r128f(BX * R::s);
  // species q of the group at oS + q * 2 * sbox (t), + sbox (t-dt)
  static constexpr int oS = 0;
  static constexpr int oSP = sbox;
  static constexpr int oU = kScGroup * 2 * sbox;
  static constexpr int oV = oU + r128f(BX * R::u);
  static constexpr int oW = oV + r128f(BX * R::v);
  static constexpr int oR = oW + r128f(BX * R::w);
  static constexpr int stage = oR + (TURB ? r128f(BX * R::r) : 0);   // floats per ring stage
  static constexpr uint32_t tx_bytes =
      4u * BX * (kScGroup * 2 * R::s + R::u + R::v + R::w + (TURB ? R::r : 0));
  static constexpr int NF = kLevelStride;   // stride of the level table
  // ring, mbarriers, then the level table (rows 0..nk, NF floats each)
  __host__ __device__ static size_t tab_offset() { return 4 * (size_t)S * stage + 16 * (((size_t)S + 1) / 2); }
  __host__ __device__ static size_t bytes(int nk) { return tab_offset() + 4 * (size_t)(nk + 1) * NF; }
};

// Threads: 16 x 8 x 3; thread (tx, ty, tz) owns the pair of columns
// i0+2tx, i0+2tx+1 of row j0+ty of species 3g+tz and computes both with
// packed FP32x2 arithmetic (f2.cuh), so each operation serves two points.
constexpr int kScPairs = kHeviTX / 2;

template <int S, bool TURB>
__global__ void __launch_bounds__(kScPairs * kScalarTY * kScGroup)
k_scalars(const __grid_constant__ MoistMaps m, const MoistScalarArgs a) {
  // level k+2 must have been issued (at k' = k+5-S) before level k waits for it
  static_assert(S >= 6, "ring too shallow for the k-2..k+2 window");
  using L = ScLayout<S, TURB>;
  constexpr int TY = kScalarTY, BX = kHeviBoxX;
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  constexpr int NG = kMoistN / kScGroup;               // species groups
  const int grp = blockIdx.x % NG;                     // the groups of a tile are neighbours
  const int q = threadIdx.z, n = grp * kScGroup + q;   // this thread's species
  const int i0 = 2 + (blockIdx.x / NG) * kHeviTX, j0 = 2 + blockIdx.y * TY;
  const int xb = i0 - 2;                              // box x origin (multiple of 32)
  const int tx = threadIdx.x, ty = threadIdx.y, tid = (q * TY + ty) * kScPairs + tx;
  const int i = i0 + 2 * tx, j = j0 + ty;
  const bool ownA = (i <= ni - 2) && (j <= nj - 2), ownB = (i + 1 <= ni - 2) && (j <= nj - 2);
  // open x: the points in the columns next to the boundaries (i = 2, ni-2)
  const int edge = g.openx ? ((i == 2 || i == ni - 2) ? 1 : 0) | ((i + 1 == 2 || i + 1 == ni - 2) ? 2 : 0) : 0;

  extern __shared__ __align__(1024) float smem[];
  float* ring = smem;
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring + S * L::stage);
  // the level table in shared memory: every per-level constant below is one
  // shared load at a fixed offset from the level's row
  float* tab = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(smem) + L::tab_offset());
  {
    const float4* src = reinterpret_cast<const float4*>(a.lvl);
    float4* dst = reinterpret_cast<float4*>(tab);
    const int nv = (nk + 1) * L::NF / 4, nt = kScPairs * TY * kScGroup;
    for (int v = tid; v < nv; v += nt) dst[v] = __ldg(src + v);
  }
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
    for (int p = 0; p < kScGroup; ++p) {
      tma_load_3d(st + L::oS + p * 2 * L::sbox, &m.s[grp * kScGroup + p], xb, j0 - 2, z, bar);
      tma_load_3d(st + L::oSP + p * 2 * L::sbox, &m.sp[grp * kScGroup + p], xb, j0 - 2, z, bar);
    }
    tma_load_3d(st + L::oU, &m.u, xb, j0, z, bar);
    tma_load_3d(st + L::oV, &m.v, xb, j0 - 1, z, bar);
    tma_load_3d(st + L::oW, &m.w, xb, j0, z, bar);
    if constexpr (TURB) tma_load_3d(st + L::oR, &m.rkv, xb, j0 - 2, z, bar);
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
  const bool smooth = (a.smtopt % 10 == 2) || (a.smtopt % 10 == 3);
  const bool isqv = n == 0;
  const bool vsp = a.vspopt >= 1 && (isqv ? a.vsp_qv : a.vsp_q);
  float* out = a.sf[n];
  // own pair in the boxes (x offset even, so every pair load is 8-byte
  // aligned): species/viscosity rows from j0-2, u and w rows from j0, v
  // rows from j0-1
  const int ox = 2 * tx + 2, oU = ty * BX + ox, oV = (ty + 1) * BX + ox;
  const int oS = q * 2 * L::sbox + (ty + 2) * BX + ox;   // own pair of this species' boxes
  const int oR = (ty + 2) * BX + ox;                     // own pair of the viscosity box
  const long long plane = g.plane;
  long long id = g.at(i, j, 2);
  // stages of levels k-2 .. k+2 (those outside 1..nk-1 hold other levels
  // and are read only by terms the reference's clamping discards)
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
    if ((ownA || ownB) && !fail) {
      const float* ck = tab + k * L::NF;
      auto C = [&](int f, int kk) { return ck[(kk - k) * L::NF + f]; };
      auto st = [&](int d) { return stp[d + 2]; };
      const float* st0 = st(0);
      const float* S0 = st0 + L::oS + oS;
      const float* SP0 = st0 + L::oSP + oS;
      const float* U = st0 + L::oU + oU;
      const float* V = st0 + L::oV + oV;
      // rstuvwc.f90:172-210 fluxes at the faces the stencil touches
      const float r8u = C(C_RST8U, k), r8v = C(C_RST8V, k);
      const F2 fu_m1 = r8u * pair_at(U, -1), fu_0 = r8u * ld2(U);
      const F2 fu_p1 = r8u * pair_at(U, 1), fu_p2 = r8u * ld2(U + 2);
      const F2 fv_m1 = r8v * ld2(V - BX), fv_0 = r8v * ld2(V);
      const F2 fv_p1 = r8v * ld2(V + BX), fv_p2 = r8v * ld2(V + 2 * BX);
      auto WC = [&](F2 w, int kk) { return a.sthopt ? w * C(C_IJCB8W, kk) : w; };
      const F2 fw_0 = C(C_RST8W, k) * WC(ld2(st0 + L::oW + oU), k);
      const F2 fw_1 = C(C_RST8W, k + 1) * WC(ld2(st(1) + L::oW + oU), k + 1);
      const float rbct5 = .5f * (C(C_RBCT, k) + C(C_RBCT, k + 1));
      const float rst = C(C_RST, k);
      const float dtdrst = C(D_DTDRST, k);                                  // steps.f90:528

      // advs.f90:205-370
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
      const F2 f2nd = f;
      f = fourd3 * f + ((w1a + w1b) + (w2a + w2b));
      if (edge) f = sel2(edge, f2nd, f);   // open x: 2nd order in the boundary columns (advs.f90:312-350)
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

      // the species at t-dt at an offset (horizontal ones on level k only)
      auto SPo = [&](int dx, int dy, int dz) {
        return dz == 0 ? pair_at(SP0 + dy * BX, dx) : ld2(st(dz) + L::oSP + oS);
      };
      if (smooth) {
        auto A = [&](int dx, int dy, int dz) {
          const int kk = k + dz;
          const F2 v = SPo(dx, dy, dz);
          return isqv ? C(C_RBR, kk) * (v - C(C_QVBR, kk)) : C(C_RBR, kk) * v;
        };
        f = smooth_tile(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 2, A, edge);
      }
      if constexpr (TURB) {
        auto R = [&](int dx, int dy, int dz) {
          return dz == 0 ? pair_at(st0 + L::oR + oR + dy * BX, dx) : ld2(st(dz) + L::oR + oR);
        };
        f = turb_scalar_at(f, C, k, a.cpriv, a.kdiv, a.dxiv, a.dyiv, a.dziv, R, SPo);
      }
      const F2 spv = ld2(SP0);
      if (vsp && k >= a.ksp0 - 1) f = f - rbct5 * rst * (isqv ? spv - C(C_QVBR, k) : spv);
      F2 sf = spv + f * dtdrst;
      if (n < 6) sf = fmax2(sf, 0.f);
      // the pair's first index is even, so the pair store is 8-byte aligned
      auto put = [&](long long at) {
        if (ownB) *reinterpret_cast<float2*>(out + at) = sf.v;
        else out[at] = sf.v.x;
      };
      put(id);
      if (k == 2) put(id - plane);        // vbcs.f90:118
      if (k == nk - 2) put(id + plane);   // vbcs.f90:132
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

template <int S, bool TURB>
int launch_sc(const MoistScalarArgs& a, const MoistMaps& maps, cudaStream_t st) {
  using L = ScLayout<S, TURB>;
  const Grid& g = a.g;
  const size_t bytes = L::bytes(g.nk);
  if (bytes > 227 * 1024) return CRESS_E_UNSUPPORTED;
  if (cudaFuncSetAttribute(k_scalars<S, TURB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
      cudaSuccess)
    return CRESS_E_CUDA;
  const int nx = g.ni - 3, ny = g.nj - 3;
  dim3 block(kScPairs, kScalarTY, kScGroup);
  dim3 grid((nx + kHeviTX - 1) / kHeviTX * (kMoistN / kScGroup), (ny + kScalarTY - 1) / kScalarTY);
  k_scalars<S, TURB><<<grid, block, bytes, st>>>(maps, a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace

int launch_moist_scalars(const MoistScalarArgs& a, const MoistMaps& maps, cudaStream_t st) {
  if (a.g.nk < 5) return CRESS_E_UNSUPPORTED;
  return a.rkv ? launch_sc<6, true>(a, maps, st) : launch_sc<6, false>(a, maps, st);
}

}  // namespace cress

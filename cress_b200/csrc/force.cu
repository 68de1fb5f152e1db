// Large-step forcing for sm_100a: for every grid point the complete forcing
// of s_forceuvw, s_forcep and s_forcept (advopt=2, smtopt=2/3, vspopt=2,
// coropt=0/1, buyopt=1, gwmopt=0, tubopt=0/1 with isoopt=1, flat terrain)
// and the theta' step of s_steps, with the terms added in the reference's
// order:
//   ufrc/vfrc/wfrc = turbuvw + smoo4uvw + vspuvw + coriuv + buoywb + advuvw
//     (forceuvw.f90:423-626; turbuvw.f90:288-333, 795-840, 1300-1330;
//      smoo4uvw.f90:220-568, vspuvw.f90:230-408, coriuv.f90:124-182,
//      buoywb.f90:162-319, advuvw.f90:209-852)
//   pfrc  = advp + smoo4p (+ vspp)   (forcep.f90:254-311, advp.f90:249-620, smoo4p.f90:178-283)
//   ptfrc = advs + smoo4s + turbs + vsps + advbspt, ptpf = ptpp + ptfrc*2dtb/rst
//     (forcept.f90:313-446, advs.f90:189-370, smoo4s.f90:184-296,
//      vsps.f90:181-198, advbspt.f90:135-172, steps.f90:506-574)
//
// Design (2.5-D).  One block owns a 32 x 8 tile of columns of ONE output
// group (u, v, w, p', theta') and marches k upward.  For every level one
// elected thread issues the TMA boxes of the group's fields (the present
// and past level of its own variable, the advecting winds and, with
// turbulence, the past winds and the eddy viscosity) into an S-stage
// shared-memory ring guarded by mbarriers; a level stays resident while
// the march needs it (k-2 .. k+2 for the vertical smoothing).  Every
// neighbour the stencils touch is then a shared-memory read at a
// compile-time offset.  The five groups of a tile are neighbouring blocks,
// so the winds they all read come from L2 after the first.  The theta'
// and moisture values of the buoyancy are read from global memory on the
// thread's own column, each once.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "common.cuh"
#include "forcing.cuh"
#include "hevi.cuh"
#include "stencil.cuh"
#include "tma.cuh"
#include "turb.cuh"

namespace cress {
namespace {

constexpr int kNF = kLevelStride;   // stride of the k-major level table

__host__ __device__ constexpr int r128c(int n) { return (n + 31) / 32 * 32; }  // floats -> multiple of 128 B

template <int G, bool T>
struct FLayout {
  static constexpr int BX = kHeviBoxX;
  static constexpr int nf = force_nfields(G, T);
  __host__ __device__ static constexpr int off(int q) {
    int o = 0;
    for (int p = 0; p < q; ++p) o += r128c(BX * force_field_rows(G, p));
    return o;
  }
  static constexpr int stage = off(nf);   // floats per ring stage
  __host__ __device__ static constexpr uint32_t tx_bytes() {
    uint32_t b = 0;
    for (int p = 0; p < nf; ++p) b += 4u * BX * force_field_rows(G, p);
    return b;
  }
};

template <bool T>
struct FRing {
  static constexpr int S = T ? 6 : 8;   // levels in the ring (k-2 .. k+2 plus S-5 in flight)
  __host__ __device__ static constexpr int stage_max() {
    int m = 0;
    m = FLayout<0, T>::stage > m ? FLayout<0, T>::stage : m;
    m = FLayout<1, T>::stage > m ? FLayout<1, T>::stage : m;
    m = FLayout<2, T>::stage > m ? FLayout<2, T>::stage : m;
    m = FLayout<3, T>::stage > m ? FLayout<3, T>::stage : m;
    m = FLayout<4, T>::stage > m ? FLayout<4, T>::stage : m;
    return m;
  }
  static size_t bytes(int nk) {
    return 4 * ((size_t)S * stage_max() + (size_t)r128c(kNF * (nk + 1))) + 8 * (size_t)S;
  }
};

// One block of group G: tile (bx, by), march over k.
template <int G, bool T>
__device__ __forceinline__ void force_group(const ForceMaps& m, const ForceArgs& a, float* smem, int bx, int by) {
  using L = FLayout<G, T>;
  constexpr int S = FRing<T>::S, BX = kHeviBoxX, TY = kForceTY, NT = kHeviTX * TY;
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  // u points reach i = ni-1, v points j = nj-1, w points k = nk-1
  const int imax = G == 0 ? ni - 1 : ni - 2, jmax = G == 1 ? nj - 1 : nj - 2;
  const int kmax = G == 2 ? nk - 1 : nk - 2, lmax = G == 2 ? nk : nk - 1;
  const int i0 = 2 + bx * kHeviTX, j0 = 2 + by * TY;
  if (i0 > imax || j0 > jmax) return;   // the whole block: nothing of this group here
  const int xb = i0 - 2;                // box x origin (multiple of 32)
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kHeviTX + tx;
  const int i = i0 + tx, j = j0 + ty;
  const bool own = (i <= imax) && (j <= jmax);
  const int nc = nk + 1;

  float* ring = smem;
  float* cols = ring + S * FRing<T>::stage_max();   // level table: cols[k * kNF + field]
  uint64_t* bars = reinterpret_cast<uint64_t*>(cols + r128c(kNF * nc));
  fill_level_table(cols, a.col, nk, a.dtb2, tid, NT);
  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  // Levels 1..lmax are staged; level lv lives in slot (lv-1) % S.
  auto issue = [&](int lv) {
    const int s = (lv - 1) % S;
    float* st = ring + s * L::stage;
    uint64_t* bar = &bars[s];
    mbar_arrive_expect_tx(bar, L::tx_bytes());
#pragma unroll
    for (int q = 0; q < L::nf; ++q)
      tma_load_3d(st + L::off(q), &m.m[G][q], xb, j0 + force_field_r0(G, q), lv - 1, bar);
  };
  if (tid == 0)
    for (int lv = 1; lv <= min(S, lmax); ++lv) issue(lv);

  bool fail = false;
  auto wait_level = [&](int lv) {
    if (!fail && lv <= lmax) fail = !mbar_wait(&bars[(lv - 1) % S], ((lv - 1) / S) & 1);
  };
  for (int lv = 1; lv <= 3; ++lv) wait_level(lv);

  // own point of field q in its box, and the stages of levels k-2 .. k+2
  // (those outside 1..lmax hold other levels and are read only by terms
  // the reference's clamping discards)
  int ob[L::nf];
#pragma unroll
  for (int q = 0; q < L::nf; ++q) ob[q] = L::off(q) + (ty - force_field_r0(G, q)) * BX + tx + 2;
  auto slot_ptr = [&](int lv) { return ring + ((lv - 1 + S) % S) * L::stage; };
  const float* stp[5] = {slot_ptr(0), slot_ptr(1), slot_ptr(2), slot_ptr(3), slot_ptr(4)};

  const float dxiv = a.dxiv, dyiv = a.dyiv, dziv = a.dziv;
  const float oned24 = 1.f / 24.f, fourd3 = 4.f / 3.f;                  // commath.f90:63,75
  const float dxv25n = -.25f * dxiv, dyv25n = -.25f * dyiv, dzv25n = -.25f * dziv;
  const float dxv24 = oned24 * dxiv, dyv24 = oned24 * dyiv;
  const float dxv48 = .5f * dxv24, dyv48 = .5f * dyv24;
  const float dxv05n = -.5f * dxiv, dyv05n = -.5f * dyiv, dzv05n = -.5f * dziv;
  const bool smooth = (a.smtopt % 10 == 2) || (a.smtopt % 10 == 3);
  const float g05 = .5f * 9.8f;
  const long long plane = g.plane;
  long long id = g.at(i, j, 2);
  float wb_prev = 0.f;   // buoyancy term of the level below (w group)

  for (int k = 2; k <= kmax; ++k, id += plane) {
    wait_level(k + 2);
    // Every thread has finished level k-1, so the slot of level k-3 (last
    // read as k'-2 at k' = k-1) may be refilled with level k+S-3.
    __syncthreads();
    if (tid == 0 && k >= 4 && k + S - 3 <= lmax) {
      fence_proxy_async_smem();
      issue(k + S - 3);
    }
    if (own && !fail) {
      const float* ck = cols + k * kNF;
      auto C = [&](int f, int kk) { return ck[(kk - k) * kNF + f]; };
      auto X = [&](int q, int dx, int dy, int dz) { return stp[dz + 2][ob[q] + dy * BX + dx]; };
      // slots of the present u, v, w in this group's field list
      constexpr int qU = G == 1 ? 1 : (G == 2 ? 1 : (G == 0 ? 0 : 1));
      constexpr int qV = G == 0 ? 1 : (G == 1 ? 0 : 2);
      constexpr int qW = G == 0 ? 2 : (G == 1 ? 2 : (G == 2 ? 0 : 3));
      auto Uc = [&](int dx, int dy, int dz) { return X(qU, dx, dy, dz); };
      auto Vc = [&](int dx, int dy, int dz) { return X(qV, dx, dy, dz); };
      auto Wc = [&](int dx, int dy, int dz) { return X(qW, dx, dy, dz); };
      // flux helpers of rstuvwc.f90:172-210 (wc = w / jcb8w when stretched, phy2cnt.f90:219)
      auto RXU = [&](int dx, int dy, int dz) { return C(C_RST8U, k + dz) * Uc(dx, dy, dz); };
      auto RXV = [&](int dx, int dy, int dz) { return C(C_RST8V, k + dz) * Vc(dx, dy, dz); };
      auto WC = [&](int dx, int dy, int dz) {
        return a.sthopt ? Wc(dx, dy, dz) * C(C_IJCB8W, k + dz) : Wc(dx, dy, dz);
      };
      auto RXW = [&](int dx, int dy, int dz) { return C(C_RST8W, k + dz) * WC(dx, dy, dz); };

      if constexpr (G == 0) {
        // ------------------------------------------------------------ ufrc
        auto UP = [&](int dx, int dy, int dz) { return X(3, dx, dy, dz); };
        float f = 0.f;
        if constexpr (T) {   // s_turbuvw u part (turbuvw.f90:288-333) with the stresses of s_strsten
          auto VP = [&](int dx, int dy, int dz) { return X(4, dx, dy, dz); };
          auto WP = [&](int dx, int dy, int dz) { return X(5, dx, dy, dz); };
          auto RK = [&](int dx, int dy, int dz) { return X(6, dx, dy, dz); };
          const auto D = deform_at(C, UP, VP, WP, k, nk, dxiv, dyiv, dziv);
          const float jc = C(C_JCB, k), j8u = C(C_JCB8U, k);
          auto A = [&](int x) { return jc * (RK(x, 0, 0) * D.s11(x, 0, 0)); };
          auto T12 = [&](int y) {
            return .25f * D.s12(0, y, 0) * ((RK(-1, y - 1, 0) + RK(0, y, 0)) + (RK(-1, y, 0) + RK(0, y - 1, 0)));
          };
          auto Cc = [&](int y) { return (j8u + j8u) * T12(y); };
          auto T13 = [&](int z) {
            return .25f * D.s13(0, 0, z) * ((RK(-1, 0, z - 1) + RK(0, 0, z)) + (RK(-1, 0, z) + RK(0, 0, z - 1)));
          };
          f = ((A(0) - A(-1)) * dxiv + (Cc(1) - Cc(0)) * (.5f * dyiv)) + (T13(1) - T13(0)) * dziv;
        }
        if (smooth) {
          auto A = [&](int dx, int dy, int dz) {
            const int kk = k + dz;
            return C(C_RST8U, kk) * (UP(dx, dy, dz) - C(C_UBR, kk)) * C(D_IJCB8U, kk);
          };
          f = smooth_tile(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 2, A);
        }
        if (a.vspopt >= 1 && a.vsp_u && k >= a.ksp0 - 1) {
          const float r8s = .25f * (C(C_RBCT, k) + C(C_RBCT, k + 1));
          f = f - C(C_RST8U, k) * (r8s + r8s) * (UP(0, 0, 0) - C(C_UBR, k));
        }
        if (a.coropt == 1) {
          const float rst = C(C_RST, k);
          const float c0 = a.fc * rst * (Vc(-1, 0, 0) + Vc(-1, 1, 0));
          const float c1 = a.fc * rst * (Vc(0, 0, 0) + Vc(0, 1, 0));
          f = f + (c0 + c1);
        }
        // advuvw.f90:231-397
        auto t1 = [&](int x) { return (RXU(x, 0, 0) + RXU(x + 1, 0, 0)) * (Uc(x + 1, 0, 0) - Uc(x, 0, 0)) * dxv25n; };
        auto t2 = [&](int y) { return (RXV(-1, y, 0) + RXV(0, y, 0)) * (Uc(0, y, 0) - Uc(0, y - 1, 0)) * dyv25n; };
        auto t3 = [&](int z) { return (RXW(-1, 0, z) + RXW(0, 0, z)) * (Uc(0, 0, z) - Uc(0, 0, z - 1)) * dzv25n; };
        float hadv = (t1(-1) + t1(0)) + (t2(0) + t2(1));
        auto t1w = [&](int x) {
          return (RXU(x - 1, 0, 0) + RXU(x + 1, 0, 0)) * (Uc(x + 1, 0, 0) - Uc(x - 1, 0, 0)) * dxv24;
        };
        auto t2w = [&](int y) {
          return ((RXV(-1, y, 0) + RXV(0, y, 0)) + (RXV(-1, y + 1, 0) + RXV(0, y + 1, 0))) *
                 (Uc(0, y + 1, 0) - Uc(0, y - 1, 0)) * dyv48;
        };
        hadv = fourd3 * hadv + ((t1w(-1) + t1w(1)) + (t2w(-1) + t2w(1)));
        f = f + hadv + (t3(0) + t3(1));
        a.ufrc[id] = f;
      } else if constexpr (G == 1) {
        // ------------------------------------------------------------ vfrc
        auto VP = [&](int dx, int dy, int dz) { return X(3, dx, dy, dz); };
        float f = 0.f;
        if constexpr (T) {   // s_turbuvw v part (turbuvw.f90:795-840)
          auto UP = [&](int dx, int dy, int dz) { return X(4, dx, dy, dz); };
          auto WP = [&](int dx, int dy, int dz) { return X(5, dx, dy, dz); };
          auto RK = [&](int dx, int dy, int dz) { return X(6, dx, dy, dz); };
          const auto D = deform_at(C, UP, VP, WP, k, nk, dxiv, dyiv, dziv);
          const float jc = C(C_JCB, k), j8v = C(C_JCB8V, k);
          auto B = [&](int y) { return jc * (RK(0, y, 0) * D.s22(0, y, 0)); };
          auto T12 = [&](int x) {
            return .25f * D.s12(x, 0, 0) * ((RK(x - 1, -1, 0) + RK(x, 0, 0)) + (RK(x - 1, 0, 0) + RK(x, -1, 0)));
          };
          auto Cc = [&](int x) { return (j8v + j8v) * T12(x); };
          auto T23 = [&](int z) {
            return .25f * D.s23(0, 0, z) * ((RK(0, -1, z - 1) + RK(0, 0, z)) + (RK(0, -1, z) + RK(0, 0, z - 1)));
          };
          f = ((B(0) - B(-1)) * dyiv + (Cc(1) - Cc(0)) * (.5f * dxiv)) + (T23(1) - T23(0)) * dziv;
        }
        if (smooth) {
          auto A = [&](int dx, int dy, int dz) {
            const int kk = k + dz;
            return C(C_RST8V, kk) * (VP(dx, dy, dz) - C(C_VBR, kk)) * C(D_IJCB8V, kk);
          };
          f = smooth_tile(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 2, A);
        }
        if (a.vspopt >= 1 && a.vsp_v && k >= a.ksp0 - 1) {
          const float r8s = .25f * (C(C_RBCT, k) + C(C_RBCT, k + 1));
          f = f - C(C_RST8V, k) * (r8s + r8s) * (VP(0, 0, 0) - C(C_VBR, k));
        }
        if (a.coropt == 1) {
          const float rst = C(C_RST, k);
          const float c0 = -a.fc * rst * (Uc(0, -1, 0) + Uc(1, -1, 0));
          const float c1 = -a.fc * rst * (Uc(0, 0, 0) + Uc(1, 0, 0));
          f = f + (c0 + c1);
        }
        // advuvw.f90:458-624
        auto t1 = [&](int x) { return (RXU(x, -1, 0) + RXU(x, 0, 0)) * (Vc(x, 0, 0) - Vc(x - 1, 0, 0)) * dxv25n; };
        auto t2 = [&](int y) { return (RXV(0, y, 0) + RXV(0, y + 1, 0)) * (Vc(0, y + 1, 0) - Vc(0, y, 0)) * dyv25n; };
        auto t3 = [&](int z) { return (RXW(0, -1, z) + RXW(0, 0, z)) * (Vc(0, 0, z) - Vc(0, 0, z - 1)) * dzv25n; };
        float hadv = (t1(0) + t1(1)) + (t2(-1) + t2(0));
        auto t1w = [&](int x) {
          return ((RXU(x, -1, 0) + RXU(x, 0, 0)) + (RXU(x + 1, -1, 0) + RXU(x + 1, 0, 0))) *
                 (Vc(x + 1, 0, 0) - Vc(x - 1, 0, 0)) * dxv48;
        };
        auto t2w = [&](int y) {
          return (RXV(0, y - 1, 0) + RXV(0, y + 1, 0)) * (Vc(0, y + 1, 0) - Vc(0, y - 1, 0)) * dyv24;
        };
        hadv = fourd3 * hadv + ((t1w(-1) + t1w(1)) + (t2w(-1) + t2w(1)));
        f = f + hadv + (t3(0) + t3(1));
        a.vfrc[id] = f;
      } else if constexpr (G == 2) {
        // ------------------------------------------------------------ wfrc
        auto WP = [&](int dx, int dy, int dz) { return X(3, dx, dy, dz); };
        float f = 0.f;
        if constexpr (T) {   // s_turbuvw w part (turbuvw.f90:1300-1330)
          auto UP = [&](int dx, int dy, int dz) { return X(4, dx, dy, dz); };
          auto VP = [&](int dx, int dy, int dz) { return X(5, dx, dy, dz); };
          auto RK = [&](int dx, int dy, int dz) { return X(6, dx, dy, dz); };
          const auto D = deform_at(C, UP, VP, WP, k, nk, dxiv, dyiv, dziv);
          const float j8u = C(C_JCB8U, k - 1) + C(C_JCB8U, k), j8v = C(C_JCB8V, k - 1) + C(C_JCB8V, k);
          auto T33 = [&](int z) { return RK(0, 0, z) * D.s33(0, 0, z); };
          auto T31 = [&](int x) {
            return .25f * D.s13(x, 0, 0) * ((RK(x - 1, 0, -1) + RK(x, 0, 0)) + (RK(x - 1, 0, 0) + RK(x, 0, -1)));
          };
          auto T32 = [&](int y) {
            return .25f * D.s23(0, y, 0) * ((RK(0, y - 1, -1) + RK(0, y, 0)) + (RK(0, y - 1, 0) + RK(0, y, -1)));
          };
          auto Aw = [&](int x) { return j8u * T31(x); };
          auto Cw = [&](int y) { return j8v * T32(y); };
          f = (T33(0) - T33(-1)) * dziv + ((Aw(1) - Aw(0)) * (.5f * dxiv) + (Cw(1) - Cw(0)) * (.5f * dyiv));
        }
        if (smooth) {
          auto A = [&](int dx, int dy, int dz) {
            const int kk = k + dz;
            return C(C_RST8W, kk) * WP(dx, dy, dz) * C(C_IJCB8W, kk);
          };
          f = smooth_tile(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 1, A);
        }
        if (a.vspopt >= 1 && a.vsp_w && k >= a.ksp0) f = f - C(C_RBCT, k) * C(C_RST8W, k) * WP(0, 0, 0);
        // buoywb.f90:166-172 (dry), 202-299 (moist), 307-313: the term of
        // level k is formed once and reused as the level below of k+1
        float wbk = 0.f;
        if (k <= nk - 2) {
          if (!a.qv) {
            wbk = g05 * C(C_RST, k) * __ldg(a.ptp + id) * C(D_IPTBR, k);
          } else {
            const float qvd = __ldg(a.qv + id) - C(C_QVBR, k);
            const float qall = (((__ldg(a.qc + id) + __ldg(a.qr + id)) + __ldg(a.qi + id)) + __ldg(a.qs + id)) +
                               __ldg(a.qg + id);   // totalqwi.f90:163
            wbk = g05 * C(C_RST, k) *
                  ((qvd * C(D_IEPSQV, k) - (qvd + qall) * C(D_I1QV, k)) + __ldg(a.ptp + id) * C(D_IPTBR, k));
          }
        }
        if (k >= 3 && k <= nk - 2) f = f + (wb_prev + wbk);
        wb_prev = wbk;
        // advuvw.f90:685-852
        auto t1 = [&](int x) { return (RXU(x, 0, -1) + RXU(x, 0, 0)) * (Wc(x, 0, 0) - Wc(x - 1, 0, 0)) * dxv25n; };
        auto t2 = [&](int y) { return (RXV(0, y, -1) + RXV(0, y, 0)) * (Wc(0, y, 0) - Wc(0, y - 1, 0)) * dyv25n; };
        auto t3 = [&](int z) { return (RXW(0, 0, z) + RXW(0, 0, z + 1)) * (Wc(0, 0, z + 1) - Wc(0, 0, z)) * dzv25n; };
        float hadv = (t1(0) + t1(1)) + (t2(0) + t2(1));
        auto t1w = [&](int x) {
          return ((RXU(x, 0, -1) + RXU(x, 0, 0)) + (RXU(x + 1, 0, -1) + RXU(x + 1, 0, 0))) *
                 (Wc(x + 1, 0, 0) - Wc(x - 1, 0, 0)) * dxv48;
        };
        auto t2w = [&](int y) {
          return ((RXV(0, y, -1) + RXV(0, y, 0)) + (RXV(0, y + 1, -1) + RXV(0, y + 1, 0))) *
                 (Wc(0, y + 1, 0) - Wc(0, y - 1, 0)) * dyv48;
        };
        hadv = fourd3 * hadv + ((t1w(-1) + t1w(1)) + (t2w(-1) + t2w(1)));
        f = f + hadv + (t3(-1) + t3(0));
        a.wfrc[id] = f;
      } else {
        // --------------------------------------------- pfrc, theta' step
        // advs-type advection of s with fluxes FU/FV/FW (advs.f90:205-370)
        auto Sc = [&](int dx, int dy, int dz) { return X(0, dx, dy, dz); };
        auto SP = [&](int dx, int dy, int dz) { return X(4, dx, dy, dz); };
        auto adv = [&](auto FU, auto FV, auto FW) {
          auto t1 = [&](int x) { return FU(x) * (Sc(x, 0, 0) - Sc(x - 1, 0, 0)) * dxv05n; };
          auto t2 = [&](int y) { return FV(y) * (Sc(0, y, 0) - Sc(0, y - 1, 0)) * dyv05n; };
          auto t3 = [&](int z) { return FW(z) * (Sc(0, 0, z) - Sc(0, 0, z - 1)) * dzv05n; };
          float sf = (t1(0) + t1(1)) + (t2(0) + t2(1));
          auto t1w = [&](int x) { return (FU(x) + FU(x + 1)) * (Sc(x + 1, 0, 0) - Sc(x - 1, 0, 0)) * dxv24; };
          auto t2w = [&](int y) { return (FV(y) + FV(y + 1)) * (Sc(0, y + 1, 0) - Sc(0, y - 1, 0)) * dyv24; };
          sf = fourd3 * sf + ((t1w(-1) + t1w(1)) + (t2w(-1) + t2w(1)));
          return sf + (t3(0) + t3(1));
        };
        if constexpr (G == 3) {
          // pressure (advp.f90:255-291 J-weighted fluxes)
          auto FU = [&](int x) { return C(C_JCB8U, k) * Uc(x, 0, 0); };
          auto FV = [&](int y) { return C(C_JCB8V, k) * Vc(0, y, 0); };
          auto FW = [&](int z) { return C(C_JCB8W, k + z) * WC(0, 0, z); };
          float f = adv(FU, FV, FW);
          if (smooth) f = smooth_tile(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 2, SP);
          if (a.vspopt >= 1 && a.vsp_p && k >= a.ksp0 - 1)
            f = f - .5f * (C(C_RBCT, k) + C(C_RBCT, k + 1)) * C(C_JCB, k) * SP(0, 0, 0);
          a.pfrc[id] = f;
        } else {
          // theta'
          auto FU = [&](int x) { return RXU(x, 0, 0); };
          auto FV = [&](int y) { return RXV(0, y, 0); };
          auto FW = [&](int z) { return RXW(0, 0, z); };
          float f = adv(FU, FV, FW);
          if (smooth) {
            auto A = [&](int dx, int dy, int dz) { return C(C_RBR, k + dz) * SP(dx, dy, dz); };
            f = smooth_tile(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 2, A);
          }
          if constexpr (T) {   // forcept.f90:313-320, 383-393: mixing of the full theta at t-dt
            auto RK = [&](int dx, int dy, int dz) { return X(5, dx, dy, dz); };
            auto SF = [&](int dx, int dy, int dz) { return C(C_PTBR, k + dz) + SP(dx, dy, dz); };
            f = turb_scalar_at(f, C, k, a.cpriv, dxiv, dyiv, dziv, RK, SF);
          }
          if (a.vspopt >= 1 && a.vsp_pt && k >= a.ksp0 - 1)
            f = f - .5f * (C(C_RBCT, k) + C(C_RBCT, k + 1)) * C(C_RST, k) * SP(0, 0, 0);
          const float dziv25 = .25f * dziv;   // advbspt.f90:135-166
          auto pta8w = [&](int z) {
            const int kk = k + z;
            return (C(C_RBR, kk - 1) + C(C_RBR, kk)) * Wc(0, 0, z) * (C(C_PTBR, kk - 1) - C(C_PTBR, kk)) * dziv25;
          };
          f = f + (pta8w(0) + pta8w(1));
          const float dtdrst = C(D_DTDRST, k);                          // steps.f90:528
          const float ptpf = SP(0, 0, 0) + f * dtdrst;                    // steps.f90:568
          a.ptpf[id] = ptpf;
          if (k == 2) a.ptpf[id - plane] = ptpf;                          // vbcs.f90:118
          if (k == nk - 2) a.ptpf[id + plane] = ptpf;                     // vbcs.f90:132
        }
      }
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
        for (int lv = 1; lv <= lmax; ++lv)
          if ((lv - 1) % S == s) kl = lv;
        if (kl >= 0) mbar_wait(&bars[s], ((kl - 1) / S) & 1);
      }
    }
  }
}

template <bool T>
__global__ void __launch_bounds__(kHeviTX * kForceTY)
k_force(const __grid_constant__ ForceMaps m, const ForceArgs a) {
  extern __shared__ __align__(1024) float fsmem[];
  const int grp = blockIdx.x % kForceGroups;   // the five groups of a tile are neighbours
  const int bx = blockIdx.x / kForceGroups, by = blockIdx.y;
  switch (grp) {
    case 0: force_group<0, T>(m, a, fsmem, bx, by); break;
    case 1: force_group<1, T>(m, a, fsmem, bx, by); break;
    case 2: force_group<2, T>(m, a, fsmem, bx, by); break;
    case 3: force_group<3, T>(m, a, fsmem, bx, by); break;
    default: force_group<4, T>(m, a, fsmem, bx, by); break;
  }
}

template <bool T>
int launch_t(const ForceArgs& a, const ForceMaps& maps, cudaStream_t st) {
  const Grid& g = a.g;
  const size_t bytes = FRing<T>::bytes(g.nk);
  if (bytes > 227 * 1024) return CRESS_E_UNSUPPORTED;
  if (cudaFuncSetAttribute(k_force<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
    return CRESS_E_CUDA;
  // tiles cover i = 2..ni-1 and j = 2..nj-1 (the u and v points)
  const int nx = g.ni - 2, ny = g.nj - 2;
  dim3 block(kHeviTX, kForceTY);
  dim3 grid((nx + kHeviTX - 1) / kHeviTX * kForceGroups, (ny + kForceTY - 1) / kForceTY);
  k_force<T><<<grid, block, bytes, st>>>(maps, a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace

int launch_force(const ForceArgs& a, const ForceMaps& maps, cudaStream_t st) {
  if (a.g.nk < 5) return CRESS_E_UNSUPPORTED;
  return a.rkv ? launch_t<true>(a, maps, st) : launch_t<false>(a, maps, st);
}

}  // namespace cress

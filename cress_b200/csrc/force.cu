// Large-step forcing for sm_100a: for every grid point the complete forcing
// of s_forceuvw, s_forcep and s_forcept (advopt=2/3, smtopt=2/3, vspopt=2,
// coropt=0/1, buyopt=1, gwmopt=0, tubopt=0/1/2 with isoopt=1, flat terrain)
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
// Design (2.5-D).  Two kernels, each over 32 x 8 tiles of columns marching
// k upward: the momentum kernel computes the u, v and w groups of a tile
// in one block (threadIdx.z = group), the scalar kernel the p' and theta'
// groups.  For every level one elected thread issues the TMA boxes of the
// kernel's fields (forcing.cuh: the present and past levels of its
// variables, the winds and, with turbulence, the eddy viscosity) into an
// S-stage shared-memory ring guarded by mbarriers, shared by the groups of
// the block; a level stays resident while the march needs it (k-2 .. k+2
// for the vertical smoothing).  Every neighbour the stencils touch is then
// a shared-memory read at a compile-time offset.  Each thread owns a pair
// of x-neighbouring columns and computes both with packed FP32x2
// arithmetic (f2.cuh).  The theta' and moisture values of the buoyancy are
// read from global memory on the thread's own columns, each once.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "common.cuh"
#include "f2.cuh"
#include "forcing.cuh"
#include "hevi.cuh"
#include "stencil.cuh"
#include "tma.cuh"
#include "turb.cuh"

namespace cress {
namespace {

constexpr int kNF = kLevelStride;   // stride of the k-major level table
constexpr int kFPairs = kHeviTX / 2;   // threads per tile row (two columns each)

__host__ __device__ constexpr int r128c(int n) { return (n + 31) / 32 * 32; }  // floats -> multiple of 128 B

// Ring layout of kernel SG (0 momentum, 1 scalar).
template <int SG, bool T>
struct FLayout {
  static constexpr int BX = kHeviBoxX;
  static constexpr int nf = force_nslots(SG, T);
  static constexpr int ngroups = SG == 0 ? 3 : 2;
  static constexpr int S = 6;   // levels in the ring: k-2 .. k+2 and one in flight
  __host__ __device__ static constexpr int off(int s) {
    int o = 0;
    for (int p = 0; p < s; ++p) o += r128c(BX * force_slot_rows(SG, p));
    return o;
  }
  static constexpr int stage = off(nf);   // floats per ring stage
  __host__ __device__ static constexpr uint32_t tx_bytes() {
    uint32_t b = 0;
    for (int p = 0; p < nf; ++p) b += 4u * BX * force_slot_rows(SG, p);
    return b;
  }
  // ring, mbarriers, then the level table (rows 0..nk, kNF floats each)
  __host__ __device__ static size_t tab_offset() { return 4 * (size_t)S * stage + 16 * (((size_t)S + 1) / 2); }
  static size_t bytes(int nk) { return tab_offset() + 4 * (size_t)(nk + 1) * kNF; }
};

// Slot of group G's field q.  Field numbering per group: u: u, v, w, up,
// vp, wp, rkv; v: v, u, w, vp, up, wp, rkv; w: w, u, v, wp, up, vp, rkv;
// p': pp, u, v, w, ppp; theta': ptp, u, v, w, ptpp, rkv.
__host__ __device__ constexpr int force_slot(int G, int q) {
  return G == 0 ? q
       : G == 1 ? (q == 0 ? 1 : q == 1 ? 0 : q == 3 ? 4 : q == 4 ? 3 : q)
       : G == 2 ? (q == 0 ? 2 : q == 1 ? 0 : q == 2 ? 1 : q == 3 ? 5 : q == 4 ? 3 : q == 5 ? 4 : q)
       : G == 3 ? (q == 0 ? 0 : q == 1 ? 4 : q == 2 ? 5 : q == 3 ? 6 : 2)
                : (q == 0 ? 1 : q == 1 ? 4 : q == 2 ? 5 : q == 3 ? 6 : q == 4 ? 3 : 7);
}

// F2 of two consecutive floats of a global field (8-byte aligned index).
__device__ __forceinline__ F2 gld2(const float* p) { return F2{__ldg(reinterpret_cast<const float2*>(p))}; }

// The forcing of group G (0 u, 1 v, 2 w, 3 p', 4 theta') at the thread's
// pair of columns, level k.  stp[d + 2] is the ring stage of level k + d,
// rowbase the thread's own row and first column in a box, id the global
// index of the pair's first point (even), ownB whether the second point is
// owned too, wb_prev the w group's buoyancy term of the level below,
// edge the points (bit 0 first, bit 1 second) in an open-x boundary
// column, where advection and smoothing keep their 2nd-order form
// (advuvw.f90:340-430, advs.f90:312-350, advp.f90:562-600, smoo4*: the
// 4th-order loops start at i = 2+iwest).
template <int G, bool T>
__device__ __forceinline__ void force_point(const ForceArgs& a, const float* tab, const float* const* stp,
                                            int rowbase, long long id, int k, bool ownB, F2& wb_prev, int edge) {
  constexpr int SG = G <= 2 ? 0 : 1;
  using L = FLayout<SG, T>;
  constexpr int BX = kHeviBoxX;
  const int nk = a.g.nk;
  const long long plane = a.g.plane;
  const float dxiv = a.dxiv, dyiv = a.dyiv, dziv = a.dziv;
  const float oned24 = 1.f / 24.f, fourd3 = 4.f / 3.f;                  // commath.f90:63,75
  const float dxv25n = -.25f * dxiv, dyv25n = -.25f * dyiv, dzv25n = -.25f * dziv;
  const float dxv24 = oned24 * dxiv, dyv24 = oned24 * dyiv;
  const float dxv48 = .5f * dxv24, dyv48 = .5f * dyv24;
  const float dzv24 = oned24 * dziv, dzv48 = .5f * dzv24;
  const float dxv05n = -.5f * dxiv, dyv05n = -.5f * dyiv, dzv05n = -.5f * dziv;
  const bool smooth = (a.smtopt % 10 == 2) || (a.smtopt % 10 == 3);
  // advopt=3: 4th-order vertical advection on the levels 3..nk-3 (w: 3..nk-2)
  const bool adv3 = a.advopt == 3 && k >= 3 && k <= (G == 2 ? nk - 2 : nk - 3);
  const float g05 = .5f * 9.8f;
  const float* ck = tab + k * kNF;   // the level table in shared memory
  auto C = [&](int f, int kk) { return ck[(kk - k) * kNF + f]; };
  // field q of this group at the offset (dx, dy, dz), both points
  auto X = [&](int q, int dx, int dy, int dz) {
    const int s = force_slot(G, q);
    return pair_at(stp[dz + 2] + L::off(s) - force_slot_r0(SG, s) * BX + rowbase + dy * BX, dx);
  };
  // the pair's result: one 8-byte store, or the first point alone
  auto put = [&](float* out, long long at, F2 v) {
    if (ownB) *reinterpret_cast<float2*>(out + at) = v.v;
    else out[at] = v.v.x;
  };
  // present u, v, w (fields 0-2 of the momentum groups in their own order,
  // fields 1-3 of the scalar groups)
  constexpr int qU = G == 0 ? 0 : 1;
  constexpr int qV = G == 0 ? 1 : (G == 1 ? 0 : 2);
  constexpr int qW = G <= 1 ? 2 : (G == 2 ? 0 : 3);
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
    F2 f = f2(0.f);
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
      f = smooth_tile(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 2, A, edge);
    }
    if (a.vspopt >= 1 && a.vsp_u && k >= a.ksp0 - 1) {
      const float r8s = .25f * (C(C_RBCT, k) + C(C_RBCT, k + 1));
      f = f - C(C_RST8U, k) * (r8s + r8s) * (UP(0, 0, 0) - C(C_UBR, k));
    }
    if (a.coropt == 1) {
      const float rst = C(C_RST, k);
      const F2 c0 = a.fc * rst * (Vc(-1, 0, 0) + Vc(-1, 1, 0));
      const F2 c1 = a.fc * rst * (Vc(0, 0, 0) + Vc(0, 1, 0));
      f = f + (c0 + c1);
    }
    // advuvw.f90:231-397
    auto t1 = [&](int x) { return (RXU(x, 0, 0) + RXU(x + 1, 0, 0)) * (Uc(x + 1, 0, 0) - Uc(x, 0, 0)) * dxv25n; };
    auto t2 = [&](int y) { return (RXV(-1, y, 0) + RXV(0, y, 0)) * (Uc(0, y, 0) - Uc(0, y - 1, 0)) * dyv25n; };
    auto t3 = [&](int z) { return (RXW(-1, 0, z) + RXW(0, 0, z)) * (Uc(0, 0, z) - Uc(0, 0, z - 1)) * dzv25n; };
    F2 hadv = (t1(-1) + t1(0)) + (t2(0) + t2(1));
    auto t1w = [&](int x) {
      return (RXU(x - 1, 0, 0) + RXU(x + 1, 0, 0)) * (Uc(x + 1, 0, 0) - Uc(x - 1, 0, 0)) * dxv24;
    };
    auto t2w = [&](int y) {
      return ((RXV(-1, y, 0) + RXV(0, y, 0)) + (RXV(-1, y + 1, 0) + RXV(0, y + 1, 0))) *
             (Uc(0, y + 1, 0) - Uc(0, y - 1, 0)) * dyv48;
    };
    const F2 h2 = hadv;
    hadv = fourd3 * hadv + ((t1w(-1) + t1w(1)) + (t2w(-1) + t2w(1)));
    if (edge) hadv = sel2(edge, h2, hadv);
    F2 vadv = t3(0) + t3(1);
    if (adv3) {   // advuvw.f90:399-430
      auto t3w = [&](int z) {
        return ((RXW(-1, 0, z) + RXW(0, 0, z)) + (RXW(-1, 0, z + 1) + RXW(0, 0, z + 1))) *
               (Uc(0, 0, z + 1) - Uc(0, 0, z - 1)) * dzv48;
      };
      vadv = fourd3 * vadv + (t3w(-1) + t3w(1));
    }
    f = f + hadv + vadv;
    put(a.ufrc, id, f);
  } else if constexpr (G == 1) {
    // ------------------------------------------------------------ vfrc
    auto VP = [&](int dx, int dy, int dz) { return X(3, dx, dy, dz); };
    F2 f = f2(0.f);
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
      f = smooth_tile(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 2, A, edge);
    }
    if (a.vspopt >= 1 && a.vsp_v && k >= a.ksp0 - 1) {
      const float r8s = .25f * (C(C_RBCT, k) + C(C_RBCT, k + 1));
      f = f - C(C_RST8V, k) * (r8s + r8s) * (VP(0, 0, 0) - C(C_VBR, k));
    }
    if (a.coropt == 1) {
      const float rst = C(C_RST, k);
      const F2 c0 = -a.fc * rst * (Uc(0, -1, 0) + Uc(1, -1, 0));
      const F2 c1 = -a.fc * rst * (Uc(0, 0, 0) + Uc(1, 0, 0));
      f = f + (c0 + c1);
    }
    // advuvw.f90:458-624
    auto t1 = [&](int x) { return (RXU(x, -1, 0) + RXU(x, 0, 0)) * (Vc(x, 0, 0) - Vc(x - 1, 0, 0)) * dxv25n; };
    auto t2 = [&](int y) { return (RXV(0, y, 0) + RXV(0, y + 1, 0)) * (Vc(0, y + 1, 0) - Vc(0, y, 0)) * dyv25n; };
    auto t3 = [&](int z) { return (RXW(0, -1, z) + RXW(0, 0, z)) * (Vc(0, 0, z) - Vc(0, 0, z - 1)) * dzv25n; };
    F2 hadv = (t1(0) + t1(1)) + (t2(-1) + t2(0));
    auto t1w = [&](int x) {
      return ((RXU(x, -1, 0) + RXU(x, 0, 0)) + (RXU(x + 1, -1, 0) + RXU(x + 1, 0, 0))) *
             (Vc(x + 1, 0, 0) - Vc(x - 1, 0, 0)) * dxv48;
    };
    auto t2w = [&](int y) {
      return (RXV(0, y - 1, 0) + RXV(0, y + 1, 0)) * (Vc(0, y + 1, 0) - Vc(0, y - 1, 0)) * dyv24;
    };
    const F2 h2 = hadv;
    hadv = fourd3 * hadv + ((t1w(-1) + t1w(1)) + (t2w(-1) + t2w(1)));
    if (edge) hadv = sel2(edge, h2, hadv);
    F2 vadv = t3(0) + t3(1);
    if (adv3) {   // advuvw.f90:626-657
      auto t3w = [&](int z) {
        return ((RXW(0, -1, z) + RXW(0, 0, z)) + (RXW(0, -1, z + 1) + RXW(0, 0, z + 1))) *
               (Vc(0, 0, z + 1) - Vc(0, 0, z - 1)) * dzv48;
      };
      vadv = fourd3 * vadv + (t3w(-1) + t3w(1));
    }
    f = f + hadv + vadv;
    put(a.vfrc, id, f);
  } else if constexpr (G == 2) {
    // ------------------------------------------------------------ wfrc
    auto WP = [&](int dx, int dy, int dz) { return X(3, dx, dy, dz); };
    F2 f = f2(0.f);
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
      f = smooth_tile(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 1, A, edge);
    }
    if (a.vspopt >= 1 && a.vsp_w && k >= a.ksp0) f = f - C(C_RBCT, k) * C(C_RST8W, k) * WP(0, 0, 0);
    // buoywb.f90:166-172 (dry), 202-299 (moist), 307-313: the term of
    // level k is formed once and reused as the level below of k+1
    F2 wbk = f2(0.f);
    if (k <= nk - 2) {
      if (!a.qv) {
        wbk = g05 * C(C_RST, k) * gld2(a.ptp + id) * C(D_IPTBR, k);
      } else {
        const F2 qvd = gld2(a.qv + id) - C(C_QVBR, k);
        const F2 qall = (((gld2(a.qc + id) + gld2(a.qr + id)) + gld2(a.qi + id)) + gld2(a.qs + id)) +
                        gld2(a.qg + id);   // totalqwi.f90:163
        wbk = g05 * C(C_RST, k) *
              ((qvd * C(D_IEPSQV, k) - (qvd + qall) * C(D_I1QV, k)) + gld2(a.ptp + id) * C(D_IPTBR, k));
      }
    }
    if (k >= 3 && k <= nk - 2) f = f + (wb_prev + wbk);
    wb_prev = wbk;
    // advuvw.f90:685-852
    auto t1 = [&](int x) { return (RXU(x, 0, -1) + RXU(x, 0, 0)) * (Wc(x, 0, 0) - Wc(x - 1, 0, 0)) * dxv25n; };
    auto t2 = [&](int y) { return (RXV(0, y, -1) + RXV(0, y, 0)) * (Wc(0, y, 0) - Wc(0, y - 1, 0)) * dyv25n; };
    auto t3 = [&](int z) { return (RXW(0, 0, z) + RXW(0, 0, z + 1)) * (Wc(0, 0, z + 1) - Wc(0, 0, z)) * dzv25n; };
    F2 hadv = (t1(0) + t1(1)) + (t2(0) + t2(1));
    auto t1w = [&](int x) {
      return ((RXU(x, 0, -1) + RXU(x, 0, 0)) + (RXU(x + 1, 0, -1) + RXU(x + 1, 0, 0))) *
             (Wc(x + 1, 0, 0) - Wc(x - 1, 0, 0)) * dxv48;
    };
    auto t2w = [&](int y) {
      return ((RXV(0, y, -1) + RXV(0, y, 0)) + (RXV(0, y + 1, -1) + RXV(0, y + 1, 0))) *
             (Wc(0, y + 1, 0) - Wc(0, y - 1, 0)) * dyv48;
    };
    const F2 h2 = hadv;
    hadv = fourd3 * hadv + ((t1w(-1) + t1w(1)) + (t2w(-1) + t2w(1)));
    if (edge) hadv = sel2(edge, h2, hadv);
    F2 vadv = t3(-1) + t3(0);
    if (adv3) {   // advuvw.f90:854-884
      auto t3w = [&](int z) {
        return (RXW(0, 0, z - 1) + RXW(0, 0, z + 1)) * (Wc(0, 0, z + 1) - Wc(0, 0, z - 1)) * dzv24;
      };
      vadv = fourd3 * vadv + (t3w(-1) + t3w(1));
    }
    f = f + hadv + vadv;
    put(a.wfrc, id, f);
  } else {
    // --------------------------------------------- pfrc, theta' step
    // advs-type advection of s with fluxes FU/FV/FW (advs.f90:205-370)
    auto Sc = [&](int dx, int dy, int dz) { return X(0, dx, dy, dz); };
    auto SP = [&](int dx, int dy, int dz) { return X(4, dx, dy, dz); };
    auto adv = [&](auto FU, auto FV, auto FW) {
      auto t1 = [&](int x) { return FU(x) * (Sc(x, 0, 0) - Sc(x - 1, 0, 0)) * dxv05n; };
      auto t2 = [&](int y) { return FV(y) * (Sc(0, y, 0) - Sc(0, y - 1, 0)) * dyv05n; };
      auto t3 = [&](int z) { return FW(z) * (Sc(0, 0, z) - Sc(0, 0, z - 1)) * dzv05n; };
      F2 sf = (t1(0) + t1(1)) + (t2(0) + t2(1));
      auto t1w = [&](int x) { return (FU(x) + FU(x + 1)) * (Sc(x + 1, 0, 0) - Sc(x - 1, 0, 0)) * dxv24; };
      auto t2w = [&](int y) { return (FV(y) + FV(y + 1)) * (Sc(0, y + 1, 0) - Sc(0, y - 1, 0)) * dyv24; };
      const F2 s2 = sf;
      sf = fourd3 * sf + ((t1w(-1) + t1w(1)) + (t2w(-1) + t2w(1)));
      if (edge) sf = sel2(edge, s2, sf);
      F2 vadv = t3(0) + t3(1);
      if (adv3) {   // advs.f90:372-416, advp.f90:627-655
        auto t3w = [&](int z) { return (FW(z) + FW(z + 1)) * (Sc(0, 0, z + 1) - Sc(0, 0, z - 1)) * dzv24; };
        vadv = fourd3 * vadv + (t3w(-1) + t3w(1));
      }
      return sf + vadv;
    };
    if constexpr (G == 3) {
      // pressure (advp.f90:255-291 J-weighted fluxes)
      auto FU = [&](int x) { return C(C_JCB8U, k) * Uc(x, 0, 0); };
      auto FV = [&](int y) { return C(C_JCB8V, k) * Vc(0, y, 0); };
      auto FW = [&](int z) { return C(C_JCB8W, k + z) * WC(0, 0, z); };
      F2 f = adv(FU, FV, FW);
      if (smooth) f = smooth_tile(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 2, SP, edge);
      if (a.vspopt >= 1 && a.vsp_p && k >= a.ksp0 - 1)
        f = f - .5f * (C(C_RBCT, k) + C(C_RBCT, k + 1)) * C(C_JCB, k) * SP(0, 0, 0);
      put(a.pfrc, id, f);
    } else {
      // theta'
      auto FU = [&](int x) { return RXU(x, 0, 0); };
      auto FV = [&](int y) { return RXV(0, y, 0); };
      auto FW = [&](int z) { return RXW(0, 0, z); };
      F2 f = adv(FU, FV, FW);
      if (smooth) {
        auto A = [&](int dx, int dy, int dz) { return C(C_RBR, k + dz) * SP(dx, dy, dz); };
        f = smooth_tile(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 2, A, edge);
      }
      if constexpr (T) {   // forcept.f90:313-320, 383-393: mixing of the full theta at t-dt
        auto RK = [&](int dx, int dy, int dz) { return X(5, dx, dy, dz); };
        auto SF = [&](int dx, int dy, int dz) { return C(C_PTBR, k + dz) + SP(dx, dy, dz); };
        f = turb_scalar_at(f, C, k, a.cpriv, a.kdiv, dxiv, dyiv, dziv, RK, SF);
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
      const F2 ptpf = SP(0, 0, 0) + f * dtdrst;                    // steps.f90:568
      put(a.ptpf, id, ptpf);
      if (k == 2) put(a.ptpf, id - plane, ptpf);                      // vbcs.f90:118
      if (k == nk - 2) put(a.ptpf, id + plane, ptpf);                 // vbcs.f90:132
    }
  }
}

template <int SG, bool T>
__global__ void __launch_bounds__(kFPairs * kForceTY * (SG == 0 ? 3 : 2))
k_force(const __grid_constant__ ForceMaps m, const ForceArgs a) {
  using L = FLayout<SG, T>;
  constexpr int S = L::S, BX = kHeviBoxX, TY = kForceTY;
  // level k+2 must have been issued (at k' = k+5-S) before level k waits for it
  static_assert(S >= 6, "ring too shallow for the k-2..k+2 window");
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const int gz = threadIdx.z;                       // group within the kernel
  const int G = (SG == 0 ? 0 : 3) + gz;
  const int i0 = 2 + blockIdx.x * kHeviTX, j0 = 2 + blockIdx.y * TY;
  // u points reach i = ni-1 and v points j = nj-1 (momentum kernel only)
  if (i0 > (SG == 0 ? ni - 1 : ni - 2) || j0 > (SG == 0 ? nj - 1 : nj - 2)) return;
  const int xb = i0 - 2;                            // box x origin (multiple of 32)
  const int tx = threadIdx.x, ty = threadIdx.y, tid = (gz * TY + ty) * kFPairs + tx;
  const int i = i0 + 2 * tx, j = j0 + ty;
  const int imaxg = G == 0 ? ni - 1 : ni - 2, jmaxg = G == 1 ? nj - 1 : nj - 2, kmaxg = G == 2 ? nk - 1 : nk - 2;
  const bool ownA = (i <= imaxg) && (j <= jmaxg), ownB = (i + 1 <= imaxg) && (j <= jmaxg);
  // open x: the points in the columns next to the boundaries (u: i = 2 and
  // ni-1, the other groups: i = 2 and ni-2)
  const int elast = G == 0 ? ni - 1 : ni - 2;
  const int edge = g.openx ? ((i == 2 || i == elast) ? 1 : 0) | ((i + 1 == 2 || i + 1 == elast) ? 2 : 0) : 0;
  const int kmax = SG == 0 ? nk - 1 : nk - 2, lmax = SG == 0 ? nk : nk - 1;

  extern __shared__ __align__(1024) float fsmem[];
  float* ring = fsmem;
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring + S * L::stage);
  // the level table in shared memory (one shared load per constant)
  float* tab = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(fsmem) + L::tab_offset());
  {
    const float4* src = reinterpret_cast<const float4*>(a.lvl);
    float4* dst = reinterpret_cast<float4*>(tab);
    const int nv = (nk + 1) * kNF / 4, nt = kFPairs * TY * L::ngroups;
    for (int v = tid; v < nv; v += nt) dst[v] = __ldg(src + v);
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  // Levels 1..lmax are staged; level lv lives in slot (lv-1) % S.
  int issued = 0;   // highest level thread 0 has issued
  auto issue = [&](int lv) {
    issued = lv;
    const int s = (lv - 1) % S;
    float* st = ring + s * L::stage;
    uint64_t* bar = &bars[s];
    mbar_arrive_expect_tx(bar, L::tx_bytes());
#pragma unroll
    for (int q = 0; q < L::nf; ++q)
      tma_load_3d(st + L::off(q), &m.m[SG][q], xb, j0 + force_slot_r0(SG, q), lv - 1, bar);
  };
  if (tid == 0)
    for (int lv = 1; lv <= min(S, lmax); ++lv) issue(lv);

  bool fail = false;
  auto wait_level = [&](int lv) {
    if (!fail && lv <= lmax) fail = !mbar_wait(&bars[(lv - 1) % S], ((lv - 1) / S) & 1);
  };
  for (int lv = 1; lv <= 3; ++lv) wait_level(lv);

  // stages of levels k-2 .. k+2 (those outside 1..lmax hold other levels
  // and are read only by terms the reference's clamping discards)
  auto slot_ptr = [&](int lv) { return ring + ((lv - 1 + S) % S) * L::stage; };
  const float* stp[5] = {slot_ptr(0), slot_ptr(1), slot_ptr(2), slot_ptr(3), slot_ptr(4)};
  const int rowbase = ty * BX + 2 * tx + 2;         // even: every pair load is 8-byte aligned
  const long long plane = g.plane;
  long long id = g.at(i, j, 2);
  F2 wb_prev = f2(0.f);

  for (int k = 2; k <= kmax; ++k, id += plane) {
    wait_level(k + 2);
    // Every thread has finished level k-1, so the slot of level k-3 (last
    // read as k'-2 at k' = k-1) may be refilled with level k+S-3.
    __syncthreads();
    if (tid == 0 && !fail && k >= 4 && k + S - 3 <= lmax) {   // refill only after its copy was seen to land
      fence_proxy_async_smem();
      issue(k + S - 3);
    }
    if ((ownA || ownB) && !fail && k <= kmaxg) {
      if constexpr (SG == 0) {
        if (gz == 0) force_point<0, T>(a, tab, stp, rowbase, id, k, ownB, wb_prev, edge);
        else if (gz == 1) force_point<1, T>(a, tab, stp, rowbase, id, k, ownB, wb_prev, edge);
        else force_point<2, T>(a, tab, stp, rowbase, id, k, ownB, wb_prev, edge);
      } else {
        if (gz == 0) force_point<3, T>(a, tab, stp, rowbase, id, k, ownB, wb_prev, edge);
        else force_point<4, T>(a, tab, stp, rowbase, id, k, ownB, wb_prev, edge);
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
        for (int lv = 1; lv <= issued; ++lv)
          if ((lv - 1) % S == s) kl = lv;
        if (kl >= 0) mbar_wait(&bars[s], ((kl - 1) / S) & 1);
      }
    }
  }
}

template <int SG, bool T>
int launch_sg(const ForceArgs& a, const ForceMaps& maps, cudaStream_t st) {
  using L = FLayout<SG, T>;
  const Grid& g = a.g;
  const size_t bytes = L::bytes(g.nk);
  if (bytes > 227 * 1024) return CRESS_E_UNSUPPORTED;
  if (cudaFuncSetAttribute(k_force<SG, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
    return CRESS_E_CUDA;
  // momentum tiles cover i = 2..ni-1 and j = 2..nj-1 (the u and v points),
  // scalar tiles the interior
  const int nx = SG == 0 ? g.ni - 2 : g.ni - 3, ny = SG == 0 ? g.nj - 2 : g.nj - 3;
  dim3 block(kFPairs, kForceTY, L::ngroups);
  dim3 grid((nx + kHeviTX - 1) / kHeviTX, (ny + kForceTY - 1) / kForceTY);
  k_force<SG, T><<<grid, block, bytes, st>>>(maps, a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace

int launch_force(const ForceArgs& a, const ForceMaps& maps, cudaStream_t st) {
  if (a.g.nk < 5) return CRESS_E_UNSUPPORTED;
  int rc = a.rkv ? launch_sg<0, true>(a, maps, st) : launch_sg<0, false>(a, maps, st);
  if (rc) return rc;
  return a.rkv ? launch_sg<1, true>(a, maps, st) : launch_sg<1, false>(a, maps, st);
}

}  // namespace cress

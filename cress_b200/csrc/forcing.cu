// Large-step kernels for sm_100a: momentum / pressure / theta' forcing, the
// leapfrog theta' update, the Asselin filter and the periodic ghost planes.
//
// k_force computes, for every grid point it owns, the complete forcing of
// s_forceuvw, s_forcep and s_forcept (tubopt=0, advopt=2, smtopt=2/3,
// vspopt=2, coropt=0/1, buyopt=1, gwmopt=0, flat terrain) and the theta'
// step of s_steps, with the terms added in the reference's order:
//   ufrc/vfrc/wfrc = smoo4uvw + vspuvw + coriuv + buoywb + advuvw
//     (forceuvw.f90:423-626; smoo4uvw.f90:220-568, vspuvw.f90:230-408,
//      coriuv.f90:124-182, buoywb.f90:162-319, advuvw.f90:209-852)
//   pfrc = advp + smoo4p (+ vspp)   (forcep.f90:254-311, advp.f90:249-620, smoo4p.f90:178-283)
//   ptfrc = advs + smoo4s + vsps + advbspt, ptpf = ptpp + ptfrc*2dtb/rst
//     (forcept.f90:344-446, advs.f90:189-370, smoo4s.f90:184-296,
//      vsps.f90:181-198, advbspt.f90:135-172, steps.f90:506-574)
// Each point recomputes the intermediate fluxes of its neighbours from the
// inputs (served by L1/L2) instead of writing the reference's temporary
// arrays, so the only HBM traffic is one read of the inputs and one write
// of the outputs.
#include <cuda_runtime.h>
#include "common.cuh"
#include "forcing.cuh"
#include "hevi.cuh"
#include "stencil.cuh"
#include "turb.cuh"

namespace cress {
namespace {

constexpr float kEpsva = .622f;   // rd/rv, comphy.f90:79

__device__ __forceinline__ float ld(const float* f, long long idx) { return __ldg(f + idx); }

// blockIdx.z runs over k = 2..nk-1 within one output group, then over the
// groups (0: ufrc, 1: vfrc, 2: wfrc, 3: pfrc and theta'), so the four
// stencils of a point run in different threads.
__global__ void __launch_bounds__(256) k_force(const ForceArgs a) {
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int grp = blockIdx.z / (nk - 2);
  const int k = 2 + blockIdx.z % (nk - 2);
  if (i > ni - 1 || j > nj - 1 || grp > 3) return;
  const long long px = g.px, pl = g.plane;
  const long long id = g.at(i, j, k);
  const int nc = nk + 1;
  const float* col = a.col;
  auto C = [&](int f, int kk) { return __ldg(col + f * nc + kk); };
  const float dxiv = a.dxiv, dyiv = a.dyiv, dziv = a.dziv;
  const float oned24 = 1.f / 24.f, fourd3 = 4.f / 3.f;                  // commath.f90:63,75
  const float dxv25n = -.25f * dxiv, dyv25n = -.25f * dyiv, dzv25n = -.25f * dziv;
  const float dxv24 = oned24 * dxiv, dyv24 = oned24 * dyiv;
  const float dxv48 = .5f * dxv24, dyv48 = .5f * dyv24;
  const float dxv05n = -.5f * dxiv, dyv05n = -.5f * dyiv, dzv05n = -.5f * dziv;
  const bool smooth = (a.smtopt % 10 == 2) || (a.smtopt % 10 == 3);
  const float g05 = .5f * 9.8f;
  // flux helpers of rstuvwc.f90:172-210 (wc = w / jcb8w when stretched, phy2cnt.f90:219)
  auto RXU = [&](long long p, int kk) { return C(C_RST8U, kk) * ld(a.u, p); };
  auto RXV = [&](long long p, int kk) { return C(C_RST8V, kk) * ld(a.v, p); };
  auto WC = [&](long long p, int kk) { return a.sthopt ? ld(a.w, p) / C(C_JCB8W, kk) : ld(a.w, p); };
  auto RXW = [&](long long p, int kk) { return C(C_RST8W, kk) * WC(p, kk); };

  // ---------------------------------------------------------------- ufrc
  const Deform D{col, nc, nk, a.up, a.vp, a.wp, px, pl, dxiv, dyiv, dziv};
  auto RKV = [&](long long p) { return __ldg(a.rkv + p); };
  if (grp == 0 && j <= nj - 2 && k <= nk - 2) {
    float f = 0.f;
    if (a.rkv) {   // s_turbuvw u part (turbuvw.f90:288-333) with the stresses of s_strsten
      const float jc = C(C_JCB, k), j8u = C(C_JCB8U, k);
      auto A = [&](long long p) { return jc * (RKV(p) * D.s11(p, k)); };
      auto T12 = [&](long long p) {
        return .25f * D.s12(p, k) * ((RKV(p - 1 - px) + RKV(p)) + (RKV(p - 1) + RKV(p - px)));
      };
      auto Cc = [&](long long p) { return (j8u + j8u) * T12(p); };
      auto T13 = [&](long long p, int kk) {
        return .25f * D.s13(p, kk) * ((RKV(p - 1 - pl) + RKV(p)) + (RKV(p - 1) + RKV(p - pl)));
      };
      f = ((A(id) - A(id - 1)) * dxiv + (Cc(id + px) - Cc(id)) * (.5f * dyiv)) +
          (T13(id + pl, k + 1) - T13(id, k)) * dziv;
    }
    if (smooth) {
      auto A = [&](int dx, int dy, int dz) {
        const int kk = k + dz;
        return C(C_RST8U, kk) * (ld(a.up, id + dx + dy * px + dz * pl) - C(C_UBR, kk)) / C(C_JCB8U, kk);
      };
      f = smooth_into(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 2, A);
    }
    if (a.vspopt >= 1 && a.vsp_u && k >= a.ksp0 - 1) {
      const float r8s = .25f * (C(C_RBCT, k) + C(C_RBCT, k + 1));
      f = f - C(C_RST8U, k) * (r8s + r8s) * (ld(a.up, id) - C(C_UBR, k));
    }
    if (a.coropt == 1) {
      const float rst = C(C_RST, k);
      const float c0 = a.fc * rst * (ld(a.v, id - 1) + ld(a.v, id - 1 + px));
      const float c1 = a.fc * rst * (ld(a.v, id) + ld(a.v, id + px));
      f = f + (c0 + c1);
    }
    // advuvw.f90:231-397
    auto U = [&](long long p) { return ld(a.u, p); };
    auto t1 = [&](long long p) { return (RXU(p, k) + RXU(p + 1, k)) * (U(p + 1) - U(p)) * dxv25n; };
    auto t2 = [&](long long p) { return (RXV(p - 1, k) + RXV(p, k)) * (U(p) - U(p - px)) * dyv25n; };
    auto t3 = [&](long long p, int kk) {
      return (RXW(p - 1, kk) + RXW(p, kk)) * (U(p) - U(p - pl)) * dzv25n;
    };
    float hadv = (t1(id - 1) + t1(id)) + (t2(id) + t2(id + px));
    auto t1w = [&](long long p) { return (RXU(p - 1, k) + RXU(p + 1, k)) * (U(p + 1) - U(p - 1)) * dxv24; };
    auto t2w = [&](long long p) {
      return ((RXV(p - 1, k) + RXV(p, k)) + (RXV(p - 1 + px, k) + RXV(p + px, k))) * (U(p + px) - U(p - px)) * dyv48;
    };
    hadv = fourd3 * hadv + ((t1w(id - 1) + t1w(id + 1)) + (t2w(id - px) + t2w(id + px)));
    f = f + hadv + (t3(id, k) + t3(id + pl, k + 1));
    a.ufrc[id] = f;
  }
  // ---------------------------------------------------------------- vfrc
  if (grp == 1 && i <= ni - 2 && k <= nk - 2) {
    float f = 0.f;
    if (a.rkv) {   // s_turbuvw v part (turbuvw.f90:795-840)
      const float jc = C(C_JCB, k), j8v = C(C_JCB8V, k);
      auto B = [&](long long p) { return jc * (RKV(p) * D.s22(p, k)); };
      auto T12 = [&](long long p) {
        return .25f * D.s12(p, k) * ((RKV(p - 1 - px) + RKV(p)) + (RKV(p - 1) + RKV(p - px)));
      };
      auto Cc = [&](long long p) { return (j8v + j8v) * T12(p); };
      auto T23 = [&](long long p, int kk) {
        return .25f * D.s23(p, kk) * ((RKV(p - px - pl) + RKV(p)) + (RKV(p - px) + RKV(p - pl)));
      };
      f = ((B(id) - B(id - px)) * dyiv + (Cc(id + 1) - Cc(id)) * (.5f * dxiv)) +
          (T23(id + pl, k + 1) - T23(id, k)) * dziv;
    }
    if (smooth) {
      auto A = [&](int dx, int dy, int dz) {
        const int kk = k + dz;
        return C(C_RST8V, kk) * (ld(a.vp, id + dx + dy * px + dz * pl) - C(C_VBR, kk)) / C(C_JCB8V, kk);
      };
      f = smooth_into(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 2, A);
    }
    if (a.vspopt >= 1 && a.vsp_v && k >= a.ksp0 - 1) {
      const float r8s = .25f * (C(C_RBCT, k) + C(C_RBCT, k + 1));
      f = f - C(C_RST8V, k) * (r8s + r8s) * (ld(a.vp, id) - C(C_VBR, k));
    }
    if (a.coropt == 1) {
      const float rst = C(C_RST, k);
      const float c0 = -a.fc * rst * (ld(a.u, id - px) + ld(a.u, id - px + 1));
      const float c1 = -a.fc * rst * (ld(a.u, id) + ld(a.u, id + 1));
      f = f + (c0 + c1);
    }
    // advuvw.f90:458-624
    auto V = [&](long long p) { return ld(a.v, p); };
    auto t1 = [&](long long p) { return (RXU(p - px, k) + RXU(p, k)) * (V(p) - V(p - 1)) * dxv25n; };
    auto t2 = [&](long long p) { return (RXV(p, k) + RXV(p + px, k)) * (V(p + px) - V(p)) * dyv25n; };
    auto t3 = [&](long long p, int kk) {
      return (RXW(p - px, kk) + RXW(p, kk)) * (V(p) - V(p - pl)) * dzv25n;
    };
    float hadv = (t1(id) + t1(id + 1)) + (t2(id - px) + t2(id));
    auto t1w = [&](long long p) {
      return ((RXU(p - px, k) + RXU(p, k)) + (RXU(p + 1 - px, k) + RXU(p + 1, k))) * (V(p + 1) - V(p - 1)) * dxv48;
    };
    auto t2w = [&](long long p) { return (RXV(p - px, k) + RXV(p + px, k)) * (V(p + px) - V(p - px)) * dyv24; };
    hadv = fourd3 * hadv + ((t1w(id - 1) + t1w(id + 1)) + (t2w(id - px) + t2w(id + px)));
    f = f + hadv + (t3(id, k) + t3(id + pl, k + 1));
    a.vfrc[id] = f;
  }
  // ---------------------------------------------------------------- wfrc
  if (grp == 2 && i <= ni - 2 && j <= nj - 2) {
    float f = 0.f;
    if (a.rkv) {   // s_turbuvw w part (turbuvw.f90:1300-1330)
      const float j8u = C(C_JCB8U, k - 1) + C(C_JCB8U, k), j8v = C(C_JCB8V, k - 1) + C(C_JCB8V, k);
      auto T33 = [&](long long p, int kk) { return RKV(p) * D.s33(p, kk); };
      auto T31 = [&](long long p) {
        return .25f * D.s13(p, k) * ((RKV(p - 1 - pl) + RKV(p)) + (RKV(p - 1) + RKV(p - pl)));
      };
      auto T32 = [&](long long p) {
        return .25f * D.s23(p, k) * ((RKV(p - px - pl) + RKV(p)) + (RKV(p - px) + RKV(p - pl)));
      };
      auto Aw = [&](long long p) { return j8u * T31(p); };
      auto Cw = [&](long long p) { return j8v * T32(p); };
      f = (T33(id, k) - T33(id - pl, k - 1)) * dziv +
          ((Aw(id + 1) - Aw(id)) * (.5f * dxiv) + (Cw(id + px) - Cw(id)) * (.5f * dyiv));
    }
    if (smooth) {
      auto A = [&](int dx, int dy, int dz) {
        const int kk = k + dz;
        return C(C_RST8W, kk) * ld(a.wp, id + dx + dy * px + dz * pl) / C(C_JCB8W, kk);
      };
      f = smooth_into(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 1, A);
    }
    if (a.vspopt >= 1 && a.vsp_w && k >= a.ksp0) f = f - C(C_RBCT, k) * C(C_RST8W, k) * ld(a.wp, id);
    if (k >= 3 && k <= nk - 2) {   // buoywb.f90:166-172 (dry), 202-299 (moist), 307-313
      auto wb8s = [&](long long p, int kk) {
        if (!a.qv) return g05 * C(C_RST, kk) * ld(a.ptp, p) / C(C_PTBR, kk);
        const float qvbr = C(C_QVBR, kk);
        const float qvd = ld(a.qv, p) - qvbr;
        const float qall = (((ld(a.qc, p) + ld(a.qr, p)) + ld(a.qi, p)) + ld(a.qs, p)) + ld(a.qg, p);  // totalqwi.f90:163
        return g05 * C(C_RST, kk) *
               ((qvd / (kEpsva + qvbr) - (qvd + qall) / (1.f + qvbr)) + ld(a.ptp, p) / C(C_PTBR, kk));
      };
      f = f + (wb8s(id - pl, k - 1) + wb8s(id, k));
    }
    // advuvw.f90:685-852
    auto W = [&](long long p) { return ld(a.w, p); };
    auto t1 = [&](long long p) { return (RXU(p - pl, k - 1) + RXU(p, k)) * (W(p) - W(p - 1)) * dxv25n; };
    auto t2 = [&](long long p) { return (RXV(p - pl, k - 1) + RXV(p, k)) * (W(p) - W(p - px)) * dyv25n; };
    auto t3 = [&](long long p, int kk) {
      return (RXW(p, kk) + RXW(p + pl, kk + 1)) * (W(p + pl) - W(p)) * dzv25n;
    };
    float hadv = (t1(id) + t1(id + 1)) + (t2(id) + t2(id + px));
    auto t1w = [&](long long p) {
      return ((RXU(p - pl, k - 1) + RXU(p, k)) + (RXU(p + 1 - pl, k - 1) + RXU(p + 1, k))) * (W(p + 1) - W(p - 1)) * dxv48;
    };
    auto t2w = [&](long long p) {
      return ((RXV(p - pl, k - 1) + RXV(p, k)) + (RXV(p + px - pl, k - 1) + RXV(p + px, k))) * (W(p + px) - W(p - px)) * dyv48;
    };
    hadv = fourd3 * hadv + ((t1w(id - 1) + t1w(id + 1)) + (t2w(id - px) + t2w(id + px)));
    f = f + hadv + (t3(id - pl, k - 1) + t3(id, k));
    a.wfrc[id] = f;
  }
  // ------------------------------------------------- pfrc, theta' step
  if (grp == 3 && i <= ni - 2 && j <= nj - 2 && k <= nk - 2) {
    // advs-type advection of s with fluxes FU/FV/FW (advs.f90:205-370)
    auto adv = [&](const float* s, auto FU, auto FV, auto FW) {
      auto S = [&](long long p) { return ld(s, p); };
      auto t1 = [&](long long p) { return FU(p) * (S(p) - S(p - 1)) * dxv05n; };
      auto t2 = [&](long long p) { return FV(p) * (S(p) - S(p - px)) * dyv05n; };
      auto t3 = [&](long long p, int kk) { return FW(p, kk) * (S(p) - S(p - pl)) * dzv05n; };
      float sf = (t1(id) + t1(id + 1)) + (t2(id) + t2(id + px));
      auto t1w = [&](long long p) { return (FU(p) + FU(p + 1)) * (S(p + 1) - S(p - 1)) * dxv24; };
      auto t2w = [&](long long p) { return (FV(p) + FV(p + px)) * (S(p + px) - S(p - px)) * dyv24; };
      sf = fourd3 * sf + ((t1w(id - 1) + t1w(id + 1)) + (t2w(id - px) + t2w(id + px)));
      return sf + (t3(id, k) + t3(id + pl, k + 1));
    };
    // pressure (advp.f90:255-291 J-weighted fluxes)
    {
      auto FU = [&](long long p) { return C(C_JCB8U, k) * ld(a.u, p); };
      auto FV = [&](long long p) { return C(C_JCB8V, k) * ld(a.v, p); };
      auto FW = [&](long long p, int kk) { return C(C_JCB8W, kk) * WC(p, kk); };
      float f = adv(a.pp, FU, FV, FW);
      if (smooth) {
        auto A = [&](int dx, int dy, int dz) { return ld(a.ppp, id + dx + dy * px + dz * pl); };
        f = smooth_into(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 2, A);
      }
      if (a.vspopt >= 1 && a.vsp_p && k >= a.ksp0 - 1)
        f = f - .5f * (C(C_RBCT, k) + C(C_RBCT, k + 1)) * C(C_JCB, k) * ld(a.ppp, id);
      a.pfrc[id] = f;
    }
    // theta'
    {
      auto FU = [&](long long p) { return RXU(p, k); };
      auto FV = [&](long long p) { return RXV(p, k); };
      auto FW = [&](long long p, int kk) { return RXW(p, kk); };
      float f = adv(a.ptp, FU, FV, FW);
      if (smooth) {
        auto A = [&](int dx, int dy, int dz) { return C(C_RBR, k + dz) * ld(a.ptpp, id + dx + dy * px + dz * pl); };
        f = smooth_into(f, a.smtopt, a.smhcoe, a.smvcoe, k, 2, nk - 2, A);
      }
      if (a.rkv) {   // forcept.f90:313-320, 383-393: mixing of the full theta at t-dt
        auto S = [&](long long p, int kk) { return C(C_PTBR, kk) + ld(a.ptpp, p); };
        f = turb_scalar(f, a.rkv, col, nc, id, k, px, pl, a.cpriv, dxiv, dyiv, dziv, S);
      }
      if (a.vspopt >= 1 && a.vsp_pt && k >= a.ksp0 - 1)
        f = f - .5f * (C(C_RBCT, k) + C(C_RBCT, k + 1)) * C(C_RST, k) * ld(a.ptpp, id);
      const float dziv25 = .25f * dziv;   // advbspt.f90:135-166
      auto pta8w = [&](long long p, int kk) {
        return (C(C_RBR, kk - 1) + C(C_RBR, kk)) * ld(a.w, p) * (C(C_PTBR, kk - 1) - C(C_PTBR, kk)) * dziv25;
      };
      f = f + (pta8w(id, k) + pta8w(id + pl, k + 1));
      const float dtdrst = a.dtb2 / C(C_RST, k);                     // steps.f90:528
      const float ptpf = ld(a.ptpp, id) + f * dtdrst;                 // steps.f90:568
      a.ptpf[id] = ptpf;
      if (k == 2) a.ptpf[id - pl] = ptpf;                             // vbcs.f90:118
      if (k == nk - 2) a.ptpf[id + pl] = ptpf;                        // vbcs.f90:132
    }
  }
}

// s_timeflt, SrcOrig/timeflt.f90:335-404 on the interior (ghosts are
// refilled by k_halo afterwards).
__global__ void __launch_bounds__(256) k_timeflt(const FilterArgs a) {
  const Grid g = a.g;
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > g.ni - 1 || j > g.nj - 1 || k > g.nk) return;
  const long long id = g.at(i, j, k);
  const float fc = a.filcoe, m1fc2 = 1.f - 2.f * a.filcoe;
  const bool si = i <= g.ni - 2, sj = j <= g.nj - 2;
  if (k <= g.nk - 1) {
    if (sj) a.u[id] = m1fc2 * a.u[id] + fc * (a.uf[id] + a.up[id]);
    if (si) a.v[id] = m1fc2 * a.v[id] + fc * (a.vf[id] + a.vp[id]);
    if (si && sj) {
      a.pp[id] = m1fc2 * a.pp[id] + fc * (a.ppf[id] + a.ppp[id]);
      a.ptp[id] = m1fc2 * a.ptp[id] + fc * (a.ptpf[id] + a.ptpp[id]);
    }
  }
  if (si && sj) a.w[id] = m1fc2 * a.w[id] + fc * (a.wf[id] + a.wp[id]);
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
// ni+1} (j = 2..nj-2), one level per blockIdx.y; per field the staggering
// decides which of them are ghosts.  Sources are never ghosts, so the
// order of the copies does not matter.
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
  for (int n = 0; n < a.n; ++n) {
    const int st = a.stag[n];
    const bool gx = (st == STAG_U) ? (i <= 1 || i >= ni) : (i <= 1 || (i >= ni - 1 && i <= ni));
    const bool gy = (st == STAG_V) ? (j <= 1 || j >= nj) : (j <= 1 || (j >= nj - 1 && j <= nj));
    const bool inx = (st == STAG_U) ? (i <= ni + 1) : (i <= ni);
    const bool iny = (st == STAG_V) ? (j <= nj + 1) : (j <= nj);
    if (!(gx || gy) || !inx || !iny) continue;
    const int si = gx ? wrap(i, ni) : i;
    const int sj = gy ? wrap(j, nj) : j;
    float* f = a.f[n];
    f[g.at(i, j, k)] = f[g.at(si, sj, k)];
  }
}

}  // namespace

int launch_force(const ForceArgs& a, cudaStream_t st) {
  dim3 b(32, 8, 1);
  dim3 gr((a.g.ni - 2 + 31) / 32, (a.g.nj - 2 + 7) / 8, (a.g.nk - 2) * 4);
  k_force<<<gr, b, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

int launch_timeflt(const FilterArgs& a, cudaStream_t st) {
  dim3 b(32, 8, 1);
  dim3 gr((a.g.ni - 2 + 31) / 32, (a.g.nj - 2 + 7) / 8, a.g.nk);
  k_timeflt<<<gr, b, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

int launch_halo(const HaloArgs& a, cudaStream_t st) {
  const int frame = 5 * (a.g.ni + 2) + 5 * (a.g.nj - 3);
  dim3 gr((frame + 127) / 128, a.g.nk, 1);
  k_halo<<<gr, 128, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace cress

// Fused HE-VE acoustic substep for sm_100a (impopt=0): one pass of s_heve
// (SrcOrig/heve.f90:337-406, gwmopt=0, flat terrain, no map factors,
// periodic lateral boundaries on one GPU, rigid bottom and lid):
//   pgrad + diver3d (divergence damping)   pgrad.f90:251-395, diver3d.f90:182-326
//   stepuv + bcycle + vbcu/vbcv            stepuv.f90:288-424
//   buoywse (buyopt=1)                     buoywse.f90:135-187
//   stepwe + bcycle + phy2cnt + vbcw       stepwe.f90:255-370, phy2cnt.f90:193-227
//   diverpe, advbspe                       diverpe.f90:153-169, advbspe.f90:118-135
//   steppe + bcycle + vbcp                 steppe.f90:218-323
//
// Design.  As k_hevi2 (hevi2.cu): a block of 32 x 4 threads owns a 32 x 8
// tile of columns, two rows per thread packed into FP32x2 lanes, and
// marches k upward through a TMA ring of the old u, v, w, p' and the
// four forcings.  Everything is explicit in k, so one upward pass does the
// whole substep: at level k the thread forms the damped pressure, the new
// u and v, the new w of level k (from the vertical pressure gradient and
// buoyancy of levels k-1 and k) and then the new p' of level k-1, which
// needs the new w of k-1 and k.
//
// A reference detail kept for parity: stepwe updates w on levels 2..nk-1,
// phy2cnt turns that into the contravariant wc, and only then vbcw sets w
// itself to 0 on levels 2 and nk-1.  diverpe (and the next substep's
// divergence damping) therefore see a nonzero wc there.  Those two planes
// of wc live in a side buffer (ping-pong between substeps); wc of levels 1
// and nk is never written and stays 0.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "common.cuh"
#include "f2.cuh"
#include "hevi.cuh"
#include "tma.cuh"

namespace cress {

namespace {

constexpr int kVTY = 8;      // tile rows
constexpr int kVRows = 4;    // thread rows (two tile rows each)

__host__ __device__ constexpr int r128e(int n) { return (n + 31) / 32 * 32; }

template <int S>
struct HeLayout {
  using R = HeviRows<kVTY>;
  static constexpr int BX = kHeviBoxX;
  static constexpr int oU = 0;
  static constexpr int oV = oU + r128e(BX * R::u);
  static constexpr int oW = oV + r128e(BX * R::v);
  static constexpr int oP = oW + r128e(BX * R::w);
  static constexpr int oUF = oP + r128e(BX * R::p);
  static constexpr int oVF = oUF + r128e(BX * R::uf);
  static constexpr int oWF = oVF + r128e(BX * R::vf);
  static constexpr int oPF = oWF + r128e(BX * R::wf);
  static constexpr int stage = oPF + r128e(BX * R::pf);
  static constexpr uint32_t tx_bytes =
      4u * BX * (R::u + R::v + R::w + R::p + R::uf + R::vf + R::wf + R::pf);
  static constexpr int t3h_floats = r128e((kVTY + 2) * BX);
  static size_t bytes() { return 4 * ((size_t)S * stage + 2 * (size_t)t3h_floats) + 8 * (size_t)S; }
};

template <int S, int DIV, bool STH, bool BUY>
__global__ void __launch_bounds__(kHeviTX * kVRows, 4)
k_heve(const __grid_constant__ HeviMaps m, const HeviArgs a) {
  using L = HeLayout<S>;
  constexpr int TX = kHeviTX, TY = kVTY, BX = kHeviBoxX;
  const unsigned full = 0xffffffffu;
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = 2 + blockIdx.x * TX, j0 = 2 + blockIdx.y * TY;
  const int xb = i0 - 2;  // box x origin (multiple of 32)
  const int ilast = min(i0 + TX - 1, ni - 2), jlast = min(j0 + TY - 1, nj - 2);
  const int i = i0 + tx, jA = j0 + 2 * ty, jB = jA + 1;
  const bool ownA = (i <= ilast) && (jA <= jlast), ownB = (i <= ilast) && (jB <= jlast);
  const bool ei = (i <= 3) || (i >= ni - 2);
  const bool edgeA = ei || (jA <= 3) || (jA >= nj - 2), edgeB = ei || (jB <= 3) || (jB >= nj - 2);
  const bool xlast = (i == ilast) && (i + 1 == ni - 1);
  const bool ylastA = (jA == jlast) && (jA + 1 == nj - 1), ylastB = (jB == jlast) && (jB + 1 == nj - 1);

  extern __shared__ __align__(1024) float smem[];
  float* ring = smem;
  float* t3hb = ring + S * L::stage;          // 2 x [(TY+2)][BX], rows from j0-1, x from i0-2
  uint64_t* bars = reinterpret_cast<uint64_t*>(t3hb + 2 * L::t3h_floats);
  auto CK = [&](int kk, int f) { return __ldg(a.lvl + kk * kLevelStride + f); };
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
    tma_load_3d(st + L::oU, &m.u, xb, j0 - 1, z, bar);
    tma_load_3d(st + L::oV, &m.v, xb, j0 - 1, z, bar);
    tma_load_3d(st + L::oW, &m.w, xb, j0 - 1, z, bar);
    tma_load_3d(st + L::oP, &m.p, xb, j0 - 1, z, bar);
    tma_load_3d(st + L::oUF, &m.uf, xb, j0, z, bar);
    tma_load_3d(st + L::oVF, &m.vf, xb, j0, z, bar);
    tma_load_3d(st + L::oWF, &m.wf, xb, j0, z, bar);
    tma_load_3d(st + L::oPF, &m.pf, xb, j0, z, bar);
  };
  if (tid == 0)
    for (int lv = 1; lv <= min(S, lmax); ++lv) issue(lv);

  constexpr int NH = 2 * TX + 2 * TY;
  int hx = 0, hy = 0;
  {
    int n = tid;
    if (n < TX) { hx = n + 2; hy = 0; }
    else if ((n -= TX) < TX) { hx = n + 2; hy = TY + 1; }
    else if ((n -= TX) < TY) { hx = 1; hy = n + 1; }
    else { n -= TY; hx = TX + 2; hy = n + 1; }
  }
  const bool has_halo = tid < NH;
  const int ox = tx + 2;
  const int oyA = 2 * ty + 1, oyB = oyA + 1;   // own rows in the boxes that start at j0-1
  const int fyA = 2 * ty, fyB = fyA + 1;       // own rows in the forcing boxes (from j0)
  const float dts = a.dts, dxiv = a.dxiv, dyiv = a.dyiv, dziv = a.dziv;
  const float g05 = a.g05, g05n = a.g05n;
  const int plane = (int)g.plane, px = g.px;
  // the old wc of levels 2 and nk-1 at the box point (x, y): the side
  // buffer, or (first substep) phy2cnt of the old w
  auto wc_side = [&](int kk, const float* W, int x, int y) -> float {
    if (a.wc_from_w) return STH ? W[y * BX + x] * CK(kk, C_IJCB8W) : W[y * BX + x];
    const int gi = xb + x, gj = j0 - 1 + y;
    if (gi > ni + 1 || gj > nj + 1) return 0.f;   // beyond the array: feeds no owned point
    return __ldg(a.wc_old + (kk == 2 ? 0 : plane) + gi + px * gj);
  };
  // the new wc of levels 2 and nk-1 into the side buffer (and its periodic images)
  auto put_side = [&](int kk, int j, float v) {
    float* base = a.wc_new + (kk == 2 ? 0 : plane);
    const Grid g2{g.ni, g.nj, 1, g.px, g.py, g.plane};
    store_periodic(base, g2, STAG_S, i, j, 1, v);
  };

  F2 t3v_prev = f2(0.f), wb8s_prev = f2(0.f);   // level k-1, rows A and B
  F2 wcn_prev = f2(0.f), wadv_prev = f2(0.f);   // new wc and new w (after vbcw) of level k-1
  F2 hdiv_prev = f2(0.f), pp_prev = f2(0.f), pf_prev = f2(0.f);
  float p2A = 0.f, p2B = 0.f, p3A = 0.f, p3B = 0.f, pkA = 0.f, pkB = 0.f;
  float w3A = 0.f, w3B = 0.f, wkA = 0.f, wkB = 0.f;
  bool fail = false;
  auto wait_level = [&](int lv) {
    if (!fail && lv <= lmax) fail = !mbar_wait(&bars[(lv - 1) % S], ((lv - 1) / S) & 1);
  };
  wait_level(1);
  int idA = (int)g.at(i, jA, 1);

  for (int k = 1; k <= nk - 1; ++k, idA += plane) {
    const int idB = idA + px;
    wait_level(k + 1);
    float* t3h = t3hb + (k & 1) * L::t3h_floats;
    const float* st0 = ring + ((k - 1) % S) * L::stage;
    const float* st1 = ring + (k % S) * L::stage;   // level k+1 (not staged for k = nk-1)
    const float* U = st0 + L::oU;
    const float* V = st0 + L::oV;
    const float* W0 = st0 + L::oW;
    const float* W1 = st1 + L::oW;
    const float* P = st0 + L::oP;
    const float* UF = st0 + L::oUF;
    const float* VF = st0 + L::oVF;
    const float* WF = st0 + L::oWF;
    const float* PF = st0 + L::oPF;
    const float rst8u = CK(k, C_RST8U), rst8v = CK(k, C_RST8V);
    const float rst8wk = CK(k, C_RST8W), rst8wk1 = CK(k + 1, C_RST8W);
    const float jcbk = CK(k, C_JCB), ijcbk = CK(k, C_IJCB);
    // the old contravariant w of levels k and k+1 at a box point
    auto wc_at = [&](int kk, const float* W, int x, int y) -> float {
      if (kk == 1 || kk == nk) return 0.f;
      if (kk == 2 || kk == nk - 1) return wc_side(kk, W, x, y);
      return STH ? W[y * BX + x] * CK(kk, C_IJCB8W) : W[y * BX + x];
    };
    // diver3d.f90:318 on the old winds
    auto div3d_at = [&](int x, int y) {
      const float wck = wc_at(k, W0, x, y), wck1 = wc_at(k + 1, W1, x, y);
      return (rst8wk * wck - rst8wk1 * wck1) * dziv +
             ((rst8u * U[y * BX + x] - rst8u * U[y * BX + x + 1]) * dxiv +
              (rst8v * V[y * BX + x] - rst8v * V[(y + 1) * BX + x]) * dyiv);
    };
    auto col2 = [&](const float* base, int oy) { return f2(base[oy * BX + ox], base[(oy + 1) * BX + ox]); };
    const F2 div = f2(div3d_at(ox, oyA), div3d_at(ox, oyB));
    const F2 pp = col2(P, oyA);
    const F2 t3v = (DIV >= 1) ? pp + a.divcv * jcbk * div : pp;                    // pgrad.f90:300
    const bool uvlev = k >= 2 && k <= nk - 2;   // levels with u, v and p' updates
    F2 tc = f2(0.f);
    if (uvlev) {
      F2 th;                                                                       // pgrad.f90:341,363
      if constexpr (DIV == 2) th = pp + a.divch * div * ijcbk;
      else if constexpr (DIV == 1) th = pp + a.divcv * jcbk * div;
      else th = pp;
      tc = jcbk * th;
      t3h[oyA * BX + ox] = tc.v.x;
      t3h[oyB * BX + ox] = tc.v.y;
      if (has_halo) {
        const float dh = div3d_at(hx, hy), ph = P[hy * BX + hx];
        float thh;
        if constexpr (DIV == 2) thh = ph + a.divch * dh * ijcbk;
        else if constexpr (DIV == 1) thh = ph + a.divcv * jcbk * dh;
        else thh = ph;
        t3h[hy * BX + hx] = jcbk * thh;
      }
    }
    // Every thread has finished level k-1 and written this level's t3h,
    // so the slot of level k-1 may be refilled with level k+S-1.
    __syncthreads();
    if (tid == 0 && !fail && k >= 2 && k + S - 1 <= lmax) {   // refill only after its copy was seen to land
      fence_proxy_async_smem();
      issue(k + S - 1);
    }

    // -- stepuv at levels 2..nk-2 (the faces as in k_hevi2) --------------
    F2 hdiv = f2(0.f);
    if (uvlev) {
      const float irst8u = CK(k, C_IRST8U), irst8v = CK(k, C_IRST8V);
      const F2 un0 = col2(U, oyA) + dts * (col2(UF, fyA) + (col2(t3h - 1, oyA) - tc) * dxiv) * irst8u;
      F2 un1 = f2(__shfl_down_sync(full, un0.v.x, 1), __shfl_down_sync(full, un0.v.y, 1));
      if (tx == TX - 1)
        un1 = col2(U + 1, oyA) + dts * (col2(UF + 1, fyA) + (tc - col2(t3h + 1, oyA)) * dxiv) * irst8u;
      const F2 vs = col2(V, oyA) + dts * (col2(VF, fyA) + (f2(t3h[(oyA - 1) * BX + ox], tc.v.x) - tc) * dyiv) * irst8v;
      const float vf2 = V[(oyB + 1) * BX + ox] +
                        dts * (VF[(fyB + 1) * BX + ox] + (tc.v.y - t3h[(oyB + 1) * BX + ox]) * dyiv) * irst8v;
      const F2 vn = f2(vs.v.y, vf2);
      const bool kend = (k == 2) || (k == nk - 2);
      auto store_uv = [&](bool edge, bool ylast, int j, int id, float u0, float u1, float v0, float v1) {
        if (edge) {
          store_periodic(a.u_new, g, STAG_U, i, j, k, u0);
          store_periodic(a.v_new, g, STAG_V, i, j, k, v0);
        } else {
          a.u_new[id] = u0;
          a.v_new[id] = v0;
        }
        if (xlast) store_periodic(a.u_new, g, STAG_U, i + 1, j, k, u1);
        if (ylast) store_periodic(a.v_new, g, STAG_V, i, j + 1, k, v1);
        if (kend) {   // vbcu.f90:120,134 (and vbcv)
          const int kc = k == 2 ? 1 : nk - 1;
          store_periodic(a.u_new, g, STAG_U, i, j, kc, u0);
          store_periodic(a.v_new, g, STAG_V, i, j, kc, v0);
          if (xlast) store_periodic(a.u_new, g, STAG_U, i + 1, j, kc, u1);
          if (ylast) store_periodic(a.v_new, g, STAG_V, i, j + 1, kc, v1);
        }
      };
      if (ownA) store_uv(edgeA, ylastA, jA, idA, un0.v.x, un1.v.x, vs.v.x, vn.v.x);
      if (ownB) store_uv(edgeB, ylastB, jB, idB, un0.v.y, un1.v.y, vs.v.y, vn.v.y);
      // horizontal part of diverpe's divergence (jcb-weighted new winds)
      const float jcb8u = CK(k, C_JCB8U), jcb8v = CK(k, C_JCB8V);
      hdiv = (jcb8u * un0 - jcb8u * un1) * dxiv + (jcb8v * vs - jcb8v * vn) * dyiv;
    }

    // -- stepwe at level k (2..nk-1): w + dts (wfrc + wpg + buoyancy) / rst8w
    F2 wb8s = f2(0.f);
    if (BUY && uvlev) wb8s = pp * CK(k, C_RST) * CK(k, C_IRCSQ) * g05n;             // buoywse.f90:151
    F2 wcn = f2(0.f), wadv = f2(0.f);
    if (k >= 2) {
      F2 wsml = (t3v_prev - t3v) * dziv;                                            // pgrad.f90:320
      if (BUY && k >= 3 && k <= nk - 2) wsml = wsml + (wb8s_prev + wb8s);           // buoywse.f90:184
      const F2 wn = col2(W0, oyA) + dts * (col2(WF, fyA) + wsml) * CK(k, C_IRST8W);  // stepwe.f90:261
      wcn = STH ? wn * CK(k, C_IJCB8W) : wn;                                        // phy2cnt.f90:219
      if (k == 2 || k == nk - 1) {
        // vbcw.f90:317,481: w = 0 here; the contravariant value stays
        if (ownA) put_side(k, jA, wcn.v.x);
        if (ownB) put_side(k, jB, wcn.v.y);
        wadv = f2(0.f);
        if (ownA) store_periodic(a.w_new, g, STAG_S, i, jA, k, 0.f);
        if (ownB) store_periodic(a.w_new, g, STAG_S, i, jB, k, 0.f);
      } else {
        wadv = wn;
        if (ownA) { if (edgeA) store_periodic(a.w_new, g, STAG_S, i, jA, k, wn.v.x); else a.w_new[idA] = wn.v.x; }
        if (ownB) { if (edgeB) store_periodic(a.w_new, g, STAG_S, i, jB, k, wn.v.y); else a.w_new[idB] = wn.v.y; }
        if (k == 3) { w3A = wcn.v.x; w3B = wcn.v.y; }
        if (k == nk - 2) { wkA = wcn.v.x; wkB = wcn.v.y; }
      }
    }

    // -- diverpe, advbspe, steppe at level k-1 (2..nk-2) ---------------
    if (k >= 3) {
      const int kp = k - 1;
      const F2 pdiv = CK(kp, C_RCSQ) *
                      ((CK(kp, C_JCB8W) * wcn_prev - CK(k, C_JCB8W) * wcn) * dziv + hdiv_prev);  // diverpe.f90:169
      const F2 psml = g05 * (wadv_prev + wadv) * CK(kp, C_RST) + pdiv;                             // advbspe.f90:127
      const F2 pn = pp_prev + dts * (pf_prev + psml) * CK(kp, C_IJCB);                             // steppe.f90:224
      const int ipA = idA - plane, ipB = idB - plane;
      if (ownA) { if (edgeA) store_periodic(a.p_new, g, STAG_S, i, jA, kp, pn.v.x); else a.p_new[ipA] = pn.v.x; }
      if (ownB) { if (edgeB) store_periodic(a.p_new, g, STAG_S, i, jB, kp, pn.v.y); else a.p_new[ipB] = pn.v.y; }
      if (kp == 2) { p2A = pn.v.x; p2B = pn.v.y; }
      if (kp == 3) { p3A = pn.v.x; p3B = pn.v.y; }
      if (kp == nk - 2) { pkA = pn.v.x; pkB = pn.v.y; }
    }
    t3v_prev = t3v;
    wb8s_prev = wb8s;
    wcn_prev = wcn;
    wadv_prev = wadv;
    hdiv_prev = hdiv;
    pp_prev = pp;
    pf_prev = col2(PF, fyA);
  }

  if (__syncthreads_or(fail)) {
    if (tid == 0) {
      atomicExch(a.err, 1);
      for (int s = 0; s < S; ++s) {
        int kl = -1;
        for (int lv = 1; lv <= issued; ++lv)
          if ((lv - 1) % S == s) kl = lv;
        if (kl >= 0) mbar_wait(&bars[s], ((kl - 1) / S) & 1);
      }
    }
    return;
  }
  // vbcw.f90:285,471 images (from the contravariant w of levels 3 and
  // nk-2), vbcp.f90:126-160, and level nk of u, v, p' carried over
  auto finish = [&](bool own, bool ylast, int j, float w3, float wk, float p2, float p3, float pk) {
    if (!own) return;
    const float j8w3 = CK(3, C_JCB8W), j8wt = CK(nk - 2, C_JCB8W);
    store_periodic(a.w_new, g, STAG_S, i, j, 1, -j8w3 * w3 - 0.f);
    store_periodic(a.w_new, g, STAG_S, i, j, nk, -j8wt * wk - 0.f);
    store_periodic(a.p_new, g, STAG_S, i, j, 1, (a.bbc == 2) ? 2.f * p2 - p3 : p2);
    store_periodic(a.p_new, g, STAG_S, i, j, nk - 1, pk);
    store_periodic(a.p_new, g, STAG_S, i, j, nk, a.p_old[g.at(i, j, nk)]);
    store_periodic(a.u_new, g, STAG_U, i, j, nk, a.u_old[g.at(i, j, nk)]);
    store_periodic(a.v_new, g, STAG_V, i, j, nk, a.v_old[g.at(i, j, nk)]);
    if (xlast) store_periodic(a.u_new, g, STAG_U, i + 1, j, nk, a.u_old[g.at(i + 1, j, nk)]);
    if (ylast) store_periodic(a.v_new, g, STAG_V, i, j + 1, nk, a.v_old[g.at(i, j + 1, nk)]);
  };
  finish(ownA, ylastA, jA, w3A, wkA, p2A, p3A, pkA);
  finish(ownB, ylastB, jB, w3B, wkB, p2B, p3B, pkB);
}

template <int DIV, bool STH, bool BUY>
int launch_e(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st) {
  constexpr int S = 4;
  using L = HeLayout<S>;
  const Grid& g = a.g;
  const size_t bytes = L::bytes();
  auto kern = k_heve<S, DIV, STH, BUY>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
    return CRESS_E_CUDA;
  dim3 block(kHeviTX, kVRows);
  dim3 grid((g.ni - 3 + kHeviTX - 1) / kHeviTX, (g.nj - 3 + kVTY - 1) / kVTY);
  kern<<<grid, block, bytes, st>>>(maps, a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

template <int DIV>
int launch_e_div(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st) {
  const bool sth = a.sthopt != 0, buy = a.buyopt == 1;
  if (sth) return buy ? launch_e<DIV, true, true>(a, maps, st) : launch_e<DIV, true, false>(a, maps, st);
  return buy ? launch_e<DIV, false, true>(a, maps, st) : launch_e<DIV, false, false>(a, maps, st);
}

}  // namespace

int launch_heve_substep(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st) {
  if (a.g.count() >= (1LL << 31) || a.g.nk < 6 || !a.lvl || !a.wc_new || (!a.wc_from_w && !a.wc_old))
    return CRESS_E_UNSUPPORTED;
  switch (a.divopt) {
    case 2: return launch_e_div<2>(a, maps, st);
    case 1: return launch_e_div<1>(a, maps, st);
    default: return launch_e_div<0>(a, maps, st);
  }
}

}  // namespace cress

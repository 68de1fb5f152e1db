// Fused HE-VI acoustic substep for sm_100a.
//
// One launch = one pass of s_hevi (SrcOrig/hevi.f90:339-426) for
// impopt=1, gwmopt=0, flat terrain, no map factors, periodic lateral
// boundaries on one GPU, rigid bottom/top (bbc=tbc=2):
//   pgrad + diver3d (divergence damping)   pgrad.f90:251-395, diver3d.f90:182-326
//   stepuv + bcycle + vbcu/vbcv            stepuv.f90:288-424
//   diverpih + diver2d                     diverpih.f90:188-214
//   diverpiv, advbspi('back')              diverpiv.f90:118-130, advbspi.f90:150-165
//   pgradiv, buoywsi                       pgradiv.f90:135-170, buoywsi.f90:153-211
//   stepwi (predictor, tridiagonal, gaussel Thomas in FP64, bcycle, vbcw)
//                                          stepwi.f90:308-548, gaussel.f90:169-262
//   diverpiv, advbspi('fore'), steppi + bcycle + vbcp
//                                          advbspi.f90:167-182, steppi.f90:211-316
//
// Design: one thread owns one (i,j) column of a TX x TY tile and the block
// marches k upward.  Each level's old u, v, w, p' planes (tile + 1-2 halo)
// are staged in shared memory; the divergence-damped pressure, the new u
// and v, the horizontal and vertical divergences, the w right-hand side
// and the forward Thomas elimination are formed on the way up.  The
// modified right-hand side (double) and the backward pressure tendency
// (float) of every level are kept in shared memory; the way down does the
// back substitution and the p' update.  Old and new time levels are
// separate buffers (ping-pong across substeps), so halo reads never see a
// neighbour tile's new values.  Each field is read once and written once
// per substep from HBM, apart from tile-halo re-reads that L1/L2 serve.
//
// With a horizontally uniform base state (idealized, flat terrain) the
// tridiagonal coefficients depend on k only, so the elimination factors
// c'_k and 1/(b_k - a_k c'_{k-1}) are formed once per dts on the host and
// read as 1-D columns.
#include <cuda_runtime.h>
#include <cstdio>
#include "common.cuh"
#include "hevi.cuh"

namespace cress {

namespace {

template <int TX, int TY>
struct HeviSmem {
  float u[TY + 2][TX + 3];   // old u  at i in [i0-1, i0+TX+1], j in [j0-1, j0+TY]
  float v[TY + 3][TX + 2];   // old v  at i in [i0-1, i0+TX],   j in [j0-1, j0+TY+1]
  float w[2][TY + 2][TX + 2];// old w  at levels k (slot k&1) and k+1
  float p[TY + 2][TX + 2];   // old p' at level k
  float t3h[TY + 2][TX + 2]; // jcb*(p' + divch*div3d/jcb)  (pgrad.f90:341,363)
  float un[TY][TX + 1];      // new u on the tile's x faces
  float vn[TY + 1][TX];      // new v on the tile's y faces
};

template <int TX, int TY>
__global__ void __launch_bounds__(TX * TY)
k_hevi_substep(const HeviArgs a) {
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * TX + tx;
  const int NT = TX * TY;
  const int i0 = 2 + blockIdx.x * TX, j0 = 2 + blockIdx.y * TY;
  const int ilast = min(i0 + TX - 1, ni - 2), jlast = min(j0 + TY - 1, nj - 2);
  const int i = i0 + tx, j = j0 + ty;
  const bool own = (i <= ilast) && (j <= jlast);

  __shared__ HeviSmem<TX, TY> s;
  extern __shared__ __align__(16) unsigned char dsm[];
  // Column store: forward-eliminated RHS (double, levels 3..nk-2) and the
  // backward pressure tendency fp (float, levels 2..nk-2).
  double* fcol = reinterpret_cast<double*>(dsm);
  float* fpcol = reinterpret_cast<float*>(dsm + sizeof(double) * (size_t)(nk - 4) * NT);

  const float* __restrict__ col = a.col;   // 1-D base columns, [field*(nk+1) + k]
  const float* __restrict__ uo = a.u_old;
  const float* __restrict__ vo = a.v_old;
  const float* __restrict__ wo = a.w_old;
  const float* __restrict__ po = a.p_old;
  const int ncol = nk + 1;
#define COL(f, k) __ldg(col + (f) * ncol + (k))

  // Extents of the staged planes (clipped for partial edge tiles).
  const int ux = ilast - i0 + 4, uy = jlast - j0 + 3;   // u plane
  const int vx = ilast - i0 + 3, vy = jlast - j0 + 4;   // v plane
  const int sx = ilast - i0 + 3, sy = jlast - j0 + 3;   // w, p planes and the div3d region

  auto load_w = [&](int k, int slot) {
    for (int n = tid; n < sx * sy; n += NT) {
      int x = n % sx, y = n / sx;
      s.w[slot][y][x] = wo[g.at(i0 - 1 + x, j0 - 1 + y, k)];
    }
  };

  load_w(2, 0);

  float t3v_prev = 0.f, fpdvj_prev = 0.f, wb8s_prev = 0.f;
  double fprev = 0.0;
  const float dts = a.dts;
  const float weic1m = 1.f - a.weicoe;

  for (int k = 2; k <= nk - 2; ++k) {
    const int sk = k & 1, sk1 = (k + 1) & 1;
    // --- stage old planes at level k (w at k+1) --------------------------
    for (int n = tid; n < ux * uy; n += NT) {
      int x = n % ux, y = n / ux;
      s.u[y][x] = uo[g.at(i0 - 1 + x, j0 - 1 + y, k)];
    }
    for (int n = tid; n < vx * vy; n += NT) {
      int x = n % vx, y = n / vx;
      s.v[y][x] = vo[g.at(i0 - 1 + x, j0 - 1 + y, k)];
    }
    for (int n = tid; n < sx * sy; n += NT) {
      int x = n % sx, y = n / sx;
      s.p[y][x] = po[g.at(i0 - 1 + x, j0 - 1 + y, k)];
      s.w[sk1][y][x] = wo[g.at(i0 - 1 + x, j0 - 1 + y, k + 1)];
    }
    __syncthreads();

    // --- diver3d + divergence damping on the tile + 1 halo ---------------
    const float rst8u = COL(C_RST8U, k), rst8v = COL(C_RST8V, k);
    const float rst8wk = COL(C_RST8W, k), rst8wk1 = COL(C_RST8W, k + 1);
    const float jcbk = COL(C_JCB, k);
    const float j8wk = COL(C_JCB8W, k), j8wk1 = COL(C_JCB8W, k + 1);
    for (int n = tid; n < sx * sy; n += NT) {
      int x = n % sx, y = n / sx;
      float wck = s.w[sk][y][x], wck1 = s.w[sk1][y][x];
      if (a.sthopt) { wck = wck / j8wk; wck1 = wck1 / j8wk1; }                     // phy2cnt.f90:219
      float div = (rst8wk * wck - rst8wk1 * wck1) * a.dziv +
                  ((rst8u * s.u[y][x] - rst8u * s.u[y][x + 1]) * a.dxiv +
                   (rst8v * s.v[y][x] - rst8v * s.v[y + 1][x]) * a.dyiv);         // diver3d.f90:318
      float pp = s.p[y][x];
      float th = (a.divopt == 2) ? pp + a.divch * div / jcbk                        // pgrad.f90:341
               : (a.divopt >= 1) ? pp + a.divcv * jcbk * div : pp;                 // pgrad.f90:300
      s.t3h[y][x] = jcbk * th;                                                      // pgrad.f90:363
    }
    // The own column's vertically damped pressure (pgrad.f90:300), kept in
    // a register for wpg at this level and the next.
    float t3v = 0.f;
    if (own) {
      const int x = tx + 1, y = ty + 1;
      float wck = s.w[sk][y][x], wck1 = s.w[sk1][y][x];
      if (a.sthopt) { wck = wck / j8wk; wck1 = wck1 / j8wk1; }
      float div = (rst8wk * wck - rst8wk1 * wck1) * a.dziv +
                  ((rst8u * s.u[y][x] - rst8u * s.u[y][x + 1]) * a.dxiv +
                   (rst8v * s.v[y][x] - rst8v * s.v[y + 1][x]) * a.dyiv);
      float pp = s.p[y][x];
      t3v = (a.divopt >= 1) ? pp + a.divcv * jcbk * div : pp;
    }
    __syncthreads();

    // --- stepuv: new u on faces i0..ilast+1, new v on faces j0..jlast+1 ---
    if (own) {
      const long long id = g.at(i, j, k);
      float upg = (s.t3h[ty + 1][tx] - s.t3h[ty + 1][tx + 1]) * a.dxiv;            // pgrad.f90:379
      float un = s.u[ty + 1][tx + 1] + dts * (__ldg(a.ufrc + id) + upg) / rst8u;  // stepuv.f90:294
      float vpg = (s.t3h[ty][tx + 1] - s.t3h[ty + 1][tx + 1]) * a.dyiv;            // pgrad.f90:389
      float vn = s.v[ty + 1][tx + 1] + dts * (__ldg(a.vfrc + id) + vpg) / rst8v;  // stepuv.f90:304
      s.un[ty][tx] = un;
      s.vn[ty][tx] = vn;
      store_periodic(a.u_new, g, STAG_U, i, j, k, un);
      store_periodic(a.v_new, g, STAG_V, i, j, k, vn);
      if (k == 2) { store_periodic(a.u_new, g, STAG_U, i, j, 1, un);            // vbcu.f90:120
                    store_periodic(a.v_new, g, STAG_V, i, j, 1, vn); }
      if (k == nk - 2) { store_periodic(a.u_new, g, STAG_U, i, j, nk - 1, un);  // vbcu.f90:134
                         store_periodic(a.v_new, g, STAG_V, i, j, nk - 1, vn); }
      if (i == ilast) {  // east face of the tile
        const int xe = tx + 2;
        float upg2 = (s.t3h[ty + 1][xe - 1] - s.t3h[ty + 1][xe]) * a.dxiv;
        float un2 = s.u[ty + 1][xe] + dts * (__ldg(a.ufrc + id + 1) + upg2) / rst8u;
        s.un[ty][tx + 1] = un2;
        if (i + 1 == ni - 1) {   // the reference also updates u(ni-1) (stepuv.f90:293)
          store_periodic(a.u_new, g, STAG_U, i + 1, j, k, un2);
          if (k == 2) store_periodic(a.u_new, g, STAG_U, i + 1, j, 1, un2);
          if (k == nk - 2) store_periodic(a.u_new, g, STAG_U, i + 1, j, nk - 1, un2);
        }
      }
      if (j == jlast) {  // north face of the tile
        const int yn = ty + 2;
        float vpg2 = (s.t3h[yn - 1][tx + 1] - s.t3h[yn][tx + 1]) * a.dyiv;
        float vn2 = s.v[yn][tx + 1] + dts * (__ldg(a.vfrc + id + g.px) + vpg2) / rst8v;
        s.vn[ty + 1][tx] = vn2;
        if (j + 1 == nj - 1) {
          store_periodic(a.v_new, g, STAG_V, i, j + 1, k, vn2);
          if (k == 2) store_periodic(a.v_new, g, STAG_V, i, j + 1, 1, vn2);
          if (k == nk - 2) store_periodic(a.v_new, g, STAG_V, i, j + 1, nk - 1, vn2);
        }
      }
    }
    __syncthreads();

    // --- column work: fp (back), fw, w predictor, forward elimination -----
    if (own) {
      const long long id = g.at(i, j, k);
      const float jcb8u = COL(C_JCB8U, k), jcb8v = COL(C_JCB8V, k);
      const float rcsq = COL(C_RCSQ, k), rst = COL(C_RST, k), rbr = COL(C_RBR, k);
      float phd = (jcb8u * s.un[ty][tx] - jcb8u * s.un[ty][tx + 1]) * a.dxiv +
                  (jcb8v * s.vn[ty][tx] - jcb8v * s.vn[ty + 1][tx]) * a.dyiv;     // diver2d.f90:288
      phd = rcsq * phd;                                                              // diverpih.f90:208
      const float wk = s.w[sk][ty + 1][tx + 1], wk1 = s.w[sk1][ty + 1][tx + 1];
      const float pvd = rcsq * (wk - wk1) * a.dziv;                                  // diverpiv.f90:124
      const float fp = __ldg(a.pfrc + id) + phd +
                       weic1m * (a.g05 * (wk + wk1) * rst + pvd);                    // advbspi.f90:158
      fpcol[(k - 2) * NT + tid] = fp;
      const float fpdvj = fp / jcbk;                                                 // pgradiv.f90:149
      const float wb8s = (s.p[ty + 1][tx + 1] * rst + fp * rbr * a.dtw) / rcsq * a.g05n;  // buoywsi.f90:171
      if (k >= 3) {
        const float wpg = (t3v_prev - t3v) * a.dziv;                                 // pgrad.f90:320
        float fw = __ldg(a.wfrc + id) + wpg + (fpdvj_prev - fpdvj) * a.dtdzw;        // pgradiv.f90:163
        if (a.buyopt == 1) fw = fw + (wb8s_prev + wb8s);                             // buoywsi.f90:205
        const float wrhs = wk + dts * fw / COL(C_RST8W, k);                          // stepwi.f90:325
        // gaussel.f90:189-240 in double with precomputed 1-D factors
        const double rr = (double)__ldg(a.thom_rr + k), aa = __ldg(a.thom_aa + k);
        double f = (k == 3) ? (double)wrhs * aa : ((double)wrhs - rr * fprev) * aa;
        fcol[(k - 3) * NT + tid] = f;
        fprev = f;
      }
      t3v_prev = t3v;
      fpdvj_prev = fpdvj;
      wb8s_prev = wb8s;
    }
    // The next iteration's staging overwrites s.u/s.v/s.p; s.un/s.vn are
    // rewritten only after two more barriers.
    __syncthreads();
  }

  // --- way down: back substitution, w BCs, p' update ----------------------
  if (own) {
    const float dziv = a.dziv;
    float wup = 0.f;          // w(k+1) as float; w(nk-1)=0 (vbcw.f90:481)
    double wupd = 0.0;        // w(k+1) as double for the recurrence
    float w3 = 0.f, wkend = 0.f, p2 = 0.f, p3 = 0.f, pkend = 0.f;
    for (int k = nk - 2; k >= 2; --k) {
      float wk;
      if (k >= 3) {
        double f = fcol[(k - 3) * NT + tid];
        double wd = (k == nk - 2) ? f : f - __ldg(a.thom_cp + k) * wupd;            // gaussel.f90:254
        wupd = wd;
        wk = (float)wd;
        store_periodic(a.w_new, g, STAG_S, i, j, k, wk);
        if (k == 3) w3 = wk;
        if (k == nk - 2) wkend = wk;
      } else {
        wk = 0.f;             // vbcw.f90:317 (flat terrain)
      }
      const long long id = g.at(i, j, k);
      const float rcsq = COL(C_RCSQ, k), rst = COL(C_RST, k), jcb = COL(C_JCB, k);
      const float pvd = rcsq * (wk - wup) * dziv;                                     // diverpiv.f90:124
      const float fp = fpcol[(k - 2) * NT + tid] + a.weicoe * (a.g05 * (wk + wup) * rst + pvd);  // advbspi.f90:175
      const float pn = po[id] + dts * fp / jcb;                                      // steppi.f90:217
      store_periodic(a.p_new, g, STAG_S, i, j, k, pn);
      if (k == 2) p2 = pn;
      if (k == 3) p3 = pn;
      if (k == nk - 2) pkend = pn;
      wup = wk;
    }
    // vbcw.f90:285,317,471,481 (flat terrain; wc = w / jcb8w when stretched)
    const float j8w3 = COL(C_JCB8W, 3), j8wt = COL(C_JCB8W, nk - 2);
    const float wc3 = a.sthopt ? w3 / j8w3 : w3;
    const float wct = a.sthopt ? wkend / j8wt : wkend;
    store_periodic(a.w_new, g, STAG_S, i, j, 1, -j8w3 * wc3 - 0.f);
    store_periodic(a.w_new, g, STAG_S, i, j, 2, 0.f);
    store_periodic(a.w_new, g, STAG_S, i, j, nk - 1, 0.f);
    store_periodic(a.w_new, g, STAG_S, i, j, nk, -j8wt * wct - 0.f);
    // vbcp.f90:126-160
    store_periodic(a.p_new, g, STAG_S, i, j, 1, (a.bbc == 2) ? 2.f * p2 - p3 : p2);
    store_periodic(a.p_new, g, STAG_S, i, j, nk - 1, pkend);
    // Level nk of u, v, p' is not touched by the small step: carry it over.
    store_periodic(a.p_new, g, STAG_S, i, j, nk, po[g.at(i, j, nk)]);
    store_periodic(a.u_new, g, STAG_U, i, j, nk, uo[g.at(i, j, nk)]);
    store_periodic(a.v_new, g, STAG_V, i, j, nk, vo[g.at(i, j, nk)]);
    if (i == ilast && i + 1 == ni - 1)
      store_periodic(a.u_new, g, STAG_U, i + 1, j, nk, uo[g.at(i + 1, j, nk)]);
    if (j == jlast && j + 1 == nj - 1)
      store_periodic(a.v_new, g, STAG_V, i, j + 1, nk, vo[g.at(i, j + 1, nk)]);
  }
#undef COL
}

template <int TX, int TY>
int launch_hevi_t(const HeviArgs& a, cudaStream_t st) {
  const Grid& g = a.g;
  const int nx = g.ni - 3, ny = g.nj - 3;
  dim3 block(TX, TY);
  dim3 grid((nx + TX - 1) / TX, (ny + TY - 1) / TY);
  size_t dyn = sizeof(double) * (size_t)(g.nk - 4) * TX * TY + sizeof(float) * (size_t)(g.nk - 3) * TX * TY;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_hevi_substep<TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  if (dyn + sizeof(HeviSmem<TX, TY>) > 220 * 1024) return CRESS_E_UNSUPPORTED;
  k_hevi_substep<TX, TY><<<grid, block, dyn, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace

int launch_hevi_substep(const HeviArgs& a, int tile, cudaStream_t st) {
  switch (tile) {
    case 1: return launch_hevi_t<32, 2>(a, st);
    case 2: return launch_hevi_t<32, 8>(a, st);
    case 3: return launch_hevi_t<16, 8>(a, st);
    default: return launch_hevi_t<32, 4>(a, st);
  }
}

}  // namespace cress

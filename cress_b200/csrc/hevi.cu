// Fused HE-VI acoustic substep for sm_100a.
//
// One launch = one pass of s_hevi (SrcOrig/hevi.f90:339-426) for
// impopt=1, gwmopt=0, flat terrain, no map factors, periodic lateral
// boundaries on one GPU, rigid bottom/top (bbc=tbc=2):
//   pgrad + diver3d (divergence damping)   pgrad.f90:251-395, diver3d.f90:182-326
//   stepuv + bcycle + vbcu/vbcv            stepuv.f90:288-424
//   diverpih + diver2d                     diverpih.f90:188-214, diver2d.f90:280-295
//   diverpiv, advbspi('back')              diverpiv.f90:118-130, advbspi.f90:150-165
//   pgradiv, buoywsi                       pgradiv.f90:135-170, buoywsi.f90:153-211
//   stepwi (predictor, tridiagonal, gaussel Thomas in FP64, bcycle, vbcw)
//                                          stepwi.f90:308-548, gaussel.f90:169-262
//   diverpiv, advbspi('fore'), steppi + bcycle + vbcp
//                                          advbspi.f90:167-182, steppi.f90:211-316
//
// Design.  A block owns a 32 x TY tile of (i,j) columns, one thread per
// column, and marches k upward (2.5-D).  For every level one elected thread
// issues eight TMA box loads (old u, v, w, p' with their halos and the four
// forcings) into an S-stage shared-memory ring guarded by mbarriers, so S-2
// levels are in flight while the block computes.  Per level each thread
// forms the divergence-damped pressure of its own column (plus one halo
// point), then, after one barrier, the new u on its west and east faces, the
// new v on its south and north faces, the horizontal divergence of the new
// winds, the backward pressure tendency, the w right-hand side and one step
// of the forward Thomas elimination.  The eliminated right-hand sides stay
// in shared memory as doubles; the backward pressure tendency is parked in
// the new p' array (an L2 round trip that its final value overwrites).  The
// way down does the back substitution, the p' update and the boundary
// rows.  Old and new time levels are separate buffers (ping-pong across
// substeps), so halo reads never see a neighbour tile's new values.
//
// With a horizontally uniform base state the tridiagonal coefficients
// depend on k only: the elimination factors c'_k and 1/(b_k - a_k c'_{k-1})
// come precomputed (double) from the host.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "common.cuh"
#include "hevi.cuh"
#include "tma.cuh"

namespace cress {

namespace {

constexpr int r128(int n) { return (n + 31) / 32 * 32; }  // floats -> multiple of 128 B

// FT: element type of the column store of eliminated right-hand sides
// (double by default; float halves the store and doubles resident blocks,
// with the elimination recurrence itself still in double).  GS: park the
// eliminated right-hand sides (as float) in the new w array instead of
// shared memory; the way down reads each one back just before it writes
// the final w there (an L2 round trip), which frees the block's largest
// shared-memory buffer for more resident blocks.
template <int TY, int S, typename FT = double, bool GS = false>
struct HeviLayout {
  using R = HeviRows<TY>;
  static constexpr int BX = kHeviBoxX;
  static constexpr int oU = 0;
  static constexpr int oV = oU + r128(BX * R::u);
  static constexpr int oW = oV + r128(BX * R::v);
  static constexpr int oP = oW + r128(BX * R::w);
  static constexpr int oUF = oP + r128(BX * R::p);
  static constexpr int oVF = oUF + r128(BX * R::uf);
  static constexpr int oWF = oVF + r128(BX * R::vf);
  static constexpr int oPF = oWF + r128(BX * R::wf);
  static constexpr int stage = oPF + r128(BX * R::pf);  // floats per ring stage
  static constexpr uint32_t tx_bytes =
      4u * BX * (R::u + R::v + R::w + R::p + R::uf + R::vf + R::wf + R::pf);
  static constexpr int t3h_floats = r128((TY + 2) * BX);
  __host__ __device__ static size_t cols_floats(int nk) { return (size_t)((C_NFIELDS * (nk + 1) + 31) / 32 * 32); }
  // ring, t3h (two buffers), columns, mbarriers, the elimination factors
  // (aa, cp as double, rr as float) and the column store
  __host__ __device__ static size_t bytes(int nk) {
    return 4 * ((size_t)S * stage + 2 * (size_t)t3h_floats + cols_floats(nk)) + 8 * (size_t)S +
           16 * (size_t)(nk + 2) + (GS ? 0 : sizeof(FT) * (size_t)(nk - 4) * (kHeviTX * TY)) +
           4 * (size_t)(nk + 2);
  }
};

template <int TY, int S, typename FT, bool GS>
__global__ void __launch_bounds__(kHeviTX * TY, GS ? 24 / TY : 1)
k_hevi_substep(const __grid_constant__ HeviMaps m, const HeviArgs a) {
  using L = HeviLayout<TY, S, FT, GS>;
  constexpr int TX = kHeviTX, BX = kHeviBoxX, NT = TX * TY;
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = 2 + blockIdx.x * TX, j0 = 2 + blockIdx.y * TY;
  const int xb = i0 - 2;  // box x origin (multiple of 32)
  const int ilast = min(i0 + TX - 1, ni - 2), jlast = min(j0 + TY - 1, nj - 2);
  const int i = i0 + tx, j = j0 + ty;
  const bool own = (i <= ilast) && (j <= jlast);
  const int ncol = nk + 1;
  // Columns whose values the periodic wrap also copies into ghost cells.
  const bool edge = (i <= 3) || (i >= ni - 2) || (j <= 3) || (j >= nj - 2);

  extern __shared__ __align__(1024) float smem[];
  float* ring = smem;
  float* t3hb = ring + S * L::stage;               // 2 x [(TY+2)][BX], rows from j0-1, x from i0-2
  float* cols = t3hb + 2 * L::t3h_floats;          // [C_NFIELDS][nk+1]
  uint64_t* bars = reinterpret_cast<uint64_t*>(cols + L::cols_floats(nk));
  double* thd = reinterpret_cast<double*>(bars + S);   // aa[k] then cp[k], k = 0..nk+1
  FT* fcol = reinterpret_cast<FT*>(thd + 2 * (nk + 2));  // [(nk-4)][NT]
  float* thr = reinterpret_cast<float*>(fcol) + (GS ? 0 : (sizeof(FT) / 4) * (size_t)(nk - 4) * NT);  // rr[k]

  for (int n = tid; n < C_NFIELDS * ncol; n += NT) cols[n] = __ldg(a.col + n);
  for (int n = tid; n <= nk + 1; n += NT) {
    thd[n] = __ldg(a.thom_aa + n);
    thd[nk + 2 + n] = __ldg(a.thom_cp + n);
    thr[n] = __ldg(a.thom_rr + n);
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  // Levels 2..nk-1 are staged (w is needed one level above the top update).
  const int klast = nk - 1;
  int issued = 1;   // highest level thread 0 has issued
  auto issue = [&](int k) {
    issued = k;
    const int s = (k - 2) % S;
    float* st = ring + s * L::stage;
    uint64_t* bar = &bars[s];
    const int z = k - 1;
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
    for (int k = 2; k <= min(S, klast); ++k) issue(k);

  // Halo points of the damped-pressure plane: the rows south/north of the
  // tile and the columns west/east of it (2*TX + 2*TY points, spread over
  // the threads; box coordinates).
  constexpr int NH = 2 * TX + 2 * TY;
  auto halo_xy = [&](int n, int& hx, int& hy) {
    if (n < TX) { hx = n + 2; hy = 0; }
    else if ((n -= TX) < TX) { hx = n + 2; hy = TY + 1; }
    else if ((n -= TX) < TY) { hx = 1; hy = n + 1; }
    else { n -= TY; hx = TX + 2; hy = n + 1; }
  };
  const int ox = tx + 2, oy = ty + 1;  // own column in the boxes that start at j0-1
  const float dts = a.dts, dxiv = a.dxiv, dyiv = a.dyiv, dziv = a.dziv;
  const float weic1m = 1.f - a.weicoe;
  float t3v_prev = 0.f, fpdvj_prev = 0.f, wb8s_prev = 0.f;
  double fprev = 0.0;
  bool fail = false;
  const long long plane = g.plane;
  long long id = g.at(i, j, 2);

  for (int k = 2; k <= nk - 2; ++k, id += plane) {
    // One barrier per level: t3h alternates between two buffers, and the
    // stage of level k-1 is refilled only after this level's barrier, when
    // every thread has finished level k-1.
    float* t3h = t3hb + (k & 1) * L::t3h_floats;
    const int s0 = (k - 2) % S, s1 = (k - 1) % S;
    if (!fail) fail = !mbar_wait(&bars[s0], ((k - 2) / S) & 1);
    if (!fail) fail = !mbar_wait(&bars[s1], ((k - 1) / S) & 1);
    const float* U = ring + s0 * L::stage + L::oU;
    const float* V = ring + s0 * L::stage + L::oV;
    const float* W0 = ring + s0 * L::stage + L::oW;
    const float* W1 = ring + s1 * L::stage + L::oW;
    const float* P = ring + s0 * L::stage + L::oP;
    const float* UF = ring + s0 * L::stage + L::oUF;
    const float* VF = ring + s0 * L::stage + L::oVF;
    const float* WF = ring + s0 * L::stage + L::oWF;
    const float* PF = ring + s0 * L::stage + L::oPF;
    const float rst8u = cols[C_RST8U * ncol + k], rst8v = cols[C_RST8V * ncol + k];
    const float rst8wk = cols[C_RST8W * ncol + k], rst8wk1 = cols[C_RST8W * ncol + k + 1];
    const float jcbk = cols[C_JCB * ncol + k], ijcbk = cols[C_IJCB * ncol + k];
    const float irst8u = cols[C_IRST8U * ncol + k], irst8v = cols[C_IRST8V * ncol + k];
    const float ij8wk = cols[C_IJCB8W * ncol + k], ij8wk1 = cols[C_IJCB8W * ncol + k + 1];

    // diver3d.f90:318 (with phy2cnt.f90:219 for the contravariant w)
    auto div3d_at = [&](int x, int y) {
      float wck = W0[y * BX + x], wck1 = W1[y * BX + x];
      if (a.sthopt) { wck = wck * ij8wk; wck1 = wck1 * ij8wk1; }
      return (rst8wk * wck - rst8wk1 * wck1) * dziv +
             ((rst8u * U[y * BX + x] - rst8u * U[y * BX + x + 1]) * dxiv +
              (rst8v * V[y * BX + x] - rst8v * V[(y + 1) * BX + x]) * dyiv);
    };
    // pgrad.f90:300,341,363
    auto t3h_of = [&](float div, float pp) {
      float th = (a.divopt == 2) ? pp + a.divch * div * ijcbk
               : (a.divopt >= 1) ? pp + a.divcv * jcbk * div : pp;
      return jcbk * th;
    };
    const float divo = div3d_at(ox, oy);
    const float ppo = P[oy * BX + ox];
    t3h[oy * BX + ox] = t3h_of(divo, ppo);
    const float t3v = (a.divopt >= 1) ? ppo + a.divcv * jcbk * divo : ppo;  // pgrad.f90:300
    for (int n = tid; n < NH; n += NT) {
      int hx, hy;
      halo_xy(n, hx, hy);
      t3h[hy * BX + hx] = t3h_of(div3d_at(hx, hy), P[hy * BX + hx]);
    }
    __syncthreads();
    if (tid == 0 && !fail && k + S - 1 <= klast) {   // refill only after its copy was seen to land
      fence_proxy_async_smem();
      issue(k + S - 1);
    }

    // stepuv.f90:294,304 with pgrad.f90:379,389 on the four faces of the column
    const float tc = t3h[oy * BX + ox];
    const float un0 = U[oy * BX + ox] + dts * (UF[ty * BX + ox] + (t3h[oy * BX + ox - 1] - tc) * dxiv) * irst8u;
    const float un1 = U[oy * BX + ox + 1] + dts * (UF[ty * BX + ox + 1] + (tc - t3h[oy * BX + ox + 1]) * dxiv) * irst8u;
    const float vn0 = V[oy * BX + ox] + dts * (VF[ty * BX + ox] + (t3h[(oy - 1) * BX + ox] - tc) * dyiv) * irst8v;
    const float vn1 = V[(oy + 1) * BX + ox] + dts * (VF[(ty + 1) * BX + ox] + (tc - t3h[(oy + 1) * BX + ox]) * dyiv) * irst8v;

    if (own) {
      if (edge) {
        store_periodic(a.u_new, g, STAG_U, i, j, k, un0);
        store_periodic(a.v_new, g, STAG_V, i, j, k, vn0);
      } else {
        a.u_new[id] = un0;
        a.v_new[id] = vn0;
      }
      if (k == 2) { store_periodic(a.u_new, g, STAG_U, i, j, 1, un0);          // vbcu.f90:120
                    store_periodic(a.v_new, g, STAG_V, i, j, 1, vn0); }
      if (k == nk - 2) { store_periodic(a.u_new, g, STAG_U, i, j, nk - 1, un0); // vbcu.f90:134
                         store_periodic(a.v_new, g, STAG_V, i, j, nk - 1, vn0); }
      if (i == ilast && i + 1 == ni - 1) {  // stepuv.f90:293 updates u(ni-1) too
        store_periodic(a.u_new, g, STAG_U, i + 1, j, k, un1);
        if (k == 2) store_periodic(a.u_new, g, STAG_U, i + 1, j, 1, un1);
        if (k == nk - 2) store_periodic(a.u_new, g, STAG_U, i + 1, j, nk - 1, un1);
      }
      if (j == jlast && j + 1 == nj - 1) {  // stepuv.f90:302 updates v(nj-1) too
        store_periodic(a.v_new, g, STAG_V, i, j + 1, k, vn1);
        if (k == 2) store_periodic(a.v_new, g, STAG_V, i, j + 1, 1, vn1);
        if (k == nk - 2) store_periodic(a.v_new, g, STAG_V, i, j + 1, nk - 1, vn1);
      }

      const float jcb8u = cols[C_JCB8U * ncol + k], jcb8v = cols[C_JCB8V * ncol + k];
      const float rcsq = cols[C_RCSQ * ncol + k], rst = cols[C_RST * ncol + k];
      const float rbr = cols[C_RBR * ncol + k];
      float phd = (jcb8u * un0 - jcb8u * un1) * dxiv + (jcb8v * vn0 - jcb8v * vn1) * dyiv;  // diver2d.f90:288
      phd = rcsq * phd;                                                                       // diverpih.f90:208
      const float wk = W0[oy * BX + ox], wk1 = W1[oy * BX + ox];
      const float pvd = rcsq * (wk - wk1) * dziv;                                             // diverpiv.f90:124
      const float fp = PF[ty * BX + ox] + phd + weic1m * (a.g05 * (wk + wk1) * rst + pvd);    // advbspi.f90:158
      a.p_new[id] = fp;  // parked until the way down
      const float fpdvj = fp * ijcbk;                                                          // pgradiv.f90:149
      const float wb8s = (ppo * rst + fp * rbr * a.dtw) * cols[C_IRCSQ * ncol + k] * a.g05n;                      // buoywsi.f90:171
      if (k >= 3) {
        const float wpg = (t3v_prev - t3v) * dziv;                                            // pgrad.f90:320
        float fw = WF[ty * BX + ox] + wpg + (fpdvj_prev - fpdvj) * a.dtdzw;                   // pgradiv.f90:163
        if (a.buyopt == 1) fw = fw + (wb8s_prev + wb8s);                                      // buoywsi.f90:205
        const float wrhs = wk + dts * fw * cols[C_IRST8W * ncol + k];                          // stepwi.f90:325
        // gaussel.f90:189-240 in double with the 1-D factors
        const double rr = (double)thr[k], aa = thd[k];
        const double f = (k == 3) ? (double)wrhs * aa : ((double)wrhs - rr * fprev) * aa;
        if constexpr (GS) a.w_new[id] = (float)f;
        else fcol[(k - 3) * NT + tid] = (FT)f;
        fprev = f;
      }
      t3v_prev = t3v;
      fpdvj_prev = fpdvj;
      wb8s_prev = wb8s;
    }
  }

  if (__syncthreads_or(fail)) {
    // A bounded wait gave up: record it, let the copies still in flight
    // land (bounded again) so no TMA write outlives the block, and leave.
    if (tid == 0) {
      atomicExch(a.err, 1);
      for (int s = 0; s < S; ++s) {
        int kl = -1;
        for (int k = 2; k <= issued; ++k)
          if ((k - 2) % S == s) kl = k;
        if (kl >= 0) mbar_wait(&bars[s], ((kl - 2) / S) & 1);
      }
    }
    return;
  }

  // --- way down: back substitution, w boundary rows, p' update ------------
  if (own) {
    float wup = 0.f;          // w(k+1) as float; w(nk-1) = 0 (vbcw.f90:481)
    double wupd = 0.0;        // w(k+1) as double for the recurrence
    float w3 = 0.f, wkend = 0.f, p2 = 0.f, p3 = 0.f, pkend = 0.f;
    long long idk = g.at(i, j, nk - 2);
    // loads run two levels ahead of their use (parked fp, old p', parked f)
    float fp0 = a.p_new[idk], po0 = a.p_old[idk], fp1 = 0.f, po1 = 0.f;
    float f0 = GS ? a.w_new[idk] : 0.f, f1 = 0.f;
    if (nk - 3 >= 2) { fp1 = a.p_new[idk - plane]; po1 = a.p_old[idk - plane]; }
    if (GS && nk - 3 >= 3) f1 = a.w_new[idk - plane];
    for (int k = nk - 2; k >= 2; --k, idk -= plane) {
      const float fpb = fp0, po = po0, fg = f0;
      fp0 = fp1; po0 = po1; f0 = f1;
      if (k - 2 >= 2) { fp1 = a.p_new[idk - 2 * plane]; po1 = a.p_old[idk - 2 * plane]; }
      if (GS && k - 2 >= 3) f1 = a.w_new[idk - 2 * plane];
      float wk;
      if (k >= 3) {
        const double f = GS ? (double)fg : (double)fcol[(k - 3) * NT + tid];
        const double wd = (k == nk - 2) ? f : f - thd[nk + 2 + k] * wupd;                     // gaussel.f90:254
        wupd = wd;
        wk = (float)wd;
        if (edge) store_periodic(a.w_new, g, STAG_S, i, j, k, wk);
        else a.w_new[idk] = wk;
        if (k == 3) w3 = wk;
        if (k == nk - 2) wkend = wk;
      } else {
        wk = 0.f;  // vbcw.f90:317 (flat terrain)
      }
      const float rcsq = cols[C_RCSQ * ncol + k], rst = cols[C_RST * ncol + k];
      const float pvd = rcsq * (wk - wup) * dziv;                                              // diverpiv.f90:124
      const float fp = fpb + a.weicoe * (a.g05 * (wk + wup) * rst + pvd);                        // advbspi.f90:175
      const float pn = po + dts * fp * cols[C_IJCB * ncol + k];                                                     // steppi.f90:217
      if (edge) store_periodic(a.p_new, g, STAG_S, i, j, k, pn);
      else a.p_new[idk] = pn;
      if (k == 2) p2 = pn;
      if (k == 3) p3 = pn;
      if (k == nk - 2) pkend = pn;
      wup = wk;
    }
    // vbcw.f90:285,317,471,481 (flat terrain; wc = w / jcb8w when stretched)
    const float j8w3 = cols[C_JCB8W * ncol + 3], j8wt = cols[C_JCB8W * ncol + nk - 2];
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
    store_periodic(a.p_new, g, STAG_S, i, j, nk, a.p_old[g.at(i, j, nk)]);
    store_periodic(a.u_new, g, STAG_U, i, j, nk, a.u_old[g.at(i, j, nk)]);
    store_periodic(a.v_new, g, STAG_V, i, j, nk, a.v_old[g.at(i, j, nk)]);
    if (i == ilast && i + 1 == ni - 1)
      store_periodic(a.u_new, g, STAG_U, i + 1, j, nk, a.u_old[g.at(i + 1, j, nk)]);
    if (j == jlast && j + 1 == nj - 1)
      store_periodic(a.v_new, g, STAG_V, i, j + 1, nk, a.v_old[g.at(i, j + 1, nk)]);
  }
}

template <int TY, int S, typename FT, bool GS = false>
int launch_t(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st) {
  using L = HeviLayout<TY, S, FT, GS>;
  const Grid& g = a.g;
  const int nx = g.ni - 3, ny = g.nj - 3;
  const size_t bytes = L::bytes(g.nk);
  if (bytes > 227 * 1024) return CRESS_E_UNSUPPORTED;
  if (cudaFuncSetAttribute(k_hevi_substep<TY, S, FT, GS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)bytes) != cudaSuccess)
    return CRESS_E_CUDA;
  dim3 block(kHeviTX, TY);
  dim3 grid((nx + kHeviTX - 1) / kHeviTX, (ny + TY - 1) / TY);
  k_hevi_substep<TY, S, FT, GS><<<grid, block, bytes, st>>>(maps, a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace

// Tile ids.  0 (the default): k_hevi2 (hevi2.cu), 32 x 8 columns per block
// with two rows per thread; 11: the same with a 3-stage ring and the level
// table read from global memory (more resident blocks).  10: 32 x 4 columns, 4-stage ring, the
// eliminated right-hand sides parked (float) in the new w array; 6: the
// same with a 5-stage ring; 7 and 8: 32 x 8 and 32 x 2.  1, 2 and 9 keep
// them in shared memory as float (32 x 2, 32 x 8, 32 x 4); 3-5 as double
// (both recurrences always run in double).
int hevi_tile_rows(int tile) {
  switch (tile) {
    case 0: case 11: case 12: case 13: return 8;
    case 1: case 4: case 8: return 2;
    case 2: case 5: case 7: return 8;
    default: return 4;
  }
}

int launch_hevi2(const HeviArgs& a, const HeviMaps& maps, int variant, cudaStream_t st);

int launch_hevi_substep(const HeviArgs& a, const HeviMaps& maps, int tile, cudaStream_t st) {
  switch (tile) {
    case 0: return launch_hevi2(a, maps, 0, st);
    case 11: return launch_hevi2(a, maps, 1, st);
    case 12: return launch_hevi3(a, maps, st);
    case 13: return launch_hevi4(a, maps, st);
    case 1: return launch_t<2, 5, float>(a, maps, st);
    case 2: return launch_t<8, 4, float>(a, maps, st);
    case 3: return launch_t<4, 5, double>(a, maps, st);
    case 4: return launch_t<2, 6, double>(a, maps, st);
    case 5: return launch_t<8, 4, double>(a, maps, st);
    case 6: return launch_t<4, 5, float, true>(a, maps, st);
    case 7: return launch_t<8, 5, float, true>(a, maps, st);
    case 8: return launch_t<2, 6, float, true>(a, maps, st);
    case 9: return launch_t<4, 4, float>(a, maps, st);
    default: return launch_t<4, 4, float, true>(a, maps, st);
  }
}

}  // namespace cress

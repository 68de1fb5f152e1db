// Fused HE-VI acoustic substep for sm_100a, two rows per thread (the
// default tile).  Same operators, order of terms and boundary rules as
// k_hevi_substep (hevi.cu: s_hevi, SrcOrig/hevi.f90:339-426, impopt=1,
// flat terrain, periodic lateral boundaries, rigid lid):
//   pgrad + diver3d, stepuv, diverpih + diver2d, diverpiv, advbspi,
//   pgradiv, buoywsi, stepwi with the FP64 Thomas solve (gaussel), steppi.
//
// Design.  A block of 32 x 4 threads owns a 32 x 8 tile of columns; thread
// (tx, ty) owns the columns (i0+tx, j0+2ty) and (i0+tx, j0+2ty+1) and
// marches both up k, then down.  Levels stream through an S-stage TMA ring
// as in k_hevi_substep.  Per level and thread:
//   * the damped pressure of its two columns (registers and shared memory)
//     plus at most one of the 80 halo points of the tile;
//   * the west u face of each column; the east face is the west face of
//     the next lane (a shuffle), only lane 31 forms its own;
//   * three v faces (south of the first row, between the rows, north of the
//     second), where one thread per row would form four;
//   * two independent Thomas recurrences (instruction-level parallelism).
// The two rows' single-precision arithmetic runs as packed FP32x2
// instructions (f2.cuh), one instruction for both rows.  Per-level constants come from a k-major table in shared memory, so each
// is one load at a fixed offset.  Eliminated right-hand sides are parked
// (float) in the new w array and the backward pressure tendency in the new
// p' array, as in the GS variant of k_hevi_substep.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>
#include "common.cuh"
#include "f2.cuh"
#include "hevi.cuh"
#include "tma.cuh"

namespace cress {

namespace {

constexpr int kH2TY = 8;      // tile rows
constexpr int kH2Rows = 4;    // thread rows (two tile rows each)
constexpr int kHNF = 24;      // stride (floats) of the k-major column table (>= C_NFIELDS)

__host__ __device__ constexpr int r128h(int n) { return (n + 31) / 32 * 32; }

template <int S>
struct H2Layout {
  using R = HeviRows<kH2TY>;
  static constexpr int BX = kHeviBoxX;
  static constexpr int oU = 0;
  static constexpr int oV = oU + r128h(BX * R::u);
  static constexpr int oW = oV + r128h(BX * R::v);
  static constexpr int oP = oW + r128h(BX * R::w);
  static constexpr int oUF = oP + r128h(BX * R::p);
  static constexpr int oVF = oUF + r128h(BX * R::uf);
  static constexpr int oWF = oVF + r128h(BX * R::vf);
  static constexpr int oPF = oWF + r128h(BX * R::wf);
  static constexpr int stage = oPF + r128h(BX * R::pf);
  static constexpr uint32_t tx_bytes =
      4u * BX * (R::u + R::v + R::w + R::p + R::uf + R::vf + R::wf + R::pf);
  static constexpr int t3h_floats = r128h((kH2TY + 2) * BX);
  __host__ __device__ static int cols_floats(int nk) { return r128h(kHNF * (nk + 2)); }
  // ring, t3h (two buffers), k-major columns, mbarriers, aa and cp
  // (double), rr (float); with the level table in global memory (GT) only
  // the ring, t3h and the mbarriers
  __host__ __device__ static size_t bytes(int nk, bool gt) {
    if (gt) return 4 * ((size_t)S * stage + 2 * (size_t)t3h_floats) + 8 * (size_t)S;
    return 4 * ((size_t)S * stage + 2 * (size_t)t3h_floats + (size_t)cols_floats(nk)) + 8 * (size_t)S +
           16 * (size_t)(nk + 2) + 4 * (size_t)(nk + 2);
  }
};

// DIV = divopt, STH = stretched grid (sthopt != 0), BUY = buyopt == 1: the
// options are template parameters, so the level loop carries no branches
// on them.  GT: the per-level columns and the elimination factors are read
// from global memory (the level table, a.lvl) instead of being copied into
// shared memory, which leaves room for more resident blocks.
// One tile (bx, by) of one substep; m and a stay in the memory they came
// from (kernel parameters, or an ensemble's job array in global memory).
template <int S, int DIV, bool STH, bool BUY, bool GT>
__device__ __forceinline__ void hevi2_tile(const HeviMaps& m, const HeviArgs& a, int bx, int by) {
  using L = H2Layout<S>;
  constexpr int TX = kHeviTX, TY = kH2TY, BX = kHeviBoxX, NT = TX * kH2Rows;
  const unsigned full = 0xffffffffu;
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = 2 + bx * TX, j0 = 2 + by * TY;
  const int xb = i0 - 2;  // box x origin (multiple of 32)
  const int ilast = min(i0 + TX - 1, ni - 2), jlast = min(j0 + TY - 1, nj - 2);
  const int i = i0 + tx, jA = j0 + 2 * ty, jB = jA + 1;
  const bool ownA = (i <= ilast) && (jA <= jlast), ownB = (i <= ilast) && (jB <= jlast);
  const int ncol = nk + 1;
  // Columns whose values the periodic wrap also copies into ghost cells.
  const bool ei = (i <= 3) || (i >= ni - 2);
  const bool edgeA = ei || (jA <= 3) || (jA >= nj - 2), edgeB = ei || (jB <= 3) || (jB >= nj - 2);
  // the faces stepuv also updates at i = ni-1 and j = nj-1 (stepuv.f90:293,302)
  const bool xlast = (i == ilast) && (i + 1 == ni - 1);
  const bool ylastA = (jA == jlast) && (jA + 1 == nj - 1), ylastB = (jB == jlast) && (jB + 1 == nj - 1);

  extern __shared__ __align__(1024) float smem[];
  float* ring = smem;
  float* t3hb = ring + S * L::stage;          // 2 x [(TY+2)][BX], rows from j0-1, x from i0-2
  float* cols = t3hb + 2 * L::t3h_floats;     // cols[k * kHNF + field] (shared-table variant)
  uint64_t* bars = reinterpret_cast<uint64_t*>(GT ? cols : cols + L::cols_floats(nk));
  double* thd = reinterpret_cast<double*>(bars + S);       // aa[k] then cp[k], k = 0..nk+1
  float* thr = reinterpret_cast<float*>(thd + 2 * (nk + 2));  // rr[k]
  if constexpr (!GT) {
    for (int n = tid; n < C_NFIELDS * ncol; n += NT) {
      const int f = n / ncol, kk = n - f * ncol;
      cols[kk * kHNF + f] = __ldg(a.col + n);
    }
    for (int n = tid; n <= nk + 1; n += NT) {
      thd[n] = __ldg(a.thom_aa + n);
      thd[nk + 2 + n] = __ldg(a.thom_cp + n);
      thr[n] = __ldg(a.thom_rr + n);
    }
  }
  // column field f of level kk, and the elimination factors
  auto CK = [&](int kk, int f) { return GT ? __ldg(a.lvl + kk * kLevelStride + f) : cols[kk * kHNF + f]; };
  auto TH_AA = [&](int kk) { return GT ? __ldg(a.thom_aa + kk) : thd[kk]; };
  auto TH_CP = [&](int kk) { return GT ? __ldg(a.thom_cp + kk) : thd[nk + 2 + kk]; };
  auto TH_RR = [&](int kk) { return GT ? __ldg(a.thom_rr + kk) : thr[kk]; };
  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  // Levels 2..nk-1 are staged (w is needed one level above the top update).
  // Thread 0 issues them in order; `issued` is the highest level issued.
  const int klast = nk - 1;
  int issued = 1;
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

  // Halo point of the damped-pressure plane handled by this thread (box
  // coordinates): rows south/north of the tile, columns west/east of it.
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
  const float weic1m = 1.f - a.weicoe;
  F2 t3v_prev = f2(0.f), fpdvj_prev = f2(0.f), wb8s_prev = f2(0.f);   // rows A, B
  double fA_prev = 0.0, fB_prev = 0.0;
  bool fail = false;
  // 32-bit element indices (the launcher checks that every field fits)
  const int plane = (int)g.plane, px = g.px;
  int idA = (int)g.at(i, jA, 2);

  for (int k = 2; k <= nk - 2; ++k, idA += plane) {
    const int idB = idA + px;
    // One barrier per level: t3h alternates between two buffers, and the
    // stage of level k-1 is refilled only after this level's barrier.
    float* t3h = t3hb + (k & 1) * L::t3h_floats;
    const int s0 = (k - 2) % S, s1 = (k - 1) % S;
    if (!fail && k == 2) fail = !mbar_wait(&bars[s0], 0, a.spin);
    if (!fail) fail = !mbar_wait(&bars[s1], ((k - 1) / S) & 1, a.spin);
    const float* st0 = ring + s0 * L::stage;
    const float* U = st0 + L::oU;
    const float* V = st0 + L::oV;
    const float* W0 = st0 + L::oW;
    const float* W1 = ring + s1 * L::stage + L::oW;
    const float* P = st0 + L::oP;
    const float* UF = st0 + L::oUF;
    const float* VF = st0 + L::oVF;
    const float* WF = st0 + L::oWF;
    const float* PF = st0 + L::oPF;
    const float rst8u = CK(k, C_RST8U), rst8v = CK(k, C_RST8V);
    const float rst8wk = CK(k, C_RST8W), rst8wk1 = CK(k + 1, C_RST8W);
    const float jcbk = CK(k, C_JCB), ijcbk = CK(k, C_IJCB);
    const float irst8u = CK(k, C_IRST8U), irst8v = CK(k, C_IRST8V);
    const float ij8wk = CK(k, C_IJCB8W), ij8wk1 = CK(k + 1, C_IJCB8W);

    // diver3d.f90:318 (with phy2cnt.f90:219 for the contravariant w)
    auto div3d_at = [&](int x, int y) {
      float wck = W0[y * BX + x], wck1 = W1[y * BX + x];
      if constexpr (STH) { wck = wck * ij8wk; wck1 = wck1 * ij8wk1; }
      return (rst8wk * wck - rst8wk1 * wck1) * dziv +
             ((rst8u * U[y * BX + x] - rst8u * U[y * BX + x + 1]) * dxiv +
              (rst8v * V[y * BX + x] - rst8v * V[(y + 1) * BX + x]) * dyiv);
    };
    // pgrad.f90:300,341,363
    auto t3h_of = [&](float div, float pp) {
      float th;
      if constexpr (DIV == 2) th = pp + a.divch * div * ijcbk;
      else if constexpr (DIV == 1) th = pp + a.divcv * jcbk * div;
      else th = pp;
      return jcbk * th;
    };
    // rows A and B of the thread packed into the two lanes of F2 (f2.cuh):
    // every operation below is one packed instruction for both rows
    auto col2 = [&](const float* base, int oy) { return f2(base[oy * BX + ox], base[(oy + 1) * BX + ox]); };
    F2 wc0 = col2(W0, oyA), wc1 = col2(W1, oyA);
    if constexpr (STH) { wc0 = wc0 * ij8wk; wc1 = wc1 * ij8wk1; }
    const F2 div = (rst8wk * wc0 - rst8wk1 * wc1) * dziv +
                   ((rst8u * col2(U, oyA) - rst8u * col2(U + 1, oyA)) * dxiv +
                    (rst8v * col2(V, oyA) - rst8v * col2(V + BX, oyA)) * dyiv);      // diver3d.f90:318
    const F2 pp = col2(P, oyA);
    F2 th;                                                                         // pgrad.f90:341,363
    if constexpr (DIV == 2) th = pp + a.divch * div * ijcbk;
    else if constexpr (DIV == 1) th = pp + a.divcv * jcbk * div;
    else th = pp;
    const F2 tc = jcbk * th;
    t3h[oyA * BX + ox] = tc.v.x;
    t3h[oyB * BX + ox] = tc.v.y;
    const F2 t3v = (DIV >= 1) ? pp + a.divcv * jcbk * div : pp;                    // pgrad.f90:300
    if (has_halo) t3h[hy * BX + hx] = t3h_of(div3d_at(hx, hy), P[hy * BX + hx]);
    __syncthreads();
    // a stage is refilled only by a thread 0 that saw its previous copy land
    if (tid == 0 && !fail && k + S - 1 <= klast) {
      fence_proxy_async_smem();
      issue(k + S - 1);
    }

    // stepuv.f90:294,304 with pgrad.f90:379,389: west u faces, the east
    // face from the next lane (lane 31 forms its own)
    const F2 un0 = col2(U, oyA) + dts * (col2(UF, fyA) + (col2(t3h - 1, oyA) - tc) * dxiv) * irst8u;
    F2 un1 = f2(__shfl_down_sync(full, un0.v.x, 1), __shfl_down_sync(full, un0.v.y, 1));
    if (tx == TX - 1)
      un1 = col2(U + 1, oyA) + dts * (col2(UF + 1, fyA) + (tc - col2(t3h + 1, oyA)) * dxiv) * irst8u;
    // v faces south of rows A and B (the one between the rows serves both),
    // and north of row B
    const F2 vs = col2(V, oyA) + dts * (col2(VF, fyA) + (f2(t3h[(oyA - 1) * BX + ox], tc.v.x) - tc) * dyiv) * irst8v;
    const float vf2 = V[(oyB + 1) * BX + ox] +
                      dts * (VF[(fyB + 1) * BX + ox] + (tc.v.y - t3h[(oyB + 1) * BX + ox]) * dyiv) * irst8v;
    const F2 vn = f2(vs.v.y, vf2);

    const float jcb8u = CK(k, C_JCB8U), jcb8v = CK(k, C_JCB8V);
    const float rcsq = CK(k, C_RCSQ), rst = CK(k, C_RST), rbr = CK(k, C_RBR), ircsq = CK(k, C_IRCSQ);
    const float irst8w = CK(k, C_IRST8W);
    // the stores of stepuv for one row
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
      if (kend) {   // vbcu.f90:120,134 (and vbcv): levels 1 and nk-1 copy levels 2 and nk-2
        const int kc = k == 2 ? 1 : nk - 1;
        store_periodic(a.u_new, g, STAG_U, i, j, kc, u0);
        store_periodic(a.v_new, g, STAG_V, i, j, kc, v0);
        if (xlast) store_periodic(a.u_new, g, STAG_U, i + 1, j, kc, u1);
        if (ylast) store_periodic(a.v_new, g, STAG_V, i, j + 1, kc, v1);
      }
    };
    if (ownA) store_uv(edgeA, ylastA, jA, idA, un0.v.x, un1.v.x, vs.v.x, vn.v.x);
    if (ownB) store_uv(edgeB, ylastB, jB, idB, un0.v.y, un1.v.y, vs.v.y, vn.v.y);

    F2 phd = (jcb8u * un0 - jcb8u * un1) * dxiv + (jcb8v * vs - jcb8v * vn) * dyiv;    // diver2d.f90:288
    phd = rcsq * phd;                                                                   // diverpih.f90:208
    const F2 wk = col2(W0, oyA), wk1 = col2(W1, oyA);
    const F2 pvd = rcsq * (wk - wk1) * dziv;                                            // diverpiv.f90:124
    const F2 fp = col2(PF, fyA) + phd + weic1m * (a.g05 * (wk + wk1) * rst + pvd);      // advbspi.f90:158
    if (ownA) a.p_new[idA] = fp.v.x;   // parked until the way down
    if (ownB) a.p_new[idB] = fp.v.y;
    const F2 fpdvj = fp * ijcbk;                                                        // pgradiv.f90:149
    const F2 wb8s = (pp * rst + fp * rbr * a.dtw) * ircsq * a.g05n;                     // buoywsi.f90:171
    if (k >= 3) {
      const F2 wpg = (t3v_prev - t3v) * dziv;                                           // pgrad.f90:320
      F2 fw = col2(WF, fyA) + wpg + (fpdvj_prev - fpdvj) * a.dtdzw;                     // pgradiv.f90:163
      if constexpr (BUY) fw = fw + (wb8s_prev + wb8s);                                  // buoywsi.f90:205
      const F2 wrhs = wk + dts * fw * irst8w;                                           // stepwi.f90:325
      // gaussel.f90:189-240 in double with the 1-D factors, one recurrence per row
      const double rr = (double)TH_RR(k), aa = TH_AA(k);
      const double fA = (k == 3) ? (double)wrhs.v.x * aa : ((double)wrhs.v.x - rr * fA_prev) * aa;
      const double fB = (k == 3) ? (double)wrhs.v.y * aa : ((double)wrhs.v.y - rr * fB_prev) * aa;
      if (ownA) a.w_new[idA] = (float)fA;   // parked until the way down
      if (ownB) a.w_new[idB] = (float)fB;
      fA_prev = fA;
      fB_prev = fB;
    }
    t3v_prev = t3v;
    fpdvj_prev = fpdvj;
    wb8s_prev = wb8s;
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

  // --- way down: back substitution, p' update, both rows interleaved;
  // loads run two levels ahead (their level clamped at 2, where the values
  // are not used).  cp(nk-2) = 0 makes the recurrence the identity at the
  // top level, so every level 3..nk-2 takes the same path. -------------
  struct Col {
    float wup = 0.f;        // w(k+1) as float; w(nk-1) = 0 (vbcw.f90:481)
    double wupd = 0.0;      // w(k+1) as double for the recurrence
    float wkend = 0.f, p3 = 0.f, pkend = 0.f;
    float fp0 = 0.f, po0 = 0.f, f0 = 0.f, fp1 = 0.f, po1 = 0.f, f1 = 0.f;
    int idk = 0;
  };
  Col cA, cB;
  auto start = [&](Col& c, bool own, int id_top) {
    c.idk = id_top;
    if (!own) return;
    c.fp0 = a.p_new[id_top]; c.po0 = a.p_old[id_top]; c.f0 = a.w_new[id_top];
    c.fp1 = a.p_new[id_top - plane]; c.po1 = a.p_old[id_top - plane]; c.f1 = a.w_new[id_top - plane];
  };
  const int idtopA = (int)g.at(i, jA, nk - 2);
  start(cA, ownA, idtopA);
  start(cB, ownB, idtopA + px);
  // the p' update of steppi from w(k) and w(k+1) (diverpiv.f90:124,
  // advbspi.f90:175, steppi.f90:217)
  auto pnew = [&](const Col& c, float wk, float fpb, float po, int k) {
    const float pvd = CK(k, C_RCSQ) * (wk - c.wup) * dziv;
    const float fp = fpb + a.weicoe * (a.g05 * (wk + c.wup) * CK(k, C_RST) + pvd);
    return po + dts * fp * CK(k, C_IJCB);
  };
  auto down = [&](Col& c, bool own, bool edge, int j, int k) {
    if (!own) return;
    const float fpb = c.fp0, po = c.po0, fg = c.f0;
    c.fp0 = c.fp1; c.po0 = c.po1; c.f0 = c.f1;
    const int idk = c.idk;
    const int idl = idk - (k - 2 >= 2 ? 2 : k - 2) * plane;   // level max(k-2, 2)
    c.fp1 = a.p_new[idl]; c.po1 = a.p_old[idl]; c.f1 = a.w_new[idl];
    const double wd = (double)fg - TH_CP(k) * c.wupd;   // gaussel.f90:254
    c.wupd = wd;
    const float wk = (float)wd;
    const float pn = pnew(c, wk, fpb, po, k);
    if (edge) {
      store_periodic(a.w_new, g, STAG_S, i, j, k, wk);
      store_periodic(a.p_new, g, STAG_S, i, j, k, pn);
    } else {
      a.w_new[idk] = wk;
      a.p_new[idk] = pn;
    }
    if (k == nk - 2) { c.wkend = wk; c.pkend = pn; }
    c.p3 = pn;   // the value of level 3 after the loop
    c.wup = wk;
    c.idk = idk - plane;
  };
  for (int k = nk - 2; k >= 3; --k) {
    down(cA, ownA, edgeA, jA, k);
    down(cB, ownB, edgeB, jB, k);
  }
  // level 2: w(2) = 0 (vbcw.f90:317, flat terrain), then the boundary rows
  // of vbcw.f90:285,317,471,481 (wc = w / jcb8w when stretched) and
  // vbcp.f90:126-160, and level nk of u, v, p' carried over (the small
  // step does not touch it)
  auto finish = [&](Col& c, bool own, bool edge, bool ylast, int j) {
    if (!own) return;
    const float p2 = pnew(c, 0.f, c.fp0, c.po0, 2);
    if (edge) store_periodic(a.p_new, g, STAG_S, i, j, 2, p2);
    else a.p_new[c.idk] = p2;
    const float w3 = c.wup;
    const float j8w3 = CK(3, C_JCB8W), j8wt = CK(nk - 2, C_JCB8W);
    const float wc3 = STH ? w3 / j8w3 : w3;
    const float wct = STH ? c.wkend / j8wt : c.wkend;
    store_periodic(a.w_new, g, STAG_S, i, j, 1, -j8w3 * wc3 - 0.f);
    store_periodic(a.w_new, g, STAG_S, i, j, 2, 0.f);
    store_periodic(a.w_new, g, STAG_S, i, j, nk - 1, 0.f);
    store_periodic(a.w_new, g, STAG_S, i, j, nk, -j8wt * wct - 0.f);
    store_periodic(a.p_new, g, STAG_S, i, j, 1, (a.bbc == 2) ? 2.f * p2 - c.p3 : p2);
    store_periodic(a.p_new, g, STAG_S, i, j, nk - 1, c.pkend);
    store_periodic(a.p_new, g, STAG_S, i, j, nk, a.p_old[g.at(i, j, nk)]);
    store_periodic(a.u_new, g, STAG_U, i, j, nk, a.u_old[g.at(i, j, nk)]);
    store_periodic(a.v_new, g, STAG_V, i, j, nk, a.v_old[g.at(i, j, nk)]);
    if (xlast) store_periodic(a.u_new, g, STAG_U, i + 1, j, nk, a.u_old[g.at(i + 1, j, nk)]);
    if (ylast) store_periodic(a.v_new, g, STAG_V, i, j + 1, nk, a.v_old[g.at(i, j + 1, nk)]);
  };
  finish(cA, ownA, edgeA, ylastA, jA);
  finish(cB, ownB, edgeB, ylastB, jB);
}

template <int S, int DIV, bool STH, bool BUY, bool GT>
__global__ void __launch_bounds__(kHeviTX * kH2Rows, GT ? 5 : 4)
k_hevi2(const __grid_constant__ HeviMaps m, const HeviArgs a) {
  hevi2_tile<S, DIV, STH, BUY, GT>(m, a, blockIdx.x, blockIdx.y);
}

// Every member of an ensemble in one launch: block b belongs to the member
// whose first_block is the largest not above b (the jobs are in block
// order), which runs its tile b - first_block.
template <int S, int DIV, bool STH, bool BUY>
__global__ void __launch_bounds__(kHeviTX * kH2Rows, 4)
k_hevi2_batch(const HeviJob* __restrict__ jobs, int njobs) {
  int lo = 0, hi = njobs - 1;
  const int b = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].first_block <= b) lo = mid;
    else hi = mid - 1;
  }
  const HeviJob& job = jobs[lo];
  const int t = b - job.first_block;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    // the maps were copied into global memory by the host: make that copy
    // visible to the tensor-map proxy before the first TMA load reads them
    const CUtensorMap* mp = &job.maps.u;
    for (int q = 0; q < 8; ++q)
      asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(mp + q) : "memory");
  }
  hevi2_tile<S, DIV, STH, BUY, false>(job.maps, job.args, t % job.tiles_x, t / job.tiles_x);
}

template <int S, bool GT, int DIV, bool STH, bool BUY>
int launch_h2(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st) {
  using L = H2Layout<S>;
  const Grid& g = a.g;
  const int nx = g.ni - 3, ny = g.nj - 3;
  const size_t bytes = L::bytes(g.nk, GT);
  if (bytes > 227 * 1024) return CRESS_E_UNSUPPORTED;
  auto kern = k_hevi2<S, DIV, STH, BUY, GT>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
    return CRESS_E_CUDA;
  dim3 block(kHeviTX, kH2Rows);
  dim3 grid((nx + kHeviTX - 1) / kHeviTX, (ny + kH2TY - 1) / kH2TY);
  kern<<<grid, block, bytes, st>>>(maps, a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

template <int S, bool GT, int DIV>
int launch_h2_div(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st) {
  const bool sth = a.sthopt != 0, buy = a.buyopt == 1;
  if (sth) return buy ? launch_h2<S, GT, DIV, true, true>(a, maps, st) : launch_h2<S, GT, DIV, true, false>(a, maps, st);
  return buy ? launch_h2<S, GT, DIV, false, true>(a, maps, st) : launch_h2<S, GT, DIV, false, false>(a, maps, st);
}

template <int S, bool GT>
int launch_h2_opts(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st) {
  switch (a.divopt) {
    case 2: return launch_h2_div<S, GT, 2>(a, maps, st);
    case 1: return launch_h2_div<S, GT, 1>(a, maps, st);
    default: return launch_h2_div<S, GT, 0>(a, maps, st);
  }
}

}  // namespace

// variant 0: 4-stage ring, level table in shared memory; 1: 3-stage ring,
// level table and elimination factors read from global memory (needs a.lvl)
int launch_hevi2(const HeviArgs& a, const HeviMaps& maps, int variant, cudaStream_t st) {
  if (a.g.count() >= (1LL << 31) || a.g.nk < 6) return CRESS_E_UNSUPPORTED;   // 32-bit indices; levels 2..nk-2 >= 3
  if (variant == 1) return a.lvl ? launch_h2_opts<3, true>(a, maps, st) : CRESS_E_UNSUPPORTED;
  return launch_h2_opts<4, false>(a, maps, st);
}

// Tiles of tile 0 (32 x 8 columns) of a member's grid.
void hevi_job_tiles(const Grid& g, int* tx, int* ty) {
  *tx = (g.ni - 3 + kHeviTX - 1) / kHeviTX;
  *ty = (g.nj - 3 + kH2TY - 1) / kH2TY;
}

template <int DIV, bool STH, bool BUY>
static int launch_batch_t(const HeviJob* jobs_d, int njobs, int nblocks, int nk_max, cudaStream_t st) {
  constexpr int S = 4;
  using L = H2Layout<S>;
  const size_t bytes = L::bytes(nk_max, false);
  if (bytes > 227 * 1024) return CRESS_E_UNSUPPORTED;
  auto kern = k_hevi2_batch<S, DIV, STH, BUY>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
    return CRESS_E_CUDA;
  kern<<<nblocks, dim3(kHeviTX, kH2Rows), bytes, st>>>(jobs_d, njobs);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

int launch_hevi_batch(const HeviJob* jobs_d, int njobs, int nblocks, int nk_max, int divopt, bool sth, bool buy,
                      cudaStream_t st) {
  auto pick = [&](auto div) -> int {
    constexpr int D = decltype(div)::value;
    if (sth) return buy ? launch_batch_t<D, true, true>(jobs_d, njobs, nblocks, nk_max, st)
                        : launch_batch_t<D, true, false>(jobs_d, njobs, nblocks, nk_max, st);
    return buy ? launch_batch_t<D, false, true>(jobs_d, njobs, nblocks, nk_max, st)
               : launch_batch_t<D, false, false>(jobs_d, njobs, nblocks, nk_max, st);
  };
  switch (divopt) {
    case 2: return pick(std::integral_constant<int, 2>{});
    case 1: return pick(std::integral_constant<int, 1>{});
    default: return pick(std::integral_constant<int, 0>{});
  }
}

}  // namespace cress

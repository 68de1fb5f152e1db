// Fused HE-VI acoustic substep with the whole column kept on chip (tile 12).
// Same operators, order of terms and boundary rules as k_hevi2 (s_hevi,
// SrcOrig/hevi.f90:339-426, impopt=1, flat terrain, periodic lateral or
// open x boundaries, rigid lid): pgrad + diver3d, stepuv, diverpih +
// diver2d, diverpiv, advbspi, pgradiv, buoywsi, stepwi with the FP64
// Thomas solve (gaussel), steppi.
//
// What differs from k_hevi2 is where the column waits between the way up
// (forward elimination) and the way down (back substitution):
//   * the eliminated right-hand side of each level stays in FP64 in tensor
//     memory (tcgen05.st / tcgen05.ld, 4 columns per level for the two
//     columns a thread owns; 256 tensor-memory columns per block, two
//     blocks per SM), so the solve is FP64 end to end;
//   * the explicit part of the new p', p_old + dts fp_explicit / jcb, is
//     parked in shared memory (one float2 per level and thread);
// so a substep reads u, v, w, p' and the four forcings once and writes the
// new u, v, w, p' once: no parked values cross HBM and old p' is read once.
// The p' update is regrouped as (p_old + dts fp_e / jcb) + dts fp_w / jcb,
// where the reference forms p_old + dts (fp_e + fp_w) / jcb (steppi.f90:217);
// the two differ by FP32 rounding only.
//
// Per-level constants and the elimination factors come from a level table
// in global memory (nine 16-byte loads per level, L1-resident, issued one
// level ahead), each float stored twice so the loads yield ready operand
// pairs for the packed FP32x2 arithmetic.  Blocks
// that touch the domain's edges take a path with the ownership checks and
// the periodic ghost stores; every other block stores plainly.
//
// Waits on the TMA ring are bounded (HeviArgs::spin).  A wait that gives
// up makes thread 0 stop issuing copies; after the level loop the block
// records the failure, waits for the copies it issued and frees its tensor
// memory before it leaves.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "common.cuh"
#include "f2.cuh"
#include "hevi.cuh"
#include "tma.cuh"
#include "umma.cuh"

namespace cress {

namespace {

constexpr int kH3TX = 32;        // tile width (one column per lane)
constexpr int kH3TY = 8;         // tile rows (two per thread)
constexpr int kH3Rows = 4;       // thread rows
constexpr int kH3NT = kH3TX * kH3Rows;
constexpr uint32_t kH3TmemCols = 256;
constexpr int kH3MinSmem = 80 * 1024;   // at most two blocks (2 x 256 tensor-memory columns) per SM

__host__ __device__ constexpr int r32(int n) { return (n + 31) / 32 * 32; }

template <int S>
struct H3Layout {
  using R = HeviRows<kH3TY>;
  static constexpr int BX = kHeviBoxX;
  static constexpr int oU = 0;
  static constexpr int oV = oU + r32(BX * R::u);
  static constexpr int oW = oV + r32(BX * R::v);
  static constexpr int oP = oW + r32(BX * R::w);
  static constexpr int oUF = oP + r32(BX * R::p);
  static constexpr int oVF = oUF + r32(BX * R::uf);
  static constexpr int oWF = oVF + r32(BX * R::vf);
  static constexpr int oPF = oWF + r32(BX * R::wf);
  static constexpr int stage = oPF + r32(BX * R::pf);
  static constexpr uint32_t tx_bytes =
      4u * BX * (R::u + R::v + R::w + R::p + R::uf + R::vf + R::wf + R::pf);
  static constexpr int t3h_floats = r32((kH3TY + 2) * BX);
  // ring, t3h (two buffers), parked p' (levels 2..nk-2, float2 per thread), mbarriers
  __host__ __device__ static size_t bytes(int nk) {
    return 4 * ((size_t)S * stage + 2 * (size_t)t3h_floats) + 8 * (size_t)(nk - 3) * kH3NT + 8 * (size_t)S;
  }
};

__device__ __forceinline__ uint32_t lo32(double d) { return (uint32_t)__double2loint(d); }
__device__ __forceinline__ uint32_t hi32(double d) { return (uint32_t)__double2hiint(d); }
__device__ __forceinline__ double mk64(uint32_t lo, uint32_t hi) { return __hiloint2double((int)hi, (int)lo); }

// One tile of one substep.  EDGE: the tile touches a domain edge (partial
// ownership, periodic ghost images, the faces at ni-1 / nj-1).
template <int S, int DIV, bool STH, bool BUY, bool EDGE>
__device__ __forceinline__ void hevi3_tile(const HeviMaps& m, const HeviArgs& a, float* smem, uint32_t tmem) {
  using L = H3Layout<S>;
  constexpr int TX = kH3TX, TY = kH3TY, BX = kHeviBoxX, NT = kH3NT;
  const unsigned full = 0xffffffffu;
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = 2 + blockIdx.x * TX, j0 = 2 + blockIdx.y * TY;
  const int xb = i0 - 2;  // box x origin (multiple of 32)
  const int i = i0 + tx, jA = j0 + 2 * ty, jB = jA + 1;
  bool ownA = true, ownB = true, edgeA = false, edgeB = false, xlast = false, ylastA = false, ylastB = false;
  if constexpr (EDGE) {
    const int ilast = min(i0 + TX - 1, ni - 2), jlast = min(j0 + TY - 1, nj - 2);
    ownA = (i <= ilast) && (jA <= jlast);
    ownB = (i <= ilast) && (jB <= jlast);
    const bool ei = (i <= 3) || (i >= ni - 2);
    edgeA = ei || (jA <= 3) || (jA >= nj - 2);
    edgeB = ei || (jB <= 3) || (jB >= nj - 2);
    xlast = (i == ilast) && (i + 1 == ni - 1);
    ylastA = (jA == jlast) && (jA + 1 == nj - 1);
    ylastB = (jB == jlast) && (jB + 1 == nj - 1);
  }

  float* ring = smem;
  float* t3hb = ring + S * L::stage;                                       // 2 x [(TY+2)][BX]
  float2* qs = reinterpret_cast<float2*>(t3hb + 2 * L::t3h_floats);        // [(k-2) * NT + tid]
  uint64_t* bars = reinterpret_cast<uint64_t*>(qs + (size_t)(nk - 3) * NT);
  const float4* rows = reinterpret_cast<const float4*>(a.lvl3);           // 9 vectors per level
  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  // Levels 2..nk-1 are staged (w is needed one level above the top
  // update); thread 0 issues them in order, `issued` the highest so far.
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
  const F2 dts = f2(a.dts), dxiv = f2(a.dxiv), dyiv = f2(a.dyiv), dziv = f2(a.dziv);
  const F2 weic1m = f2(1.f - a.weicoe), g05 = f2(a.g05), g05n = f2(a.g05n), dtw = f2(a.dtw),
           dtdzw = f2(a.dtdzw);
  const float divch = a.divch, divcv = a.divcv;
  const F2 divch2 = f2(divch), divcv2 = f2(divcv);
  F2 t3v_prev = f2(0.f), fpdvj_prev = f2(0.f), wb8s_prev = f2(0.f);   // rows A, B
  double fA_prev = 0.0, fB_prev = 0.0;
  bool fail = false;
  const int plane = (int)g.plane, px = g.px;
  const int id2 = (int)g.at(i, jA, 2);
  float* uA = a.u_new + id2;
  float* vA = a.v_new + id2;
  // this thread's cell in the boxes that start at j0-1 (row oyA = 2ty+1,
  // column tx+2); the forcing boxes start at j0, one row lower
  const int tofs = (2 * ty + 1) * BX + tx + 2;
  // the level table: nine vectors per level; row k's vectors 0, 2-8 and
  // row k+1's vector 1 (rst8w, ij8w one level up) are loaded one level ahead
  struct Row {
    float4 v0, v2, v3, v4, v5, v6, v7, n1;
    double aa;
  };
  auto load_row = [&](int k, Row& r) {
    const float4* p = rows + 9 * k;
    r.v0 = __ldg(p + 0); r.v2 = __ldg(p + 2); r.v3 = __ldg(p + 3); r.v4 = __ldg(p + 4);
    r.v5 = __ldg(p + 5); r.v6 = __ldg(p + 6); r.v7 = __ldg(p + 7);
    r.aa = __ldg(reinterpret_cast<const double*>(p + 8));
    r.n1 = __ldg(p + 9 + 1);
  };
  auto lo2 = [](float4 v) { return F2{make_float2(v.x, v.y)}; };   // first pair of a vector
  auto hi2 = [](float4 v) { return F2{make_float2(v.z, v.w)}; };   // second pair
  Row cur, nxt;
  load_row(2, cur);
  float4 v1k = __ldg(rows + 9 * 2 + 1);   // row k's vector 1

  for (int k = 2; k <= nk - 2; ++k, uA += plane, vA += plane) {
    if (k + 1 <= nk - 2) load_row(k + 1, nxt);
    // one barrier per level: t3h alternates between two buffers, and the
    // stage of level k-1 is refilled only after this level's barrier
    float* t3h = t3hb + (k & 1) * L::t3h_floats;
    const int s0 = (k - 2) % S, s1 = (k - 1) % S;
    if (!fail && k == 2) fail = !mbar_wait(&bars[s0], 0, a.spin);
    if (!fail) fail = !mbar_wait(&bars[s1], ((k - 1) / S) & 1, a.spin);
    const float* st0 = ring + s0 * L::stage;
    const float* W1s = ring + s1 * L::stage + L::oW;
    const float* tb = st0 + tofs;         // own cell (row A) in every box of level k
    const float* tw1 = W1s + tofs;        // own cell in level k+1's w box
    float* th0 = t3h + tofs;              // own cell in the damped-pressure plane
    const F2 rst8u = lo2(cur.v0), rst8v = hi2(cur.v0);
    const F2 rst8wk = lo2(v1k), ij8wk = hi2(v1k), rst8wk1 = lo2(cur.n1), ij8wk1 = hi2(cur.n1);
    const F2 jcbk = lo2(cur.v2), ijcbk = hi2(cur.v2), irst8u = lo2(cur.v3), irst8v = hi2(cur.v3);

    // diver3d.f90:318 (with phy2cnt.f90:219 for the contravariant w) at a halo point
    const float* U = st0 + L::oU;
    const float* V = st0 + L::oV;
    const float* W0 = st0 + L::oW;
    const float* P = st0 + L::oP;
    auto div3d_at = [&](int x, int y) {
      float wck = W0[y * BX + x], wck1 = W1s[y * BX + x];
      if constexpr (STH) { wck = wck * ij8wk.v.x; wck1 = wck1 * ij8wk1.v.x; }
      return (rst8wk.v.x * wck - rst8wk1.v.x * wck1) * dziv.v.x +
             ((rst8u.v.x * U[y * BX + x] - rst8u.v.x * U[y * BX + x + 1]) * dxiv.v.x +
              (rst8v.v.x * V[y * BX + x] - rst8v.v.x * V[(y + 1) * BX + x]) * dyiv.v.x);
    };
    // pgrad.f90:300,341,363
    auto t3h_of = [&](float div, float pp) {
      float th;
      if constexpr (DIV == 2) th = pp + divch * div * ijcbk.v.x;
      else if constexpr (DIV == 1) th = pp + divcv * jcbk.v.x * div;
      else th = pp;
      return jcbk.v.x * th;
    };
    // rows A and B of the thread in the two lanes of F2: one packed
    // instruction for both rows (offsets relative to the own cell)
    auto at2 = [&](const float* base, int off) { return f2(base[off], base[off + BX]); };
    F2 wc0 = at2(tb, L::oW), wc1 = at2(tw1, 0);
    if constexpr (STH) { wc0 = wc0 * ij8wk; wc1 = wc1 * ij8wk1; }
    const F2 uo = at2(tb, L::oU), vo = at2(tb, L::oV);
    const F2 div = (rst8wk * wc0 - rst8wk1 * wc1) * dziv +
                   ((rst8u * uo - rst8u * at2(tb, L::oU + 1)) * dxiv +
                    (rst8v * vo - rst8v * at2(tb, L::oV + BX)) * dyiv);      // diver3d.f90:318
    const F2 pp = at2(tb, L::oP);
    F2 th;                                                                   // pgrad.f90:341,363
    if constexpr (DIV == 2) th = pp + divch2 * div * ijcbk;
    else if constexpr (DIV == 1) th = pp + divcv2 * jcbk * div;
    else th = pp;
    const F2 tc = jcbk * th;
    th0[0] = tc.v.x;
    th0[BX] = tc.v.y;
    const F2 t3v = (DIV >= 1) ? pp + divcv2 * jcbk * div : pp;               // pgrad.f90:300
    if (has_halo) t3h[hy * BX + hx] = t3h_of(div3d_at(hx, hy), P[hy * BX + hx]);
    // the rest of this level's own inputs, read before the barrier
    const F2 uf = at2(tb, L::oUF - BX), vf = at2(tb, L::oVF - BX), wf = at2(tb, L::oWF - BX),
             pf = at2(tb, L::oPF - BX);
    const float vo2 = tb[L::oV + 2 * BX], vf2f = tb[L::oVF + BX];
    const F2 wk = at2(tb, L::oW), wk1 = at2(tw1, 0);
    __syncthreads();
    if (tid == 0 && !fail && k + S - 1 <= klast) {   // refill only after its copy was seen to land
      fence_proxy_async_smem();
      issue(k + S - 1);
    }

    // stepuv.f90:294,304 with pgrad.f90:379,389: west u faces, the east
    // face from the next lane (lane 31 forms its own)
    const F2 un0 = uo + dts * (uf + (at2(th0, -1) - tc) * dxiv) * irst8u;
    F2 un1 = f2(__shfl_down_sync(full, un0.v.x, 1), __shfl_down_sync(full, un0.v.y, 1));
    if (tx == TX - 1)
      un1 = at2(tb, L::oU + 1) + dts * (at2(tb, L::oUF - BX + 1) + (tc - at2(th0, 1)) * dxiv) * irst8u;
    // v faces south of rows A and B (the one between the rows serves both),
    // and north of row B
    const F2 vs = vo + dts * (vf + (f2(th0[-BX], tc.v.x) - tc) * dyiv) * irst8v;
    const float vn2 = vo2 + a.dts * (vf2f + (tc.v.y - th0[2 * BX]) * a.dyiv) * irst8v.v.x;
    const F2 vn = f2(vs.v.y, vn2);

    const F2 jcb8u = lo2(cur.v4), jcb8v = hi2(cur.v4), rcsq = lo2(cur.v5), rst = hi2(cur.v5);
    const F2 rbr = lo2(cur.v6), ircsq = hi2(cur.v6), irst8w = lo2(cur.v7);
    const bool kend = (k == 2) || (k == nk - 2);
    if constexpr (!EDGE) {
      uA[0] = un0.v.x; uA[px] = un0.v.y;
      vA[0] = vs.v.x; vA[px] = vs.v.y;
      if (kend) {   // vbcu.f90:120,134 (and vbcv): levels 1 and nk-1 copy levels 2 and nk-2
        const int dk = (k == 2 ? -1 : 1) * plane;
        uA[dk] = un0.v.x; uA[dk + px] = un0.v.y;
        vA[dk] = vs.v.x; vA[dk + px] = vs.v.y;
      }
    } else {
      auto store_uv = [&](bool edge, bool ylast, int j, float u0, float u1, float v0, float v1) {
        if (edge) {
          store_periodic(a.u_new, g, STAG_U, i, j, k, u0);
          store_periodic(a.v_new, g, STAG_V, i, j, k, v0);
        } else {
          a.u_new[g.at(i, j, k)] = u0;
          a.v_new[g.at(i, j, k)] = v0;
        }
        if (xlast) store_periodic(a.u_new, g, STAG_U, i + 1, j, k, u1);
        if (ylast) store_periodic(a.v_new, g, STAG_V, i, j + 1, k, v1);
        if (kend) {
          const int kc = k == 2 ? 1 : nk - 1;
          store_periodic(a.u_new, g, STAG_U, i, j, kc, u0);
          store_periodic(a.v_new, g, STAG_V, i, j, kc, v0);
          if (xlast) store_periodic(a.u_new, g, STAG_U, i + 1, j, kc, u1);
          if (ylast) store_periodic(a.v_new, g, STAG_V, i, j + 1, kc, v1);
        }
      };
      if (ownA) store_uv(edgeA, ylastA, jA, un0.v.x, un1.v.x, vs.v.x, vn.v.x);
      if (ownB) store_uv(edgeB, ylastB, jB, un0.v.y, un1.v.y, vs.v.y, vn.v.y);
    }

    F2 phd = (jcb8u * un0 - jcb8u * un1) * dxiv + (jcb8v * vs - jcb8v * vn) * dyiv;    // diver2d.f90:288
    phd = rcsq * phd;                                                                   // diverpih.f90:208
    const F2 pvd = rcsq * (wk - wk1) * dziv;                                            // diverpiv.f90:124
    const F2 fp = pf + phd + weic1m * (g05 * (wk + wk1) * rst + pvd);                   // advbspi.f90:158
    const F2 q = pp + dts * fp * ijcbk;           // steppi.f90:217, explicit part of the new p'
    qs[(k - 2) * NT + tid] = q.v;
    const F2 fpdvj = fp * ijcbk;                                                        // pgradiv.f90:149
    const F2 wb8s = (pp * rst + fp * rbr * dtw) * ircsq * g05n;                         // buoywsi.f90:171
    if (k >= 3) {
      const F2 wpg = (t3v_prev - t3v) * dziv;                                           // pgrad.f90:320
      F2 fw = wf + wpg + (fpdvj_prev - fpdvj) * dtdzw;                                  // pgradiv.f90:163
      if constexpr (BUY) fw = fw + (wb8s_prev + wb8s);                                  // buoywsi.f90:205
      const F2 wrhs = wk + dts * fw * irst8w;                                           // stepwi.f90:325
      // gaussel.f90:189-240 in double with the 1-D factors, one recurrence per row
      const double rr = (double)cur.v7.z, aa = cur.aa;
      const double fA = (k == 3) ? (double)wrhs.v.x * aa : ((double)wrhs.v.x - rr * fA_prev) * aa;
      const double fB = (k == 3) ? (double)wrhs.v.y * aa : ((double)wrhs.v.y - rr * fB_prev) * aa;
      tmem_st4(tmem + 4u * (uint32_t)(k - 3), lo32(fA), hi32(fA), lo32(fB), hi32(fB));
      fA_prev = fA;
      fB_prev = fB;
    }
    t3v_prev = t3v;
    fpdvj_prev = fpdvj;
    wb8s_prev = wb8s;
    v1k = cur.n1;
    cur = nxt;
  }

  if (__syncthreads_or(fail)) {
    // A bounded wait gave up: record it, let the copies still in flight
    // land (bounded again) so no TMA write outlives the block, and leave
    // (the kernel frees the tensor memory).
    if (tid == 0) {
      atomicExch(a.err, 1);
      for (int s = 0; s < S; ++s) {
        int kl = -1;
        for (int k = 2; k <= issued; ++k)
          if ((k - 2) % S == s) kl = k;
        if (kl >= 0) mbar_wait(&bars[s], ((kl - 2) / S) & 1);
      }
    }
    tmem_wait_st();
    return;
  }
  tmem_wait_st();

  // --- way down: back substitution (FP64, from tensor memory) and the p'
  // update, both rows interleaved; eight levels per tensor-memory load.
  // cp(nk-2) = 0 makes the recurrence the identity at the top level.
  const int ktop = nk - 2;
  double wdA = 0.0, wdB = 0.0;            // w(k+1) in double; w(nk-1) = 0 (vbcw.f90:481)
  F2 wup = f2(0.f), wkend = f2(0.f), pkend = f2(0.f), p3 = f2(0.f);
  const F2 weicoe = f2(a.weicoe);
  float* wT = a.w_new + (int)g.at(i, jA, ktop);
  float* pT = a.p_new + (int)g.at(i, jA, ktop);
  for (int c = (ktop - 3) / 8; c >= 0; --c) {
    uint32_t r[32];
    tmem_ld32(tmem + 32u * (uint32_t)c, r);
    tmem_wait_ld();
#pragma unroll
    for (int e = 7; e >= 0; --e) {
      const int k = 3 + 8 * c + e;
      if (k > ktop) continue;
      const float4* rp = rows + 9 * k;
      const float4 d2 = __ldg(rp + 2), d5 = __ldg(rp + 5);
      const double cpk = __ldg(reinterpret_cast<const double*>(rp + 8) + 1);
      wdA = mk64(r[4 * e], r[4 * e + 1]) - cpk * wdA;    // gaussel.f90:254
      wdB = mk64(r[4 * e + 2], r[4 * e + 3]) - cpk * wdB;
      const F2 wk = f2((float)wdA, (float)wdB);
      const F2 q = F2{qs[(k - 2) * NT + tid]};
      // steppi.f90:217 with diverpiv.f90:124 and advbspi.f90:175 (the implicit part)
      const F2 pvd = lo2(d5) * (wk - wup) * dziv;
      const F2 fpw = weicoe * (g05 * (wk + wup) * hi2(d5) + pvd);
      const F2 pn = q + dts * fpw * hi2(d2);
      const int off = (k - ktop) * plane;
      if constexpr (!EDGE) {
        wT[off] = wk.v.x; wT[off + px] = wk.v.y;
        pT[off] = pn.v.x; pT[off + px] = pn.v.y;
      } else {
        if (ownA) {
          if (edgeA) {
            store_periodic(a.w_new, g, STAG_S, i, jA, k, wk.v.x);
            store_periodic(a.p_new, g, STAG_S, i, jA, k, pn.v.x);
          } else {
            wT[off] = wk.v.x;
            pT[off] = pn.v.x;
          }
        }
        if (ownB) {
          if (edgeB) {
            store_periodic(a.w_new, g, STAG_S, i, jB, k, wk.v.y);
            store_periodic(a.p_new, g, STAG_S, i, jB, k, pn.v.y);
          } else {
            wT[off + px] = wk.v.y;
            pT[off + px] = pn.v.y;
          }
        }
      }
      if (k == ktop) { wkend = wk; pkend = pn; }
      p3 = pn;   // the value of level 3 after the loop
      wup = wk;
    }
  }
  // level 2: w(2) = 0 (vbcw.f90:317, flat terrain) and its p', then the
  // boundary rows of vbcw.f90:285,317,471,481 (wc = w / jcb8w when
  // stretched) and vbcp.f90:126-160, and level nk of u, v, p' carried over
  {
    const float4 d2 = __ldg(rows + 9 * 2 + 2), d5 = __ldg(rows + 9 * 2 + 5);
    const F2 q = F2{qs[tid]};
    const F2 w0 = f2(0.f);
    const F2 pvd = lo2(d5) * (w0 - wup) * dziv;
    const F2 fpw = weicoe * (g05 * (w0 + wup) * hi2(d5) + pvd);
    const F2 p2 = q + dts * fpw * hi2(d2);
    const float jw3 = __ldg(a.col + C_JCB8W * (nk + 1) + 3), jwt = __ldg(a.col + C_JCB8W * (nk + 1) + nk - 2);
    auto finish = [&](bool own, bool edge, bool ylast, int j, float p2v, float p3v, float w3, float wke,
                      float pke) {
      if (!own) return;
      const float wc3 = STH ? w3 / jw3 : w3;
      const float wct = STH ? wke / jwt : wke;
      if (!EDGE || !edge) a.p_new[g.at(i, j, 2)] = p2v;
      else store_periodic(a.p_new, g, STAG_S, i, j, 2, p2v);
      store_periodic(a.w_new, g, STAG_S, i, j, 1, -jw3 * wc3 - 0.f);
      store_periodic(a.w_new, g, STAG_S, i, j, 2, 0.f);
      store_periodic(a.w_new, g, STAG_S, i, j, nk - 1, 0.f);
      store_periodic(a.w_new, g, STAG_S, i, j, nk, -jwt * wct - 0.f);
      store_periodic(a.p_new, g, STAG_S, i, j, 1, (a.bbc == 2) ? 2.f * p2v - p3v : p2v);
      store_periodic(a.p_new, g, STAG_S, i, j, nk - 1, pke);
      store_periodic(a.p_new, g, STAG_S, i, j, nk, a.p_old[g.at(i, j, nk)]);
      store_periodic(a.u_new, g, STAG_U, i, j, nk, a.u_old[g.at(i, j, nk)]);
      store_periodic(a.v_new, g, STAG_V, i, j, nk, a.v_old[g.at(i, j, nk)]);
      if (xlast) store_periodic(a.u_new, g, STAG_U, i + 1, j, nk, a.u_old[g.at(i + 1, j, nk)]);
      if (ylast) store_periodic(a.v_new, g, STAG_V, i, j + 1, nk, a.v_old[g.at(i, j + 1, nk)]);
    };
    finish(ownA, edgeA, ylastA, jA, p2.v.x, p3.v.x, wup.v.x, wkend.v.x, pkend.v.x);
    finish(ownB, edgeB, ylastB, jB, p2.v.y, p3.v.y, wup.v.y, wkend.v.y, pkend.v.y);
  }
}

template <int S, int DIV, bool STH, bool BUY>
__global__ void __launch_bounds__(kH3NT, 2) k_hevi3(const __grid_constant__ HeviMaps m, const HeviArgs a) {
  extern __shared__ __align__(1024) float smem[];
  __shared__ uint32_t tmem_slot;
  const int warp = threadIdx.y;   // blockDim = (32, 4): one warp per thread row
  if (warp == 0) tmem_alloc(&tmem_slot, kH3TmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  // lanes 32w..32w+31 belong to warp w
  const uint32_t tmem = tmem_slot + ((uint32_t)(warp * 32) << 16);
  const bool edge = blockIdx.x == 0 || blockIdx.x == gridDim.x - 1 || blockIdx.y == 0 || blockIdx.y == gridDim.y - 1;
  if (edge) hevi3_tile<S, DIV, STH, BUY, true>(m, a, smem, tmem);
  else hevi3_tile<S, DIV, STH, BUY, false>(m, a, smem, tmem);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem_slot, kH3TmemCols);
  }
}

template <int S, int DIV, bool STH, bool BUY>
int launch_h3(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st) {
  using L = H3Layout<S>;
  const Grid& g = a.g;
  const size_t bytes = L::bytes(g.nk) > (size_t)kH3MinSmem ? L::bytes(g.nk) : (size_t)kH3MinSmem;
  if (bytes > 113 * 1024) return CRESS_E_UNSUPPORTED;   // two blocks per SM
  auto kern = k_hevi3<S, DIV, STH, BUY>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
    return CRESS_E_CUDA;
  const int nx = g.ni - 3, ny = g.nj - 3;
  dim3 block(kH3TX, kH3Rows);
  dim3 grid((nx + kH3TX - 1) / kH3TX, (ny + kH3TY - 1) / kH3TY);
  kern<<<grid, block, bytes, st>>>(maps, a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

template <int DIV>
int launch_h3_div(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st) {
  constexpr int S = 4;
  const bool sth = a.sthopt != 0, buy = a.buyopt == 1;
  if (sth) return buy ? launch_h3<S, DIV, true, true>(a, maps, st) : launch_h3<S, DIV, true, false>(a, maps, st);
  return buy ? launch_h3<S, DIV, false, true>(a, maps, st) : launch_h3<S, DIV, false, false>(a, maps, st);
}

}  // namespace

int launch_hevi3(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st) {
  if (!a.lvl3 || a.g.nk > kHevi3MaxNk || a.g.nk < 8 || a.g.count() >= (1LL << 31)) return CRESS_E_UNSUPPORTED;
  switch (a.divopt) {
    case 2: return launch_h3_div<2>(a, maps, st);
    case 1: return launch_h3_div<1>(a, maps, st);
    default: return launch_h3_div<0>(a, maps, st);
  }
}

}  // namespace cress

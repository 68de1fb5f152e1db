// Fused HE-VI acoustic substep with the column kept on chip, one column per
// thread (tile 13).  Same operators, order of terms and boundary rules as
// k_hevi2 / k_hevi3 (s_hevi, SrcOrig/hevi.f90:339-426, impopt=1, flat
// terrain, periodic lateral or open x boundaries, rigid lid).
//
// Layout: a block of 32 x 8 threads owns a 32 x 8 tile of columns, one per
// thread, and marches it up k through a TMA ring, then down.  Between the
// two sweeps the column stays on chip:
//   * the eliminated right-hand side of each level in FP64 in tensor memory
//     (two 32-bit columns per level; warps 0-3 use tensor-memory columns
//     0-127 of the block's 256, warps 4-7 columns 128-255, each warp its
//     own 32 lanes);
//   * the explicit part of the new p', p_old + dts fp_explicit / jcb, in
//     shared memory (one float per level and thread);
// so a substep moves u, v, w, p' and the four forcings through HBM once.
// Two blocks (16 warps) fit an SM: 2 x 256 tensor-memory columns.  Every
// thread forms the u face west of its column (the east face comes from the
// next lane) and both v faces of its column.
//
// The p' update is regrouped as (p_old + dts fp_e / jcb) + dts fp_w / jcb
// where the reference forms p_old + dts (fp_e + fp_w) / jcb (steppi.f90:
// 217); the two differ by FP32 rounding only.
//
// Waits on the TMA ring are bounded (HeviArgs::spin).  A wait that gives
// up makes thread 0 stop issuing copies; after the level loop the block
// records the failure, waits for the copies it issued and frees its tensor
// memory before it leaves.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>
#include "common.cuh"
#include "hevi.cuh"
#include "tma.cuh"
#include "umma.cuh"

namespace cress {

namespace {

constexpr int kH4TX = 32;        // tile width (one column per lane)
constexpr int kH4TY = 8;         // tile rows (one per warp)
constexpr int kH4NT = kH4TX * kH4TY;
constexpr uint32_t kH4TmemCols = 256;
constexpr int kH4MinSmem = 80 * 1024;   // at most two blocks (2 x 256 tensor-memory columns) per SM

__host__ __device__ constexpr int r32c(int n) { return (n + 31) / 32 * 32; }

template <int S>
struct H4Layout {
  using R = HeviRows<kH4TY>;
  static constexpr int BX = kHeviBoxX;
  static constexpr int oU = 0;
  static constexpr int oV = oU + r32c(BX * R::u);
  static constexpr int oW = oV + r32c(BX * R::v);
  static constexpr int oP = oW + r32c(BX * R::w);
  static constexpr int oUF = oP + r32c(BX * R::p);
  static constexpr int oVF = oUF + r32c(BX * R::uf);
  static constexpr int oWF = oVF + r32c(BX * R::vf);
  static constexpr int oPF = oWF + r32c(BX * R::wf);
  static constexpr int stage = oPF + r32c(BX * R::pf);
  static constexpr uint32_t tx_bytes =
      4u * BX * (R::u + R::v + R::w + R::p + R::uf + R::vf + R::wf + R::pf);
  static constexpr int t3h_floats = r32c((kH4TY + 2) * BX);
  // ring, t3h (two buffers), parked p' (levels 2..nk-2, one float per
  // thread), mbarriers, the way down's table (rcsq, rst, ijcb per level,
  // then cp in double)
  __host__ __device__ static size_t bytes(int nk) {
    return 4 * ((size_t)S * stage + 2 * (size_t)t3h_floats) + 4 * (size_t)(nk - 3) * kH4NT + 8 * (size_t)S +
           24 * (size_t)(nk + 1);
  }
};

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}

__device__ __forceinline__ void tmem_st2(uint32_t taddr, uint32_t a, uint32_t b) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(taddr), "r"(a), "r"(b) : "memory");
}

// What a thread keeps through the upward sweep.
struct H4Up {
  float t3v_prev = 0.f, fpdvj_prev = 0.f, wb8s_prev = 0.f;
  double f_prev = 0.0;
  bool fail = false;
  int issued = 1;          // highest level thread 0 has issued
  float* up;               // new u at (i, j, k)
  float* vp;               // new v at (i, j, k)
  float* qp;               // parked p' of level k
  float4 v0k;              // level k's first table vector (rst8u, rst8v, rst8w, ij8w)
};

// What a thread keeps unchanged through the sweep (the step's scalars
// stay in the kernel parameters, read by the arithmetic directly).
struct H4Env {
  float* ring;             // the TMA ring
  const float* rb;         // the ring shifted to this thread's cell (row ty+1, column tx+2)
  float* th;               // the damped-pressure planes shifted to this thread's cell
  uint64_t* bars;
  const float4* rows;      // the level table
  uint32_t tcol;           // this warp's tensor-memory columns
  int bx, by;              // the tile's position in the domain's tile grid
  int tid, tx, i, j, ho;
  bool has_halo, own, edge, xlast, ylast;
};

// Thread 0: stage level k (levels 2..nk-1) into ring slot (k-2) % 4.
template <int S>
__device__ __forceinline__ void h4_issue(const HeviMaps& m, const H4Env& e, H4Up& u, int k) {
  using L = H4Layout<S>;
  u.issued = k;
  const int s = (k - 2) % S;
  float* st = e.ring + s * L::stage;
  uint64_t* bar = &e.bars[s];
  const int z = k - 1, xb = e.bx * kH4TX, j0 = 2 + e.by * kH4TY;
  mbar_arrive_expect_tx(bar, L::tx_bytes);
  tma_load_3d(st + L::oU, &m.u, xb, j0 - 1, z, bar);
  tma_load_3d(st + L::oV, &m.v, xb, j0 - 1, z, bar);
  tma_load_3d(st + L::oW, &m.w, xb, j0 - 1, z, bar);
  tma_load_3d(st + L::oP, &m.p, xb, j0 - 1, z, bar);
  tma_load_3d(st + L::oUF, &m.uf, xb, j0, z, bar);
  tma_load_3d(st + L::oVF, &m.vf, xb, j0, z, bar);
  tma_load_3d(st + L::oWF, &m.wf, xb, j0, z, bar);
  tma_load_3d(st + L::oPF, &m.pf, xb, j0, z, bar);
}

// The table vectors level k needs first, loaded a level ahead: row k's
// vector 1 (jcb, ijcb, irst8u, irst8v) and row k+1's vector 0 (rst8w and
// ij8w one level up).
__device__ __forceinline__ float4 ldg_last(const float4* p) {
  float4 v;
  asm volatile("ld.global.nc.L1::evict_last.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  return v;
}
__device__ __forceinline__ double ldg_last_d(const double* p) {
  double v;
  asm volatile("ld.global.nc.L1::evict_last.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}

__device__ __forceinline__ void h4_rows(const float4* rows, int k, float4 (&r)[2]) {
  const float4* rk = rows + 5 * k;
  r[0] = ldg_last(rk + 1);
  r[1] = ldg_last(rk + 5);
}

// One level k of the upward sweep: every shared-memory access is a fixed
// offset from the thread's base pointers plus the ring slot (k - 2) % 4.
// r holds level k's first table vectors, rn receives level k+1's.
template <int S, int DIV, bool STH, bool BUY, bool EDGE>
__device__ __forceinline__ void h4_level(const HeviMaps& m, const HeviArgs& a, const H4Env& e, H4Up& u, int k,
                                         const float4 (&r)[2], float4 (&rn)[2]) {
  static_assert(S == 4, "the ring slot is (k - 2) & 3");
  using L = H4Layout<S>;
  constexpr int BX = kHeviBoxX, TX = kH4TX, NT = kH4NT;
  const int s0 = (k - 2) & 3;                       // ring slot of level k
  const int s1 = (s0 + 1) & 3;                      // ring slot of level k+1
  const int buf = k & 1;                            // damped-pressure buffer
  const int nk = a.g.nk, plane = (int)a.g.plane;
  h4_rows(e.rows, k + 1, rn);   // rows k+1 and k+2 <= nk exist for every k <= nk-2
  // level k+1's copy: its phase is the ring pass of level k+1
  const uint32_t par = (uint32_t)((k - 1) >> 2) & 1u;
  if (!u.fail) u.fail = !mbar_wait(&e.bars[s1], par, a.spin);
  const float* tb = e.rb + s0 * L::stage;           // own cell in level k's boxes
  const float* tw1 = e.rb + s1 * L::stage + L::oW;  // own cell in level k+1's w box
  float* th0 = e.th + buf * L::t3h_floats;          // own cell in this level's damped-pressure plane
  const float4 c1 = r[0], n0 = r[1];
  const float rst8u = u.v0k.x, rst8v = u.v0k.y, rst8wk = u.v0k.z, ij8wk = u.v0k.w;
  const float rst8wk1 = n0.z, ij8wk1 = n0.w;
  const float jcbk = c1.x, ijcbk = c1.y, irst8u = c1.z, irst8v = c1.w;
  const float dts = a.dts, dxiv = a.dxiv, dyiv = a.dyiv, dziv = a.dziv;

  // diver3d.f90:318 (with phy2cnt.f90:219 for the contravariant w) at the
  // cell o (an offset from the thread's own cell)
  auto div3d = [&](int o) {
    float wck = tb[L::oW + o], wck1 = tw1[o];
    if constexpr (STH) { wck = wck * ij8wk; wck1 = wck1 * ij8wk1; }
    return (rst8wk * wck - rst8wk1 * wck1) * dziv +
           ((rst8u * tb[L::oU + o] - rst8u * tb[L::oU + o + 1]) * dxiv +
            (rst8v * tb[L::oV + o] - rst8v * tb[L::oV + o + BX]) * dyiv);
  };
  // pgrad.f90:300,341,363
  auto t3h_of = [&](float div, float pp) {
    float thv;
    if constexpr (DIV == 2) thv = pp + a.divch * div * ijcbk;
    else if constexpr (DIV == 1) thv = pp + a.divcv * jcbk * div;
    else thv = pp;
    return jcbk * thv;
  };
  const float div = div3d(0);
  const float pp = tb[L::oP];
  const float tc = t3h_of(div, pp);
  th0[0] = tc;
  const float t3v = (DIV >= 1) ? pp + a.divcv * jcbk * div : pp;                       // pgrad.f90:300
  if (e.has_halo) th0[e.ho] = t3h_of(div3d(e.ho), tb[L::oP + e.ho]);
  __syncthreads();
  if (e.tid == 0 && !u.fail && k + S - 1 <= nk - 1) {   // refill only after its copy was seen to land
    fence_proxy_async_smem();
    h4_issue<S>(m, e, u, k + S - 1);
  }

  // the vectors of the level table used from here on: row k's 2, 3 and aa of 4
  const float4* rk = e.rows + 5 * k;
  const float4 c2 = ldg_last(rk + 2), c3 = ldg_last(rk + 3);
  const double aa = ldg_last_d(reinterpret_cast<const double*>(rk + 4));
  const float uo = tb[L::oU], vo = tb[L::oV], vo1 = tb[L::oV + BX];
  const float uf = tb[L::oUF - BX], vf = tb[L::oVF - BX], vf1 = tb[L::oVF], wf = tb[L::oWF - BX],
              pf = tb[L::oPF - BX];
  const float wk = tb[L::oW], wk1 = tw1[0];
  // stepuv.f90:294,304 with pgrad.f90:379,389: the west u face, the east
  // face from the next lane (lane 31 forms its own); both v faces
  const float un0 = uo + dts * (uf + (th0[-1] - tc) * dxiv) * irst8u;
  float un1 = __shfl_down_sync(0xffffffffu, un0, 1);
  if (e.tx == TX - 1) un1 = tb[L::oU + 1] + dts * (tb[L::oUF - BX + 1] + (tc - th0[1]) * dxiv) * irst8u;
  const float vs = vo + dts * (vf + (th0[-BX] - tc) * dyiv) * irst8v;
  const float vn = vo1 + dts * (vf1 + (tc - th0[BX]) * dyiv) * irst8v;

  const float jcb8u = c2.x, jcb8v = c2.y, rcsq = c2.z, rst = c2.w;
  const float rbr = c3.x, ircsq = c3.y, irst8w = c3.z;
  const bool kend = (k == 2) || (k == nk - 2);
  if constexpr (!EDGE) {
    u.up[0] = un0;
    u.vp[0] = vs;
    if (kend) {   // vbcu.f90:120,134 (and vbcv): levels 1 and nk-1 copy levels 2 and nk-2
      const int dk = (k == 2 ? -1 : 1) * plane;
      u.up[dk] = un0;
      u.vp[dk] = vs;
    }
  } else if (e.own) {
    const Grid& g = a.g;
    const int i = e.i, j = e.j;
    if (e.edge) {
      store_periodic(a.u_new, g, STAG_U, i, j, k, un0);
      store_periodic(a.v_new, g, STAG_V, i, j, k, vs);
    } else {
      u.up[0] = un0;
      u.vp[0] = vs;
    }
    if (e.xlast) store_periodic(a.u_new, g, STAG_U, i + 1, j, k, un1);
    if (e.ylast) store_periodic(a.v_new, g, STAG_V, i, j + 1, k, vn);
    if (kend) {
      const int kc = k == 2 ? 1 : nk - 1;
      store_periodic(a.u_new, g, STAG_U, i, j, kc, un0);
      store_periodic(a.v_new, g, STAG_V, i, j, kc, vs);
      if (e.xlast) store_periodic(a.u_new, g, STAG_U, i + 1, j, kc, un1);
      if (e.ylast) store_periodic(a.v_new, g, STAG_V, i, j + 1, kc, vn);
    }
  }
  u.up += plane;
  u.vp += plane;

  float phd = (jcb8u * un0 - jcb8u * un1) * dxiv + (jcb8v * vs - jcb8v * vn) * dyiv;   // diver2d.f90:288
  phd = rcsq * phd;                                                                   // diverpih.f90:208
  const float pvd = rcsq * (wk - wk1) * dziv;                                         // diverpiv.f90:124
  const float fp = pf + phd + (1.f - a.weicoe) * (a.g05 * (wk + wk1) * rst + pvd);    // advbspi.f90:158
  u.qp[0] = pp + dts * fp * ijcbk;          // steppi.f90:217, explicit part of the new p'
  u.qp += NT;
  const float fpdvj = fp * ijcbk;                                                     // pgradiv.f90:149
  const float wb8s = (pp * rst + fp * rbr * a.dtw) * ircsq * a.g05n;                  // buoywsi.f90:171
  if (k >= 3) {
    const float wpg = (u.t3v_prev - t3v) * dziv;                                      // pgrad.f90:320
    float fw = wf + wpg + (u.fpdvj_prev - fpdvj) * a.dtdzw;                           // pgradiv.f90:163
    if constexpr (BUY) fw = fw + (u.wb8s_prev + wb8s);                                // buoywsi.f90:205
    const float wrhs = wk + dts * fw * irst8w;                                        // stepwi.f90:325
    // gaussel.f90:189-240 in double with the 1-D factors
    const double rr = (double)c3.w;
    const double f = (k == 3) ? (double)wrhs * aa : ((double)wrhs - rr * u.f_prev) * aa;
    tmem_st2(e.tcol + 2u * (uint32_t)(k - 3), (uint32_t)__double2loint(f), (uint32_t)__double2hiint(f));
    u.f_prev = f;
  }
  u.t3v_prev = t3v;
  u.fpdvj_prev = fpdvj;
  u.wb8s_prev = wb8s;
  u.v0k = n0;
}

template <int S, int DIV, bool STH, bool BUY, bool EDGE>
__device__ __forceinline__ void hevi4_tile(const HeviMaps& m, const HeviArgs& a, float* smem, uint32_t tmem, int bx,
                                           int by) {
  using L = H4Layout<S>;
  constexpr int TX = kH4TX, TY = kH4TY, BX = kHeviBoxX, NT = kH4NT;
  const Grid g = a.g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  H4Env e;
  e.bx = bx;
  e.by = by;
  e.tx = threadIdx.x;
  const int ty = threadIdx.y;
  e.tid = ty * TX + e.tx;
  const int i0 = 2 + bx * TX, j0 = 2 + by * TY;
  e.i = i0 + e.tx;
  e.j = j0 + ty;
  const int tid = e.tid, i = e.i, j = e.j;
  e.own = true; e.edge = false; e.xlast = false; e.ylast = false;
  if constexpr (EDGE) {
    const int ilast = min(i0 + TX - 1, ni - 2), jlast = min(j0 + TY - 1, nj - 2);
    e.own = (i <= ilast) && (j <= jlast);
    e.edge = (i <= 3) || (i >= ni - 2) || (j <= 3) || (j >= nj - 2);
    e.xlast = (i == ilast) && (i + 1 == ni - 1);
    e.ylast = (j == jlast) && (j + 1 == nj - 1);
  }
  const int tofs = (ty + 1) * BX + e.tx + 2;   // own cell in the boxes that start at j0-1
  e.ring = smem;
  e.rb = smem + tofs;
  float* t3hb = smem + S * L::stage;                              // 2 x [(TY+2)][BX]
  e.th = t3hb + tofs;
  float* qs = t3hb + 2 * L::t3h_floats;                           // [(k-2) * NT + tid]
  e.bars = reinterpret_cast<uint64_t*>(qs + (size_t)(nk - 3) * NT);
  e.rows = reinterpret_cast<const float4*>(a.lvl4);              // 5 vectors per level
  float4* dtab = reinterpret_cast<float4*>(e.bars + S);           // [k]: rcsq, rst, ijcb of the way down
  double* cps = reinterpret_cast<double*>(dtab + nk + 1);         // [k]: cp
  for (int n = tid; n <= nk; n += NT) {
    const float4* rn = e.rows + 5 * n;
    const float4 v1 = __ldg(rn + 1), v2 = __ldg(rn + 2);
    dtab[n] = make_float4(v2.z, v2.w, v1.y, 0.f);
    cps[n] = __ldg(reinterpret_cast<const double*>(rn + 4) + 1);
  }
  // tensor-memory columns of this warp: 128 per warp quadrant pair
  e.tcol = tmem + (uint32_t)(ty >> 2) * 128u;
  // halo point of the damped-pressure plane handled by this thread: rows
  // south/north of the tile, columns west/east of it (an offset from the
  // thread's own cell)
  {
    constexpr int NH = 2 * TX + 2 * TY;
    int hx = 0, hy = 0, n = tid;
    if (n < TX) { hx = n + 2; hy = 0; }
    else if ((n -= TX) < TX) { hx = n + 2; hy = TY + 1; }
    else if ((n -= TX) < TY) { hx = 1; hy = n + 1; }
    else { n -= TY; hx = TX + 2; hy = n + 1; }
    e.has_halo = tid < NH;
    e.ho = (hy * BX + hx) - tofs;
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&e.bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  H4Up u;
  u.up = a.u_new + (int)g.at(i, j, 2);
  u.vp = a.v_new + (int)g.at(i, j, 2);
  u.qp = qs + tid;
  u.v0k = __ldg(e.rows + 2 * 5);
  if (tid == 0)
    for (int k = 2; k <= min(S, nk - 1); ++k) h4_issue<S>(m, e, u, k);
  float4 ra[2], rb[2];
  h4_rows(e.rows, 2, ra);
  // level 2 waits for its own copy as well; then levels 2, 3, 4, 5 take
  // ring slots 0, 1, 2, 3 and so on
  if (!u.fail) u.fail = !mbar_wait(&e.bars[0], 0, a.spin);
  // two levels per iteration: the damped-pressure buffer (k & 1) is
  // compile-time, the ring slot and the phase are taken at run time
  int k = 2;
  for (; k + 1 <= nk - 2; k += 2) {
    h4_level<S, DIV, STH, BUY, EDGE>(m, a, e, u, k, ra, rb);
    h4_level<S, DIV, STH, BUY, EDGE>(m, a, e, u, k + 1, rb, ra);
  }
  if (k <= nk - 2) h4_level<S, DIV, STH, BUY, EDGE>(m, a, e, u, k, ra, rb);
  const bool fail = u.fail;
  const int issued = u.issued;
  uint64_t* bars = e.bars;
  const uint32_t tcol = e.tcol;
  const int plane = (int)g.plane;
  const float dts = a.dts, dziv = a.dziv, g05 = a.g05;
  const bool own = e.own, edge = e.edge, xlast = e.xlast, ylast = e.ylast;

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
  // update; sixteen levels per tensor-memory load.  cp(nk-2) = 0 makes the
  // recurrence the identity at the top level.
  const int ktop = nk - 2;
  double wd = 0.0;   // w(k+1) in double; w(nk-1) = 0 (vbcw.f90:481)
  float wup = 0.f, wkend = 0.f, pkend = 0.f, p3 = 0.f;
  const float weicoe = a.weicoe;
  float* wT = a.w_new + (int)g.at(i, j, ktop);
  float* pT = a.p_new + (int)g.at(i, j, ktop);
  // one level: w(k) from the eliminated right-hand side (lo, hi words),
  // then p'(k); the pointers step down a level
  const float* qp = qs + (size_t)(ktop - 2) * NT + tid;
  auto down = [&](int k, uint32_t lo, uint32_t hi) {
    const float4 d = dtab[k];   // rcsq, rst, ijcb
    wd = __hiloint2double((int)hi, (int)lo) - cps[k] * wd;   // gaussel.f90:254
    const float wk = (float)wd;
    // steppi.f90:217 with diverpiv.f90:124 and advbspi.f90:175 (the implicit part)
    const float pvd = d.x * (wk - wup) * dziv;
    const float fpw = weicoe * (g05 * (wk + wup) * d.y + pvd);
    const float pn = qp[0] + dts * fpw * d.z;
    if constexpr (!EDGE) {
      wT[0] = wk;
      pT[0] = pn;
    } else if (own) {
      if (edge) {
        store_periodic(a.w_new, g, STAG_S, i, j, k, wk);
        store_periodic(a.p_new, g, STAG_S, i, j, k, pn);
      } else {
        wT[0] = wk;
        pT[0] = pn;
      }
    }
    wT -= plane;
    pT -= plane;
    qp -= NT;
    p3 = pn;   // the value of level 3 after the loop
    wup = wk;
  };
  // the top chunk of four levels (partly above ktop), then whole chunks
  int c = (ktop - 3) / 4;
  {
    uint32_t r[8];
    tmem_ld8(tcol + 8u * (uint32_t)c, r);
    tmem_wait_ld();
#pragma unroll
    for (int e = 3; e >= 0; --e) {
      const int k = 3 + 4 * c + e;
      if (k > ktop) continue;
      down(k, r[2 * e], r[2 * e + 1]);
      if (k == ktop) { wkend = wup; pkend = p3; }
    }
  }
  for (--c; c >= 0; --c) {
    uint32_t r[8];
    tmem_ld8(tcol + 8u * (uint32_t)c, r);
    tmem_wait_ld();
#pragma unroll
    for (int e = 3; e >= 0; --e) down(3 + 4 * c + e, r[2 * e], r[2 * e + 1]);
  }
  // level 2: w(2) = 0 (vbcw.f90:317, flat terrain) and its p', then the
  // boundary rows of vbcw.f90:285,317,471,481 (wc = w / jcb8w when
  // stretched) and vbcp.f90:126-160, and level nk of u, v, p' carried over
  if (!own) return;
  const float4 d = dtab[2];   // rcsq, rst, ijcb of level 2
  const float pvd = d.x * (0.f - wup) * dziv;
  const float fpw = weicoe * (g05 * (0.f + wup) * d.y + pvd);
  const float p2 = qs[tid] + dts * fpw * d.z;
  const float jw3 = __ldg(a.col + C_JCB8W * (nk + 1) + 3), jwt = __ldg(a.col + C_JCB8W * (nk + 1) + nk - 2);
  const float wc3 = STH ? wup / jw3 : wup;
  const float wct = STH ? wkend / jwt : wkend;
  if (!EDGE || !edge) a.p_new[g.at(i, j, 2)] = p2;
  else store_periodic(a.p_new, g, STAG_S, i, j, 2, p2);
  store_periodic(a.w_new, g, STAG_S, i, j, 1, -jw3 * wc3 - 0.f);
  store_periodic(a.w_new, g, STAG_S, i, j, 2, 0.f);
  store_periodic(a.w_new, g, STAG_S, i, j, nk - 1, 0.f);
  store_periodic(a.w_new, g, STAG_S, i, j, nk, -jwt * wct - 0.f);
  store_periodic(a.p_new, g, STAG_S, i, j, 1, (a.bbc == 2) ? 2.f * p2 - p3 : p2);
  store_periodic(a.p_new, g, STAG_S, i, j, nk - 1, pkend);
  store_periodic(a.p_new, g, STAG_S, i, j, nk, a.p_old[g.at(i, j, nk)]);
  store_periodic(a.u_new, g, STAG_U, i, j, nk, a.u_old[g.at(i, j, nk)]);
  store_periodic(a.v_new, g, STAG_V, i, j, nk, a.v_old[g.at(i, j, nk)]);
  if (xlast) store_periodic(a.u_new, g, STAG_U, i + 1, j, nk, a.u_old[g.at(i + 1, j, nk)]);
  if (ylast) store_periodic(a.v_new, g, STAG_V, i, j + 1, nk, a.v_old[g.at(i, j + 1, nk)]);
}

// One block: allocate the block's tensor memory, run tile (bx, by) of a
// tx_n x ty_n tile grid (the tiles on its border take the edge path), free
// the tensor memory.
template <int S, int DIV, bool STH, bool BUY>
__device__ __forceinline__ void hevi4_block(const HeviMaps& m, const HeviArgs& a, int bx, int by, int tx_n,
                                            int ty_n) {
  extern __shared__ __align__(128) float smem[];
  __shared__ uint32_t tmem_slot;
  const int warp = threadIdx.y;   // blockDim = (32, 8): one warp per thread row
  if (warp == 0) tmem_alloc(&tmem_slot, kH4TmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  // lanes 32(w % 4) .. 32(w % 4) + 31 belong to warp w
  const uint32_t tmem = tmem_slot + ((uint32_t)((warp & 3) * 32) << 16);
  const bool edge = bx == 0 || bx == tx_n - 1 || by == 0 || by == ty_n - 1;
  if (edge) hevi4_tile<S, DIV, STH, BUY, true>(m, a, smem, tmem, bx, by);
  else hevi4_tile<S, DIV, STH, BUY, false>(m, a, smem, tmem, bx, by);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem_slot, kH4TmemCols);
  }
}

template <int S, int DIV, bool STH, bool BUY>
__global__ void __launch_bounds__(kH4NT, 2) k_hevi4(const __grid_constant__ HeviMaps m, const HeviArgs a) {
  hevi4_block<S, DIV, STH, BUY>(m, a, blockIdx.x, blockIdx.y, gridDim.x, gridDim.y);
}

// Every member of an ensemble in one launch: block b belongs to the member
// whose first_block is the largest not above b (the jobs are in block
// order), which runs its tile b - first_block (the same 32 x 8 tiles as
// tile 0's batch).
template <int S, int DIV, bool STH, bool BUY>
__global__ void __launch_bounds__(kH4NT, 2) k_hevi4_batch(const HeviJob* __restrict__ jobs, int njobs) {
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
  // the member's arguments in shared memory: read every level without
  // global loads that the kernel's stores could alias
  __shared__ alignas(16) uint32_t sa_words[sizeof(HeviArgs) / 4];
  static_assert(sizeof(HeviArgs) % 4 == 0, "HeviArgs is copied as words");
  const int tid = threadIdx.y * kH4TX + threadIdx.x;
  const uint32_t* src = reinterpret_cast<const uint32_t*>(&job.args);
  for (int w = tid; w < (int)(sizeof(HeviArgs) / 4); w += kH4NT) sa_words[w] = src[w];
  __syncthreads();
  const HeviArgs& sa = *reinterpret_cast<const HeviArgs*>(sa_words);
  const int ty_n = (sa.g.nj - 3 + kH4TY - 1) / kH4TY;
  hevi4_block<S, DIV, STH, BUY>(job.maps, sa, t % job.tiles_x, t / job.tiles_x, job.tiles_x, ty_n);
}

template <int S, int DIV, bool STH, bool BUY>
int launch_h4(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st) {
  using L = H4Layout<S>;
  const Grid& g = a.g;
  const size_t bytes = L::bytes(g.nk) > (size_t)kH4MinSmem ? L::bytes(g.nk) : (size_t)kH4MinSmem;
  // two blocks per SM: 228 KB less 1 KB reserved per block and the static tensor-memory slot
  if (bytes > 113 * 1024 - 64) return CRESS_E_UNSUPPORTED;
  auto kern = k_hevi4<S, DIV, STH, BUY>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
    return CRESS_E_CUDA;
  const int nx = g.ni - 3, ny = g.nj - 3;
  dim3 block(kH4TX, kH4TY);
  dim3 grid((nx + kH4TX - 1) / kH4TX, (ny + kH4TY - 1) / kH4TY);
  kern<<<grid, block, bytes, st>>>(maps, a);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

template <int DIV>
int launch_h4_div(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st) {
  constexpr int S = 4;
  const bool sth = a.sthopt != 0, buy = a.buyopt == 1;
  if (sth) return buy ? launch_h4<S, DIV, true, true>(a, maps, st) : launch_h4<S, DIV, true, false>(a, maps, st);
  return buy ? launch_h4<S, DIV, false, true>(a, maps, st) : launch_h4<S, DIV, false, false>(a, maps, st);
}

template <int DIV, bool STH, bool BUY>
int launch_h4_batch_t(const HeviJob* jobs_d, int njobs, int nblocks, int nk_max, cudaStream_t st) {
  constexpr int S = 4;
  using L = H4Layout<S>;
  const size_t bytes = L::bytes(nk_max) > (size_t)kH4MinSmem ? L::bytes(nk_max) : (size_t)kH4MinSmem;
  // two blocks per SM, each also holding its member's arguments
  if (bytes > 113 * 1024 - 64 - sizeof(HeviArgs)) return CRESS_E_UNSUPPORTED;
  auto kern = k_hevi4_batch<S, DIV, STH, BUY>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
    return CRESS_E_CUDA;
  kern<<<nblocks, dim3(kH4TX, kH4TY), bytes, st>>>(jobs_d, njobs);
  return cudaGetLastError() == cudaSuccess ? 0 : CRESS_E_CUDA;
}

}  // namespace

int launch_hevi4_batch(const HeviJob* jobs_d, int njobs, int nblocks, int nk_max, int divopt, bool sth, bool buy,
                       cudaStream_t st) {
  if (nk_max > kHevi3MaxNk) return CRESS_E_UNSUPPORTED;
  auto pick = [&](auto div) -> int {
    constexpr int D = decltype(div)::value;
    if (sth) return buy ? launch_h4_batch_t<D, true, true>(jobs_d, njobs, nblocks, nk_max, st)
                        : launch_h4_batch_t<D, true, false>(jobs_d, njobs, nblocks, nk_max, st);
    return buy ? launch_h4_batch_t<D, false, true>(jobs_d, njobs, nblocks, nk_max, st)
               : launch_h4_batch_t<D, false, false>(jobs_d, njobs, nblocks, nk_max, st);
  };
  switch (divopt) {
    case 2: return pick(std::integral_constant<int, 2>{});
    case 1: return pick(std::integral_constant<int, 1>{});
    default: return pick(std::integral_constant<int, 0>{});
  }
}

int launch_hevi4(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st) {
  if (!a.lvl4 || a.g.nk > kHevi3MaxNk || a.g.nk < 8 || a.g.count() >= (1LL << 31)) return CRESS_E_UNSUPPORTED;
  switch (a.divopt) {
    case 2: return launch_h4_div<2>(a, maps, st);
    case 1: return launch_h4_div<1>(a, maps, st);
    default: return launch_h4_div<0>(a, maps, st);
  }
}

}  // namespace cress

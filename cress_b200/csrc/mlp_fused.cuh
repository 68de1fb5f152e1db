// Learned microphysics, fused inference for sm_100a: one persistent kernel
// takes 128-cell tiles through features -> four tcgen05 BF16 GEMMs ->
// application, with the activations kept in shared memory and the
// accumulator in tensor memory (no activation traffic to HBM).  Included by
// micro.cu only (it shares its cell loaders and Koenig tables).
//
// Roles (320 threads): warps 0-7 form the features (warps 0-3, one cell per
// thread), read the accumulators (warp w reads tensor-memory lanes
// 32(w%4).. and half of the columns), apply bias + SiLU and write the next
// layer's BF16 activations into shared memory in the K-major 128-byte
// swizzle the MMA reads; warp 8 (one lane) streams the W1, W2, W3 column
// blocks (128 output rows x 64 K, BF16) and W4 through a 2-stage TMA
// ring; warp 9 (one lane) issues the MMAs (N = 128 per block into one half
// of the 256 accumulator columns).  Two blocks share an SM.  Per tile: x_full (features
// written), then per layer acc_full (accumulator ready) and h_full (next
// activations written).  Every mbarrier wait is bounded; on expiry the
// kernel records CRESS_E_TIMEOUT, stops all roles, drains its copies and
// MMAs (bounded) and frees tensor memory.
#pragma once
#include "umma.cuh"

namespace cress {
namespace {

constexpr int kFusedThreads = 320;
constexpr int kFusedTile = 128;
constexpr uint32_t kHBytes = 4 * 16384;      // activations: 4 K-blocks of 128 x 64 bf16
constexpr uint32_t kWStage = 16384;          // one W block: 128 output rows x 64 K of W1..W3 (or 64 x 64 of W4)
constexpr uint32_t kW4Block = 8192;          // one 64 x 64 K-block of W4^T
// about 100 KB, so two blocks share an SM and one's epilogue overlaps the
// other's MMAs
constexpr uint32_t kFusedSmem = kHBytes + 2 * kWStage + 4 * (3 * kMlpH + kMlpN4) + 1024;

struct FusedMaps {
  // W1^T [256][64], W2^T, W3^T [256][256] (boxes of 128 rows), W4^T [64][256] (box 64 rows)
  CUtensorMap w1, w2, w3, w4;
};

struct FusedArgs {
  const float* w;          // present-level w (feature: vertical velocity at the cell centre)
  const float* norm;
  const float* params;     // biases at MlpLayout::B1..B4
  long long ncell;
  float resid_tol;
  int* fb_list;
  int* fb_count;
  int fb_cap;
  unsigned long long* stats;
  int* err;
};

// Row r (0..127), columns c0..c0+15 of a K-block, as 16 bf16 packed in 8 words.
__device__ __forceinline__ void store_row16(unsigned char* kblock, int r, int c0, const uint32_t (&w)[8]) {
  const int ch = (c0 >> 3);   // 16-byte chunk index within the 128-byte row (c0 % 64 / 8)
  uint4* p0 = reinterpret_cast<uint4*>(kblock + r * 128 + (((ch) ^ (r & 7)) << 4));
  uint4* p1 = reinterpret_cast<uint4*>(kblock + r * 128 + (((ch + 1) ^ (r & 7)) << 4));
  *p0 = make_uint4(w[0], w[1], w[2], w[3]);
  *p1 = make_uint4(w[4], w[5], w[6], w[7]);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}


// The eight epilogue warps.  Warps 0-3 own one cell each per tile (row =
// tensor-memory lane): features, fall speeds and the CFL limit, and at the
// end the application or the fallback; all eight turn accumulators into
// activations (warp w: lanes 32(w%4).., columns 128(w/4)..+127).
__device__ __forceinline__ void fused_epilogue(const MicroArgs& a, const FusedArgs& p, unsigned char* H,
                                               const float* bias, uint32_t tmem, uint64_t* x_full,
                                               uint64_t* h_full, uint64_t* acc_full, volatile int* vfail,
                                               long long ntiles) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lg = warp & 3, half = warp >> 2;
  const int row = lg * 32 + lane;
  const unsigned full = 0xffffffffu;
  const uint32_t lane_base = static_cast<uint32_t>(lg * 32) << 16;
  const Grid& g = a.g;
  int pha = 0;
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    if (__any_sync(full, *vfail != 0)) break;
    const long long n = t * kFusedTile + row;
    bool env = false;
    if (half == 0) {
      float f[kMlpIn];
      float lim = 3.0e38f;
      if (n < p.ncell) {
        int k;
        const long long id = cell_index(g, n, k);
        MCell c;
        load_cell(a, id, k, c);
        load_future(a, id, c);
        mlp_features(c, w_center(p.w, id, g.plane), f);
        termblk_cell(a.thresq, c);
        store_speeds(a, id, c);
        const float dzjcb = a.dz * __ldg(a.col + C_JCB * (g.nk + 1) + k);
        lim = fminf(lim, dzjcb / (c.ucq + 1.e-20f));
        lim = fminf(lim, dzjcb / (c.urq + 1.e-20f));
        lim = fminf(lim, dzjcb / (c.uiq + 1.e-20f));
        lim = fminf(lim, dzjcb / (c.usq + 1.e-20f));
        lim = fminf(lim, dzjcb / (c.ugq + 1.e-20f));
        env = true;
#pragma unroll
        for (int m = 0; m < kMlpIn; ++m) {
          const float lo = p.norm[kNormXmin + m], hi = p.norm[kNormXmax + m], mg = .05f * (hi - lo);
          env &= f[m] >= lo - mg && f[m] <= hi + mg;
        }
      } else {
#pragma unroll
        for (int m = 0; m < kMlpIn; ++m) f[m] = p.norm[kNormXmean + m];
      }
      uint32_t wd[8];
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        const float v0 = (f[2 * m] - p.norm[kNormXmean + 2 * m]) / p.norm[kNormXstd + 2 * m];
        const float v1 = (f[2 * m + 1] - p.norm[kNormXmean + 2 * m + 1]) / p.norm[kNormXstd + 2 * m + 1];
        const __nv_bfloat162 hv = __floats2bfloat162_rn(v0, v1);
        wd[m] = *reinterpret_cast<const uint32_t*>(&hv);
      }
      unsigned char* xr = H + row * 128;
#pragma unroll
      for (int ch = 0; ch < 8; ++ch) {
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (ch == 0) v = make_uint4(wd[0], wd[1], wd[2], wd[3]);
        if (ch == 1) v = make_uint4(wd[4], wd[5], wd[6], wd[7]);
        *reinterpret_cast<uint4*>(xr + ((ch ^ (row & 7)) << 4)) = v;
      }
      for (int o = 16; o > 0; o >>= 1) lim = fminf(lim, __shfl_xor_sync(full, lim, o));
      if (lane == 0 && lim < 3.0e38f) atomicMin(a.dtp_bits, __float_as_int(lim));
    }
    fence_proxy_async_smem();
    mbar_arrive(x_full);
    bool ok = true;
    for (int l = 0; l < 3; ++l) {
      ok = __all_sync(full, mbar_wait_sleep(acc_full, pha));
      pha ^= 1;
      if (!ok) break;
      tc_fence_after();
#pragma unroll 1
      for (int c0 = half * 128; c0 < half * 128 + 128; c0 += 16) {
        uint32_t r[16];
        tmem_ld16(tmem + lane_base + static_cast<uint32_t>(c0), r);
        tmem_wait_ld();
        uint32_t w[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float v0 = silu(__uint_as_float(r[2 * q]) + bias[l * kMlpH + c0 + 2 * q]);
          const float v1 = silu(__uint_as_float(r[2 * q + 1]) + bias[l * kMlpH + c0 + 2 * q + 1]);
          const __nv_bfloat162 hv = __floats2bfloat162_rn(v0, v1);
          w[q] = *reinterpret_cast<const uint32_t*>(&hv);
        }
        store_row16(H + (c0 >> 6) * 16384, row, c0 & 63, w);
      }
      tc_fence_before();
      fence_proxy_async_smem();
      mbar_arrive(h_full);
    }
    if (!ok) { *vfail = 1; break; }
    ok = __all_sync(full, mbar_wait_sleep(acc_full, pha));
    pha ^= 1;
    if (!ok) { *vfail = 1; break; }
    tc_fence_after();
    if (half == 0) {
      uint32_t r[16];
      tmem_ld16(tmem + lane_base, r);
      tmem_wait_ld();
      bool used = false, fb = false;
      if (n < p.ncell) {
        float ys[kMlpOut];
#pragma unroll
        for (int m = 0; m < kMlpOut; ++m) ys[m] = __uint_as_float(r[m]) + bias[3 * kMlpH + m];
        used = mlp_apply_cell(a, n, ys, env, p.norm, p.resid_tol);
        fb = !used;
      }
      // one set of atomics per warp: the counts of network and fallback
      // cells, and the fallback cells' slots in the list
      const unsigned mu = __ballot_sync(full, used), mf = __ballot_sync(full, fb);
      int base = 0;
      if (lane == 0) {
        if (mu) atomicAdd(p.stats, (unsigned long long)__popc(mu));
        if (mf) {
          atomicAdd(p.stats + 1, (unsigned long long)__popc(mf));
          base = atomicAdd(p.fb_count, __popc(mf));
        }
      }
      base = __shfl_sync(full, base, 0);
      if (fb) {
        const int slot = base + __popc(mf & ((1u << lane) - 1u));
        if (slot < p.fb_cap) p.fb_list[slot] = (int)n;
      }
    }
    tc_fence_before();
  }
}

__global__ void __launch_bounds__(kFusedThreads, 2)
    k_mlp_fused(const __grid_constant__ FusedMaps maps, const MicroArgs a, const FusedArgs p) {
  extern __shared__ unsigned char fsm_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(fsm_raw) + 1023) &
                                                       ~static_cast<uintptr_t>(1023));
  unsigned char* H = sm;                          // 4 K-blocks of activations (X in K-block 0)
  unsigned char* WS = sm + kHBytes;               // 2-stage W ring
  float* bias = reinterpret_cast<float*>(WS + 2 * kWStage);   // b1, b2, b3 (256 each), b4 (64)
  __shared__ __align__(8) uint64_t x_full, h_full, acc_full, w_full[2], w_empty[2], mma_done;
  __shared__ uint32_t tmem_slot;
  __shared__ int fail;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long ntiles = (p.ncell + kFusedTile - 1) / kFusedTile;
  volatile int* vfail = &fail;

  for (int n = threadIdx.x; n < 3 * kMlpH + kMlpN4; n += kFusedThreads) {
    const int l = n / kMlpH;   // 0..2: b1..b3, 3: b4
    const int off = l == 0 ? MlpLayout::B1 : l == 1 ? MlpLayout::B2 : l == 2 ? MlpLayout::B3 : MlpLayout::B4;
    bias[n] = __ldg(p.params + off + (n - l * kMlpH));
  }
  if (threadIdx.x == 0) {
    mbar_init(&x_full, 256);
    mbar_init(&h_full, 256);
    mbar_init(&acc_full, 1);
    mbar_init(&mma_done, 1);
    for (int s = 0; s < 2; ++s) {
      mbar_init(&w_full[s], 1);
      mbar_init(&w_empty[s], 1);
    }
    fence_mbar_init();
    fail = 0;
  }
  if (warp == 0) tmem_alloc(&tmem_slot, 256);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  // Per tile the W blocks stream in one order: layer 1 (K-block 0, output
  // rows 0-127 then 128-255), layers 2 and 3 (K-blocks 0-3, each in the
  // two row halves), layer 4 (K-blocks 0-3 of W4^T, 64 rows each).
  if (warp == 8) {
    // ---------------------------------------------------------- producer
    if (lane == 0) {
      int cnt = 0;
      for (long long t = blockIdx.x; t < ntiles && !*vfail; t += gridDim.x)
        for (int l = 0; l < 4 && !*vfail; ++l)
          for (int kb = 0; kb < (l == 0 ? 1 : 4) && !*vfail; ++kb)
            for (int h = 0; h < (l == 3 ? 1 : 2); ++h, ++cnt) {
              const int s = cnt & 1, r = cnt >> 1;
              if (*vfail || !mbar_wait_sleep(&w_empty[s], (r & 1) ^ 1)) { *vfail = 1; break; }
              mbar_arrive_expect_tx(&w_full[s], l == 3 ? kW4Block : kWStage);
              const CUtensorMap* mp = l == 0 ? &maps.w1 : l == 1 ? &maps.w2 : l == 2 ? &maps.w3 : &maps.w4;
              tma_load_2d(WS + s * kWStage, mp, kb * 64, h * 128, &w_full[s]);
            }
      // every copy issued lands before the block may leave: the last use of
      // each stage is waited for (bounded)
      for (int c = cnt - 1; c >= 0 && c >= cnt - 2; --c) mbar_wait(&w_full[c & 1], (c >> 1) & 1);
    }
  } else if (warp == 9) {
    // --------------------------------------------------------------- MMA
    if (lane == 0) {
      const uint32_t id128 = idesc_bf16_f32(128, 128), id64 = idesc_bf16_f32(128, 64);
      const uint32_t hs = smem_u32(H), ws = smem_u32(WS);
      int cnt = 0, phx = 0, phh = 0;
      bool ok = true;
      for (long long t = blockIdx.x; ok && t < ntiles; t += gridDim.x) {
        if (*vfail || !mbar_wait_sleep(&x_full, phx)) { ok = false; break; }
        phx ^= 1;
        for (int l = 0; l < 4 && ok; ++l) {
          if (l > 0) {
            if (*vfail || !mbar_wait_sleep(&h_full, phh)) { ok = false; break; }
            phh ^= 1;
          }
          tc_fence_after();
          for (int kb = 0; kb < (l == 0 ? 1 : 4) && ok; ++kb)
            for (int h = 0; h < (l == 3 ? 1 : 2); ++h, ++cnt) {
              const int s = cnt & 1, r = cnt >> 1;
              if (*vfail || !mbar_wait_sleep(&w_full[s], r & 1)) { ok = false; break; }
              tc_fence_after();
              // layers 1-3: N = 128 into accumulator columns 128h..; layer 4: N = 64
#pragma unroll
              for (int k = 0; k < 4; ++k)
                umma_bf16(tmem + (uint32_t)(h * 128), sw128_desc(hs + kb * 16384 + k * 32),
                          sw128_desc(ws + s * kWStage + k * 32), l == 3 ? id64 : id128, (kb | k) != 0 ? 1u : 0u);
              umma_commit(&w_empty[s]);
            }
          if (ok) umma_commit(&acc_full);
        }
      }
      if (!ok) *vfail = 1;
      umma_commit(&mma_done);   // arrives once every MMA issued above has completed
      mbar_wait(&mma_done, 0);
    }
  } else {
    fused_epilogue(a, p, H, bias, tmem, &x_full, &h_full, &acc_full, vfail, ntiles);
  }
  tc_fence_before();
  __syncthreads();
  if (*vfail && threadIdx.x == 0 && p.err) atomicExch(p.err, CRESS_E_TIMEOUT);
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

}  // namespace
}  // namespace cress

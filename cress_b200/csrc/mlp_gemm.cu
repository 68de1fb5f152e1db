// BF16 tensor-core GEMM for sm_100a (tcgen05 + TMA + tensor memory) with a
// fused bias / SiLU / SiLU-derivative epilogue: the building block of the
// microphysics MLP's training (forward, backward and weight gradients).
//
// One CTA computes a 128 x BN tile of C.  Warp 0 (one lane) streams
// 128 x 64 tiles of A and BN x 64 tiles of B with TMA (128-byte swizzle)
// into a ring of stages (2 for BN = 256, so two CTAs share an SM and one's
// epilogue overlaps the other's MMAs; 4 otherwise); warp 1 (one lane)
// issues the tcgen05.mma K steps (4 per stage) into a 128 x BN FP32
// accumulator in tensor memory and commits each stage back to its producer
// barrier; all eight warps then read the accumulator (warp w owns rows
// 32(w%4)..+31 and half of the columns) and apply the epilogue.  Every mbarrier wait is bounded: on timeout the kernel records
// CRESS_E_TIMEOUT in the error word, waits (bounded) for its issued copies
// and MMAs, frees tensor memory and returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdio>
#include <mutex>
#include "mlp.cuh"
#include "status.h"
#include "tma.cuh"
#include "umma.cuh"

namespace cress {

int set_error(int code, const char* fmt, ...);

namespace {

constexpr int kBM = 128, kBK = 64, kThreads = 256;

template <int BN>
struct GemmCfg {
  static constexpr int S = BN == 256 ? 2 : 4;
  static constexpr int A_BYTES = kBM * kBK * 2;
  static constexpr int B_BYTES = BN * kBK * 2;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int SMEM = S * STAGE + 1024;
  static constexpr uint32_t TMEM_COLS = BN < 32 ? 32 : BN;
};


template <int BN>
__global__ void __launch_bounds__(kThreads, 2)
    k_gemm_bf16(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, const GemmArgs g) {
  using Cfg = GemmCfg<BN>;
  extern __shared__ unsigned char dsm_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(dsm_raw) + 1023) &
                                                       ~static_cast<uintptr_t>(1023));
  constexpr int kStages = Cfg::S;
  __shared__ __align__(8) uint64_t full[kStages], empty[kStages], done;
  __shared__ uint32_t tmem_slot;
  __shared__ int fail;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
  const int KB = g.K / kBK;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&done, 1);
    fence_mbar_init();
    fail = 0;
  }
  if (warp == 0) tmem_alloc(&tmem_slot, Cfg::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  volatile int* vfail = &fail;

  if (warp == 0 && lane == 0) {
    // producer
    int issued = 0;
    for (int kb = 0; kb < KB; ++kb) {
      const int s = kb % kStages, r = kb / kStages;
      if (*vfail || !mbar_wait_sleep(&empty[s], (r & 1) ^ 1)) {
        *vfail = 1;
        break;
      }
      unsigned char* a = sm + s * Cfg::STAGE;
      mbar_arrive_expect_tx(&full[s], Cfg::STAGE);
      tma_load_2d(a, &ta, kb * kBK, m0, &full[s]);
      tma_load_2d(a + Cfg::A_BYTES, &tb, kb * kBK, n0, &full[s]);
      ++issued;
    }
    if (*vfail) {
      // drain: the last round issued on each stage completes after all
      // earlier ones (bounded waits; nothing to do on a second timeout)
      for (int kb = issued - 1; kb >= 0 && kb >= issued - kStages; --kb)
        mbar_wait(&full[kb % kStages], (kb / kStages) & 1);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    const uint32_t idesc = idesc_bf16_f32(kBM, BN);
    for (int kb = 0; kb < KB; ++kb) {
      const int s = kb % kStages, r = kb / kStages;
      if (*vfail || !mbar_wait_sleep(&full[s], r & 1)) {
        *vfail = 1;
        break;
      }
      tc_fence_after();
      const uint32_t a = smem_u32(sm + s * Cfg::STAGE), b = a + Cfg::A_BYTES;
#pragma unroll
      for (int k = 0; k < kBK / 16; ++k)
        umma_bf16(tmem, sw128_desc(a + k * 32), sw128_desc(b + k * 32), idesc, (kb | k) != 0 ? 1u : 0u);
      umma_commit(&empty[s]);
    }
    umma_commit(&done);   // arrives once every MMA issued above has completed
  }
  const bool waited = mbar_wait_sleep(&done, 0);
  tc_fence_after();
  const int good = __syncthreads_and(waited && !*vfail);
  if (!good) {
    if (threadIdx.x == 0 && g.err) atomicExch(g.err, CRESS_E_TIMEOUT);
  } else {
    const int lg = warp & 3;                      // lane group of tensor memory this warp may read
    const int row = m0 + lg * 32 + lane;
    constexpr int HALF = BN / 2;
#pragma unroll 1
    for (int c0 = (warp >> 2) * HALF; c0 < (warp >> 2) * HALF + HALF; c0 += 16) {
      uint32_t r[16];
      tmem_ld16(tmem + (static_cast<uint32_t>(lg * 32) << 16) + static_cast<uint32_t>(c0), r);
      tmem_wait_ld();
      const int col0 = n0 + c0;
      float a[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        float v = __uint_as_float(r[j]);
        if (g.bias) v += __ldg(g.bias + col0 + j);
        float o = v;
        if (g.act == 1) {
          o = silu(v);
        } else if (g.act == 2) {
          o = v * dsilu(__ldg(g.aux + (size_t)row * g.ldaux + col0 + j));
        }
        a[j] = o;
        r[j] = __float_as_uint(g.act == 1 ? v : o);
      }
      if (g.out_f32) {
        float4* dst = reinterpret_cast<float4*>(g.out_f32 + (size_t)row * g.ldf + col0);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          dst[q] = make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                               __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3]));
      }
      if (g.out_bf) {
        uint4* dst = reinterpret_cast<uint4*>(g.out_bf + (size_t)row * g.ldb + col0);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          uint32_t w[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const __nv_bfloat162 h = __floats2bfloat162_rn(a[8 * q + 2 * e], a[8 * q + 2 * e + 1]);
            w[e] = *reinterpret_cast<const uint32_t*>(&h);
          }
          dst[q] = make_uint4(w[0], w[1], w[2], w[3]);
        }
      }
      if (g.out_bt) {
#pragma unroll
        for (int j = 0; j < 16; ++j) g.out_bt[(size_t)(col0 + j) * g.ldt + row] = __float2bfloat16_rn(a[j]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, Cfg::TMEM_COLS);
  }
}

typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                             const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                             CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encoder() {
  static EncodeFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeFn>(p);
  });
  return fn;
}

// Row-major [rows][cols] BF16 matrix with leading dimension ld, boxes of
// `box_rows` x 64 with the 128-byte swizzle.
int encode_bf16(CUtensorMap* m, const bf16* base, int rows, int cols, int ld, int box_rows) {
  EncodeFn fn = encoder();
  if (!fn) return set_error(CRESS_E_CUDA, "cuTensorMapEncodeTiled entry point unavailable");
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {64, (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? CRESS_OK : set_error(CRESS_E_CUDA, "cuTensorMapEncodeTiled (bf16) failed (%d)", (int)r);
}

template <int BN>
int launch_gemm(const bf16* A, int lda, const bf16* B, int ldb, const GemmArgs& g, cudaStream_t st) {
  using Cfg = GemmCfg<BN>;
  CUtensorMap ta, tb;
  int rc = encode_bf16(&ta, A, g.M, g.K, lda, kBM);
  if (rc) return rc;
  if ((rc = encode_bf16(&tb, B, g.N, g.K, ldb, BN))) return rc;
  if (cudaFuncSetAttribute(k_gemm_bf16<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM) !=
      cudaSuccess)
    return set_error(CRESS_E_CUDA, "gemm smem attribute");
  dim3 grid(g.M / kBM, g.N / BN);
  k_gemm_bf16<BN><<<grid, kThreads, Cfg::SMEM, st>>>(ta, tb, g);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CRESS_OK : set_error(CRESS_E_CUDA, "gemm launch: %s", cudaGetErrorString(e));
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

}  // namespace

int encode_bf16_map(CUtensorMap* m, const bf16* base, int rows, int cols, int ld, int box_rows) {
  return encode_bf16(m, base, rows, cols, ld, box_rows);
}

int gemm_bf16(const bf16* A, int lda, const bf16* B, int ldb, const GemmArgs& g, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0 || g.K <= 0 || g.M % kBM || g.K % kBK || g.N % 64)
    return set_error(CRESS_E_ARG, "gemm: M=%d N=%d K=%d (need M%%128, N%%64, K%%64 == 0)", g.M, g.N, g.K);
  if (lda % 8 || ldb % 8 || lda < g.K || ldb < g.K || !aligned16(A) || !aligned16(B))
    return set_error(CRESS_E_ARG, "gemm: operands need 16-byte alignment and ld >= K, ld %% 8 == 0");
  if ((g.out_f32 && (g.ldf % 4 || g.ldf < g.N || !aligned16(g.out_f32))) ||
      (g.out_bf && (g.ldb % 8 || g.ldb < g.N || !aligned16(g.out_bf))) || (g.out_bt && g.ldt < g.M) ||
      (g.act == 2 && (!g.aux || g.ldaux < g.N)))
    return set_error(CRESS_E_ARG, "gemm: bad output / aux leading dimensions");
  if (g.N % 256 == 0) return launch_gemm<256>(A, lda, B, ldb, g, st);
  if (g.N % 128 == 0) return launch_gemm<128>(A, lda, B, ldb, g, st);
  return launch_gemm<64>(A, lda, B, ldb, g, st);
}

}  // namespace cress

// Learned cold-rain microphysics: the per-cell MLP (internal interface).
//
// Network 16 -> 256 -> 256 -> 256 -> 9 with SiLU, BF16 weights and
// activations, FP32 accumulation in tensor memory.  For the tensor-core
// GEMMs the input layer is padded to K = 64 and the output layer to
// N = 64 (zero rows / columns that stay zero under training).
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "status.h"

namespace cress {

typedef __nv_bfloat16 bf16;

constexpr int kMlpIn = 16;      // input features
constexpr int kMlpOut = 9;      // tendencies of qv, qc, qr, qi, qs, qg, ni, ns, ng
constexpr int kMlpK1 = 64;      // padded input width
constexpr int kMlpH = 256;      // hidden width
constexpr int kMlpN4 = 64;      // padded output width

// Parameter offsets (floats) in the master buffer: layers 1-3 keep W as
// [N][K] (the forward GEMM's B operand), layer 4 as [K][N].
struct MlpLayout {
  static constexpr int W1 = 0;                                 // [256][64]
  static constexpr int B1 = W1 + kMlpH * kMlpK1;               // [256]
  static constexpr int W2 = B1 + kMlpH;                        // [256][256]
  static constexpr int B2 = W2 + kMlpH * kMlpH;
  static constexpr int W3 = B2 + kMlpH;                        // [256][256]
  static constexpr int B3 = W3 + kMlpH * kMlpH;
  static constexpr int W4 = B3 + kMlpH;                        // [256][64] (K x N)
  static constexpr int B4 = W4 + kMlpH * kMlpN4;               // [64]
  static constexpr int N = B4 + kMlpN4;
};

// GEMM C[M x N] = A[M x K] * B[N x K]^T on the tensor cores (both operands
// BF16, K-major, row-major in global memory), FP32 accumulation, with a
// fused epilogue.  v = acc + bias[n] (bias may be null), then
//   act 0: a = v;  out_f32 = v
//   act 1: a = silu(v);  out_f32 = v (pre-activation)
//   act 2: a = v * silu'(aux[m][n]);  out_f32 = a
// out_bf = bf16(a) row-major, out_bt = bf16(a) transposed ([N][M]); any
// output may be null.  M % 128 == 0, N % 64 == 0 (N <= 256 per tile
// column), K % 64 == 0, leading dimensions multiples of 8 elements.
struct GemmArgs {
  int M, N, K;
  const float* bias;
  int act;
  const float* aux; int ldaux;
  float* out_f32; int ldf;
  bf16* out_bf; int ldb;
  bf16* out_bt; int ldt;
  int* err;
};
int gemm_bf16(const bf16* A, int lda, const bf16* B, int ldb, const GemmArgs& g, cudaStream_t st);

// Tensor map of a row-major [rows][cols] BF16 matrix (leading dimension ld)
// with boxes of box_rows x 64 and the 128-byte swizzle.
int encode_bf16_map(CUtensorMap* m, const bf16* base, int rows, int cols, int ld, int box_rows);

// SiLU of the network and its derivative through the logistic function
// sigma(x) = (1 + tanh(x/2)) / 2 on the hardware tanh (tanh.approx.f32,
// one special-function instruction, relative error about 2^-11): the
// activations are stored in BF16 (relative rounding 2^-9), so the
// approximation stays below the storage rounding, and training and
// inference use the same function.
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sigmoid_hw(float x) { return .5f + .5f * tanh_hw(.5f * x); }
__device__ __forceinline__ float silu(float v) { return v * sigmoid_hw(v); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = sigmoid_hw(z);
  return s * (1.f + z * (1.f - s));
}

}  // namespace cress

// Learned microphysics: the MLP object behind the opaque cress_mlp handle
// (internal).
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "mlp.cuh"

namespace cress {

// Normalisation block (floats): input means and scales, target means and
// scales, and the training envelope (per-input minimum and maximum of the
// transformed features).
constexpr int kNormXmean = 0, kNormXstd = kMlpIn, kNormYmean = 2 * kMlpIn, kNormYstd = 2 * kMlpIn + kMlpOut;
constexpr int kNormXmin = 2 * kMlpIn + 2 * kMlpOut, kNormXmax = kNormXmin + kMlpIn;
constexpr int kNormN = kNormXmax + kMlpIn;

struct MlpWeights {
  bf16* w1t;   // [256][64]
  bf16* w2t;   // [256][256]  (N x K)
  bf16* w2;    // [256][256]  (K x N)
  bf16* w3t;
  bf16* w3;
  bf16* w4t;   // [64][256]
  bf16* w4;    // [256][64]
};

struct Mlp {
  int device = 0;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  std::vector<void*> owned, batch_owned;
  float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  int adam_step = 0;
  MlpWeights w{};
  float* norm_d = nullptr;
  std::vector<float> norm_h;
  int* err_d = nullptr;
  float* loss_d = nullptr;
  // batch buffers
  int cap = 0;
  bf16 *xb = nullptr, *xt = nullptr;
  float* z[3] = {nullptr, nullptr, nullptr};
  bf16* h[3] = {nullptr, nullptr, nullptr};
  bf16* ht[3] = {nullptr, nullptr, nullptr};
  float *y = nullptr, *t = nullptr, *dy = nullptr, *dz = nullptr;
  bf16 *dyb = nullptr, *dyt = nullptr, *dzb = nullptr, *dzt = nullptr;
  int* idx_d = nullptr;
  // tuple store: transformed features [n][16] and raw tendencies [n][9]
  float *tx = nullptr, *ty = nullptr;
  long long ntup = 0, tcap = 0;

  int init(int dev, unsigned long long seed);
  int upload_norm();
  int refresh_bf16();
  int ensure_batch(int B);
  int forward(int B);
  int backward(int B);
  int train_batch(int B, const int* idx_host_or_null, float lr, float* loss_out);
  int check_error();
  ~Mlp();
};

}  // namespace cress

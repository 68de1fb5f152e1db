// Learned cold-rain microphysics: the MLP object, its hand-written training
// (forward, backward, Adam) on the tensor-core GEMM of mlp_gemm.cu, and
// the C-ABI entry points cress_mlp_*.
//
// Training step on a batch of B tuples (B % 128 == 0):
//   forward   Z_l = H_{l-1} W_l^T + b_l, H_l = silu(Z_l) (bf16), l = 1..3;
//             Y = H_3 W_4 + b_4 (fp32)
//   loss      L = mean over the batch and the 9 outputs of (Y - T)^2
//   backward  dY = 2 (Y - T) / (9 B); dW_4 = H_3^T dY; dH_3 = dY W_4^T;
//             dZ_l = dH_l * silu'(Z_l); dW_l^T = dZ_l^T H_{l-1};
//             dH_{l-1} = dZ_l W_l; db_l = column sums of dZ_l
//   Adam      (beta1 0.9, beta2 0.999, eps 1e-8) on the FP32 masters,
//             then the BF16 copies are refreshed.
// Every GEMM runs on gemm_bf16 (tcgen05); the epilogues write the
// activations both row-major and transposed so that the weight-gradient
// GEMMs read K-major operands.
#include <cuda_runtime.h>
#include <cmath>
#include <cstring>
#include <vector>
#include "../../include/cress_b200.h"
#include "mlp.cuh"
#include "mlp_impl.cuh"

namespace cress {

int set_error(int code, const char* fmt, ...);
int cuda_check(cudaError_t e, const char* what);

namespace {

// Counter-based uniform in [-1, 1) (splitmix64 finaliser of seed ^ index).
__host__ __device__ inline float hash_uniform(unsigned long long seed, unsigned long long i) {
  unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (float)((z >> 40) * (1.0 / 16777216.0)) * 2.f - 1.f;
}

__global__ void k_init_params(float* p, unsigned long long seed) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= MlpLayout::N) return;
  float v = 0.f;
  auto uni = [&](float fan_in) { return hash_uniform(seed, n) * sqrtf(3.f / fan_in); };
  if (n < MlpLayout::B1) {
    const int k = (n - MlpLayout::W1) % kMlpK1;
    v = k < kMlpIn ? uni((float)kMlpIn) : 0.f;
  } else if (n >= MlpLayout::W2 && n < MlpLayout::B2) {
    v = uni((float)kMlpH);
  } else if (n >= MlpLayout::W3 && n < MlpLayout::B3) {
    v = uni((float)kMlpH);
  } else if (n >= MlpLayout::W4 && n < MlpLayout::B4) {
    const int c = (n - MlpLayout::W4) % kMlpN4;
    v = c < kMlpOut ? uni((float)kMlpH) : 0.f;
  }
  p[n] = v;
}

// BF16 copies: W1t [256][64], W2t/W2 and W3t/W3 [256][256], W4t [64][256]
// and W4 [256][64] from the masters (layers 1-3 stored [N][K], layer 4 [K][N]).
__global__ void k_cast_params(const float* p, MlpWeights w) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < kMlpH * kMlpK1) w.w1t[n] = __float2bfloat16_rn(p[MlpLayout::W1 + n]);
  if (n < kMlpH * kMlpH) {
    const int r = n / kMlpH, c = n % kMlpH;
    w.w2t[n] = __float2bfloat16_rn(p[MlpLayout::W2 + n]);
    w.w2[c * kMlpH + r] = __float2bfloat16_rn(p[MlpLayout::W2 + n]);
    w.w3t[n] = __float2bfloat16_rn(p[MlpLayout::W3 + n]);
    w.w3[c * kMlpH + r] = __float2bfloat16_rn(p[MlpLayout::W3 + n]);
  }
  if (n < kMlpH * kMlpN4) {
    const int r = n / kMlpN4, c = n % kMlpN4;   // master [K=256][N=64]
    w.w4[n] = __float2bfloat16_rn(p[MlpLayout::W4 + n]);
    w.w4t[c * kMlpH + r] = __float2bfloat16_rn(p[MlpLayout::W4 + n]);
  }
}

// Batch assembly: standardized inputs (bf16, row-major padded to 64 and
// transposed) and targets from the tuple store through an index list.
__global__ void k_gather_batch(const float* tx, const float* ty, const int* idx, int B, const float* norm,
                               bf16* xb, bf16* xt, float* t) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const long long s = idx ? idx[b] : b;
  for (int c = 0; c < kMlpK1; ++c) {
    float v = 0.f;
    if (c < kMlpIn) v = (tx[s * kMlpIn + c] - norm[c]) / norm[kMlpIn + c];
    const bf16 h = __float2bfloat16_rn(v);
    xb[(size_t)b * kMlpK1 + c] = h;
    xt[(size_t)c * B + b] = h;
  }
  if (t)
    for (int c = 0; c < kMlpOut; ++c)
      t[(size_t)b * kMlpOut + c] =
          (ty[s * kMlpOut + c] - norm[2 * kMlpIn + c]) / norm[2 * kMlpIn + kMlpOut + c];
}

// dY = 2 (Y - T) / (9 B) on the 9 outputs (0 on the padding), as fp32,
// bf16 row-major and bf16 transposed; the loss sum goes to *loss.
__global__ void k_loss_grad(const float* y, const float* t, int B, float* dy, bf16* dyb, bf16* dyt,
                            float* loss) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (b < B) {
    const float sc = 2.f / (kMlpOut * (float)B);
    for (int c = 0; c < kMlpN4; ++c) {
      float g = 0.f;
      if (c < kMlpOut) {
        const float d = y[(size_t)b * kMlpN4 + c] - t[(size_t)b * kMlpOut + c];
        l += d * d;
        g = sc * d;
      }
      dy[(size_t)b * kMlpN4 + c] = g;
      const bf16 h = __float2bfloat16_rn(g);
      dyb[(size_t)b * kMlpN4 + c] = h;
      dyt[(size_t)c * B + b] = h;
    }
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l / (kMlpOut * (float)B));
}

// db[c] += sum over rows of g[r][c] (g is B x N fp32).
__global__ void k_colsum(const float* g, int B, int N, float* db) {
  const int c = blockIdx.x * 32 + threadIdx.x;
  const int r0 = blockIdx.y * 256;
  float s = 0.f;
  if (c < N)
    for (int r = r0 + threadIdx.y; r < min(B, r0 + 256); r += blockDim.y) s += g[(size_t)r * N + c];
  __shared__ float red[8][33];
  red[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && c < N) {
    for (int y = 1; y < blockDim.y; ++y) s += red[y][threadIdx.x];
    atomicAdd(db + c, s);
  }
}

__global__ void k_adam(float* p, const float* g, float* m, float* v, float lr, float c1, float c2) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= MlpLayout::N) return;
  const float gr = g[n];
  const float mm = 0.9f * m[n] + 0.1f * gr;
  const float vv = 0.999f * v[n] + 0.001f * gr * gr;
  m[n] = mm;
  v[n] = vv;
  p[n] -= lr * (mm / c1) / (sqrtf(vv / c2) + 1e-8f);
}

template <class T>
T* dalloc(std::vector<void*>& owned, size_t n) {
  void* p = nullptr;
  if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
  owned.push_back(p);
  return static_cast<T*>(p);
}

}  // namespace

// ------------------------------------------------------------------ Mlp
Mlp::~Mlp() {
  cudaSetDevice(device);
  for (void* p : owned) cudaFree(p);
  for (void* p : batch_owned) cudaFree(p);
  if (tx) cudaFree(tx);
  if (ty) cudaFree(ty);
  if (own_stream) cudaStreamDestroy(own_stream);
}

int Mlp::init(int dev, unsigned long long seed) {
  device = dev;
  int rc = cuda_check(cudaSetDevice(dev), "cudaSetDevice");
  if (rc) return rc;
  if ((rc = cuda_check(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking), "stream"))) return rc;
  stream = own_stream;
  params = dalloc<float>(owned, MlpLayout::N);
  grads = dalloc<float>(owned, MlpLayout::N);
  adam_m = dalloc<float>(owned, MlpLayout::N);
  adam_v = dalloc<float>(owned, MlpLayout::N);
  norm_d = dalloc<float>(owned, kNormN);
  err_d = dalloc<int>(owned, 1);
  loss_d = dalloc<float>(owned, 1);
  w.w1t = dalloc<bf16>(owned, kMlpH * kMlpK1);
  w.w2t = dalloc<bf16>(owned, kMlpH * kMlpH);
  w.w2 = dalloc<bf16>(owned, kMlpH * kMlpH);
  w.w3t = dalloc<bf16>(owned, kMlpH * kMlpH);
  w.w3 = dalloc<bf16>(owned, kMlpH * kMlpH);
  w.w4t = dalloc<bf16>(owned, kMlpN4 * kMlpH);
  w.w4 = dalloc<bf16>(owned, kMlpH * kMlpN4);
  if (!params || !grads || !adam_m || !adam_v || !norm_d || !err_d || !loss_d || !w.w1t || !w.w2t || !w.w2 ||
      !w.w3t || !w.w3 || !w.w4t || !w.w4)
    return set_error(CRESS_E_CUDA, "cudaMalloc of the MLP failed");
  k_init_params<<<(MlpLayout::N + 255) / 256, 256, 0, stream>>>(params, seed);
  cudaMemsetAsync(adam_m, 0, sizeof(float) * MlpLayout::N, stream);
  cudaMemsetAsync(adam_v, 0, sizeof(float) * MlpLayout::N, stream);
  cudaMemsetAsync(err_d, 0, sizeof(int), stream);
  // identity normalisation until set_norm / training computes one
  norm_h.assign(kNormN, 0.f);
  for (int c = 0; c < kMlpIn; ++c) norm_h[kMlpIn + c] = 1.f;
  for (int c = 0; c < kMlpOut; ++c) norm_h[2 * kMlpIn + kMlpOut + c] = 1.f;
  for (int c = 0; c < kMlpIn; ++c) { norm_h[kNormXmin + c] = -3.0e38f; norm_h[kNormXmax + c] = 3.0e38f; }
  if ((rc = upload_norm())) return rc;
  return refresh_bf16();
}

int Mlp::upload_norm() {
  return cuda_check(cudaMemcpyAsync(norm_d, norm_h.data(), sizeof(float) * kNormN, cudaMemcpyHostToDevice, stream),
                    "norm copy");
}

int Mlp::refresh_bf16() {
  k_cast_params<<<(kMlpH * kMlpH + 255) / 256, 256, 0, stream>>>(params, w);
  return cuda_check(cudaGetLastError(), "cast params");
}

int Mlp::ensure_batch(int B) {
  if (B <= cap) return CRESS_OK;
  for (void* p : batch_owned) cudaFree(p);
  batch_owned.clear();
  cap = 0;
  auto& o = batch_owned;
  xb = dalloc<bf16>(o, (size_t)B * kMlpK1);
  xt = dalloc<bf16>(o, (size_t)B * kMlpK1);
  for (int l = 0; l < 3; ++l) {
    z[l] = dalloc<float>(o, (size_t)B * kMlpH);
    h[l] = dalloc<bf16>(o, (size_t)B * kMlpH);
    ht[l] = dalloc<bf16>(o, (size_t)B * kMlpH);
  }
  y = dalloc<float>(o, (size_t)B * kMlpN4);
  t = dalloc<float>(o, (size_t)B * kMlpOut);
  dy = dalloc<float>(o, (size_t)B * kMlpN4);
  dyb = dalloc<bf16>(o, (size_t)B * kMlpN4);
  dyt = dalloc<bf16>(o, (size_t)B * kMlpN4);
  dz = dalloc<float>(o, (size_t)B * kMlpH);
  dzb = dalloc<bf16>(o, (size_t)B * kMlpH);
  dzt = dalloc<bf16>(o, (size_t)B * kMlpH);
  idx_d = dalloc<int>(o, (size_t)B);
  if (!xb || !xt || !z[2] || !h[2] || !ht[2] || !y || !t || !dy || !dyb || !dyt || !dz || !dzb || !dzt || !idx_d)
    return set_error(CRESS_E_CUDA, "cudaMalloc of the MLP batch buffers failed");
  cap = B;
  return CRESS_OK;
}

// Forward pass on the assembled batch (xb, xt): z, h, ht, y.
int Mlp::forward(int B) {
  int rc;
  const bf16* in = xb;
  int kin = kMlpK1;
  const bf16* wt[3] = {w.w1t, w.w2t, w.w3t};
  const int boff[3] = {MlpLayout::B1, MlpLayout::B2, MlpLayout::B3};
  for (int l = 0; l < 3; ++l) {
    GemmArgs g{};
    g.M = B; g.N = kMlpH; g.K = kin;
    g.bias = params + boff[l];
    g.act = 1;
    g.out_f32 = z[l]; g.ldf = kMlpH;
    g.out_bf = h[l]; g.ldb = kMlpH;
    g.out_bt = ht[l]; g.ldt = B;
    g.err = err_d;
    if ((rc = gemm_bf16(in, kin, wt[l], kin, g, stream))) return rc;
    in = h[l];
    kin = kMlpH;
  }
  GemmArgs g{};
  g.M = B; g.N = kMlpN4; g.K = kMlpH;
  g.bias = params + MlpLayout::B4;
  g.act = 0;
  g.out_f32 = y; g.ldf = kMlpN4;
  g.err = err_d;
  return gemm_bf16(h[2], kMlpH, w.w4t, kMlpH, g, stream);
}

// Backward pass after forward(B) and k_loss_grad: gradients into `grads`.
int Mlp::backward(int B) {
  int rc;
  cudaMemsetAsync(grads, 0, sizeof(float) * MlpLayout::N, stream);
  // layer 4: dW4 [256][64] = H3^T dY  (A = H3^T [256][B], B operand = dY^T [64][B])
  {
    GemmArgs g{};
    g.M = kMlpH; g.N = kMlpN4; g.K = B;
    g.out_f32 = grads + MlpLayout::W4; g.ldf = kMlpN4;
    g.err = err_d;
    if ((rc = gemm_bf16(ht[2], B, dyt, B, g, stream))) return rc;
    k_colsum<<<dim3((kMlpN4 + 31) / 32, (B + 255) / 256), dim3(32, 8), 0, stream>>>(dy, B, kMlpN4,
                                                                                     grads + MlpLayout::B4);
  }
  // dH3 = dY W4^T (B operand = W4 [256][64]); dZ3 = dH3 * silu'(Z3)
  const bf16* wn[3] = {nullptr, w.w2, w.w3};
  const int woff[3] = {MlpLayout::W1, MlpLayout::W2, MlpLayout::W3};
  const int boff[3] = {MlpLayout::B1, MlpLayout::B2, MlpLayout::B3};
  {
    GemmArgs g{};
    g.M = B; g.N = kMlpH; g.K = kMlpN4;
    g.act = 2; g.aux = z[2]; g.ldaux = kMlpH;
    g.out_f32 = dz; g.ldf = kMlpH;
    g.out_bf = dzb; g.ldb = kMlpH;
    g.out_bt = dzt; g.ldt = B;
    g.err = err_d;
    if ((rc = gemm_bf16(dyb, kMlpN4, w.w4, kMlpN4, g, stream))) return rc;
  }
  for (int l = 2; l >= 0; --l) {
    // dW_l^T [256][K_l] = dZ_l^T H_{l-1}  (A = dZ_l^T [256][B], B operand = H_{l-1}^T [K_l][B])
    const int kl = l == 0 ? kMlpK1 : kMlpH;
    {
      GemmArgs g{};
      g.M = kMlpH; g.N = kl; g.K = B;
      g.out_f32 = grads + woff[l]; g.ldf = kl;
      g.err = err_d;
      if ((rc = gemm_bf16(dzt, B, l == 0 ? xt : ht[l - 1], B, g, stream))) return rc;
    }
    k_colsum<<<dim3(kMlpH / 32, (B + 255) / 256), dim3(32, 8), 0, stream>>>(dz, B, kMlpH, grads + boff[l]);
    if (l == 0) break;
    // dH_{l-1} = dZ_l W_l (B operand = W_l as [K][N] = wn[l]); dZ_{l-1} = dH * silu'(Z_{l-1})
    GemmArgs g{};
    g.M = B; g.N = kMlpH; g.K = kMlpH;
    g.act = 2; g.aux = z[l - 1]; g.ldaux = kMlpH;
    g.out_f32 = dz; g.ldf = kMlpH;
    g.out_bf = dzb; g.ldb = kMlpH;
    g.out_bt = dzt; g.ldt = B;
    g.err = err_d;
    // In place on dzb: N = 256 is one tile column, so each CTA reads only
    // its own 128 rows of dzb, all of them before its epilogue writes them;
    // dz and dzt were consumed by the launches above (same stream).
    if ((rc = gemm_bf16(dzb, kMlpH, wn[l], kMlpH, g, stream))) return rc;
  }
  return CRESS_OK;
}

int Mlp::check_error() {
  int e = 0;
  int rc = cuda_check(cudaMemcpyAsync(&e, err_d, sizeof(int), cudaMemcpyDeviceToHost, stream), "err copy");
  if (rc) return rc;
  if ((rc = cuda_check(cudaStreamSynchronize(stream), "mlp sync"))) return rc;
  if (e) {
    cudaMemsetAsync(err_d, 0, sizeof(int), stream);
    return set_error(e, "MLP kernel reported error %d (bounded wait expired)", e);
  }
  return CRESS_OK;
}

int Mlp::train_batch(int B, const int* idx_host_or_null, float lr, float* loss_out) {
  int rc;
  if ((rc = ensure_batch(B))) return rc;
  const int* idx = nullptr;
  if (idx_host_or_null) {
    if ((rc = cuda_check(cudaMemcpyAsync(idx_d, idx_host_or_null, sizeof(int) * B, cudaMemcpyHostToDevice, stream),
                         "idx copy")))
      return rc;
    idx = idx_d;
  }
  k_gather_batch<<<(B + 127) / 128, 128, 0, stream>>>(tx, ty, idx, B, norm_d, xb, xt, t);
  if ((rc = forward(B))) return rc;
  cudaMemsetAsync(loss_d, 0, sizeof(float), stream);
  k_loss_grad<<<(B + 127) / 128, 128, 0, stream>>>(y, t, B, dy, dyb, dyt, loss_d);
  if ((rc = backward(B))) return rc;
  ++adam_step;
  const float c1 = 1.f - powf(0.9f, (float)adam_step), c2 = 1.f - powf(0.999f, (float)adam_step);
  k_adam<<<(MlpLayout::N + 255) / 256, 256, 0, stream>>>(params, grads, adam_m, adam_v, lr, c1, c2);
  if ((rc = refresh_bf16())) return rc;
  if (loss_out)
    return cuda_check(cudaMemcpyAsync(loss_out, loss_d, sizeof(float), cudaMemcpyDeviceToHost, stream), "loss copy");
  return CRESS_OK;
}

}  // namespace cress

// ------------------------------------------------------------------ C-ABI
namespace cress {
namespace {

__global__ void k_pack_x(const float* x, int n, int B, bf16* xb, bf16* xt) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  for (int c = 0; c < kMlpK1; ++c) {
    const float v = (b < n && c < kMlpIn) ? x[(size_t)b * kMlpIn + c] : 0.f;
    const bf16 h = __float2bfloat16_rn(v);
    xb[(size_t)b * kMlpK1 + c] = h;
    xt[(size_t)c * B + b] = h;
  }
}

// Per-column statistics of an [n][C] array: sum, sum of squares (double),
// minimum and maximum (order-preserving integer images of the floats).
__device__ __forceinline__ int ord(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float unord(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }

__global__ void k_col_stats(const float* a, long long n, int C, double* sum, double* sq, int* mn, int* mx) {
  const int c = threadIdx.y;
  if (c >= C) return;
  double s = 0, q = 0;
  int lo = 0x7FFFFFFF, hi = (int)0x80000000;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
    const float v = a[r * C + c];
    s += v;
    q += (double)v * v;
    lo = min(lo, ord(v));
    hi = max(hi, ord(v));
  }
  atomicAdd(sum + c, s);
  atomicAdd(sq + c, q);
  atomicMin(mn + c, lo);
  atomicMax(mx + c, hi);
}

__global__ void k_unord(int* v, int n) {
  const int i = threadIdx.x;
  if (i < n) v[i] = __float_as_int(unord(v[i]));
}

}  // namespace
}  // namespace cress

using cress::Mlp;
using cress::MlpLayout;

extern "C" {

int cress_mlp_param_count(void) { return MlpLayout::N; }

int cress_mlp_create(int device, unsigned long long seed, cress_mlp** out) {
  if (!out) return cress::set_error(CRESS_E_ARG, "cress_mlp_create: null output");
  *out = nullptr;
  Mlp* m = new Mlp();
  int rc = m->init(device, seed);
  if (rc) {
    delete m;
    return rc;
  }
  if ((rc = cress::cuda_check(cudaStreamSynchronize(m->stream), "mlp init"))) {
    delete m;
    return rc;
  }
  *out = reinterpret_cast<cress_mlp*>(m);
  return CRESS_OK;
}

void cress_mlp_destroy(cress_mlp* h) { delete reinterpret_cast<Mlp*>(h); }

int cress_mlp_get_params(cress_mlp* h, float* host) {
  Mlp* m = reinterpret_cast<Mlp*>(h);
  if (!m || !host) return cress::set_error(CRESS_E_ARG, "cress_mlp_get_params: null argument");
  cudaSetDevice(m->device);
  int rc = cress::cuda_check(cudaMemcpyAsync(host, m->params, sizeof(float) * MlpLayout::N, cudaMemcpyDeviceToHost,
                                             m->stream), "params copy");
  return rc ? rc : cress::cuda_check(cudaStreamSynchronize(m->stream), "params sync");
}

int cress_mlp_set_params(cress_mlp* h, const float* host) {
  Mlp* m = reinterpret_cast<Mlp*>(h);
  if (!m || !host) return cress::set_error(CRESS_E_ARG, "cress_mlp_set_params: null argument");
  cudaSetDevice(m->device);
  int rc = cress::cuda_check(cudaMemcpyAsync(m->params, host, sizeof(float) * MlpLayout::N, cudaMemcpyHostToDevice,
                                             m->stream), "params copy");
  if (rc || (rc = m->refresh_bf16())) return rc;
  return cress::cuda_check(cudaStreamSynchronize(m->stream), "params sync");
}

int cress_mlp_get_norm(cress_mlp* h, float* host) {
  Mlp* m = reinterpret_cast<Mlp*>(h);
  if (!m || !host) return cress::set_error(CRESS_E_ARG, "cress_mlp_get_norm: null argument");
  std::memcpy(host, m->norm_h.data(), sizeof(float) * cress::kNormN);
  return CRESS_OK;
}

int cress_mlp_set_norm(cress_mlp* h, const float* host) {
  Mlp* m = reinterpret_cast<Mlp*>(h);
  if (!m || !host) return cress::set_error(CRESS_E_ARG, "cress_mlp_set_norm: null argument");
  for (int c = 0; c < cress::kMlpIn; ++c)
    if (!(host[cress::kNormXstd + c] > 0.f)) return cress::set_error(CRESS_E_ARG, "input scale %d not positive", c);
  for (int c = 0; c < cress::kMlpOut; ++c)
    if (!(host[cress::kNormYstd + c] > 0.f)) return cress::set_error(CRESS_E_ARG, "target scale %d not positive", c);
  cudaSetDevice(m->device);
  m->norm_h.assign(host, host + cress::kNormN);
  int rc = m->upload_norm();
  return rc ? rc : cress::cuda_check(cudaStreamSynchronize(m->stream), "norm sync");
}

// Network function on host arrays: x [n][16] standardized inputs ->
// y [n][9] standardized outputs.
int cress_mlp_forward(cress_mlp* h, int n, const float* x, float* y) {
  Mlp* m = reinterpret_cast<Mlp*>(h);
  if (!m || !x || !y || n <= 0) return cress::set_error(CRESS_E_ARG, "cress_mlp_forward: bad argument");
  cudaSetDevice(m->device);
  const int B = (n + 127) / 128 * 128;
  int rc = m->ensure_batch(B);
  if (rc) return rc;
  float* xd = nullptr;
  if ((rc = cress::cuda_check(cudaMallocAsync(&xd, sizeof(float) * n * cress::kMlpIn, m->stream), "x alloc")))
    return rc;
  cudaMemcpyAsync(xd, x, sizeof(float) * n * cress::kMlpIn, cudaMemcpyHostToDevice, m->stream);
  cress::k_pack_x<<<(B + 127) / 128, 128, 0, m->stream>>>(xd, n, B, m->xb, m->xt);
  rc = m->forward(B);
  cudaFreeAsync(xd, m->stream);
  if (rc) return rc;
  if ((rc = cress::cuda_check(cudaMemcpy2DAsync(y, sizeof(float) * cress::kMlpOut, m->y, sizeof(float) * cress::kMlpN4,
                                                sizeof(float) * cress::kMlpOut, n, cudaMemcpyDeviceToHost, m->stream),
                              "y copy")))
    return rc;
  return m->check_error();
}

// Loss and parameter gradient (layout of cress_mlp_get_params) of one
// batch: x [n][16] standardized inputs, t [n][9] standardized targets, n a
// multiple of 128.
int cress_mlp_loss_grad(cress_mlp* h, int n, const float* x, const float* t, float* loss, float* grad) {
  Mlp* m = reinterpret_cast<Mlp*>(h);
  if (!m || !x || !t || !loss || !grad || n <= 0 || n % 128)
    return cress::set_error(CRESS_E_ARG, "cress_mlp_loss_grad: bad argument (n %% 128 == 0)");
  cudaSetDevice(m->device);
  int rc = m->ensure_batch(n);
  if (rc) return rc;
  float* xd = nullptr;
  if ((rc = cress::cuda_check(cudaMallocAsync(&xd, sizeof(float) * n * cress::kMlpIn, m->stream), "x alloc")))
    return rc;
  cudaMemcpyAsync(xd, x, sizeof(float) * n * cress::kMlpIn, cudaMemcpyHostToDevice, m->stream);
  cudaMemcpyAsync(m->t, t, sizeof(float) * n * cress::kMlpOut, cudaMemcpyHostToDevice, m->stream);
  cress::k_pack_x<<<(n + 127) / 128, 128, 0, m->stream>>>(xd, n, n, m->xb, m->xt);
  rc = m->forward(n);
  cudaFreeAsync(xd, m->stream);
  if (rc) return rc;
  cudaMemsetAsync(m->loss_d, 0, sizeof(float), m->stream);
  cress::k_loss_grad<<<(n + 127) / 128, 128, 0, m->stream>>>(m->y, m->t, n, m->dy, m->dyb, m->dyt, m->loss_d);
  if ((rc = m->backward(n))) return rc;
  cudaMemcpyAsync(loss, m->loss_d, sizeof(float), cudaMemcpyDeviceToHost, m->stream);
  cudaMemcpyAsync(grad, m->grads, sizeof(float) * MlpLayout::N, cudaMemcpyDeviceToHost, m->stream);
  return m->check_error();
}

int cress_mlp_reserve(cress_mlp* h, long long cap) {
  Mlp* m = reinterpret_cast<Mlp*>(h);
  if (!m || cap < 0) return cress::set_error(CRESS_E_ARG, "cress_mlp_reserve: bad argument");
  if (cap <= m->tcap) return CRESS_OK;
  cudaSetDevice(m->device);
  float *tx = nullptr, *ty = nullptr;
  if (cudaMalloc(&tx, sizeof(float) * cap * cress::kMlpIn) != cudaSuccess ||
      cudaMalloc(&ty, sizeof(float) * cap * cress::kMlpOut) != cudaSuccess) {
    cudaFree(tx);
    return cress::set_error(CRESS_E_CUDA, "cudaMalloc of %lld tuples failed", cap);
  }
  if (m->ntup) {
    cudaMemcpyAsync(tx, m->tx, sizeof(float) * m->ntup * cress::kMlpIn, cudaMemcpyDeviceToDevice, m->stream);
    cudaMemcpyAsync(ty, m->ty, sizeof(float) * m->ntup * cress::kMlpOut, cudaMemcpyDeviceToDevice, m->stream);
  }
  cudaStreamSynchronize(m->stream);
  cudaFree(m->tx);
  cudaFree(m->ty);
  m->tx = tx;
  m->ty = ty;
  m->tcap = cap;
  return CRESS_OK;
}

// Append tuples from the host: x [n][16] transformed (unstandardized)
// features, t [n][9] transformed targets.
int cress_mlp_add_tuples(cress_mlp* h, long long n, const float* x, const float* t) {
  Mlp* m = reinterpret_cast<Mlp*>(h);
  if (!m || !x || !t || n < 0) return cress::set_error(CRESS_E_ARG, "cress_mlp_add_tuples: bad argument");
  int rc = cress_mlp_reserve(h, m->ntup + n);
  if (rc) return rc;
  cudaMemcpyAsync(m->tx + m->ntup * cress::kMlpIn, x, sizeof(float) * n * cress::kMlpIn, cudaMemcpyHostToDevice,
                  m->stream);
  cudaMemcpyAsync(m->ty + m->ntup * cress::kMlpOut, t, sizeof(float) * n * cress::kMlpOut, cudaMemcpyHostToDevice,
                  m->stream);
  m->ntup += n;
  return cress::cuda_check(cudaStreamSynchronize(m->stream), "tuple copy");
}

int cress_mlp_get_tuples(cress_mlp* h, long long first, long long n, float* x, float* t) {
  Mlp* m = reinterpret_cast<Mlp*>(h);
  if (!m || !x || !t || first < 0 || n < 0 || first + n > m->ntup)
    return cress::set_error(CRESS_E_ARG, "cress_mlp_get_tuples: bad range");
  cudaMemcpyAsync(x, m->tx + first * cress::kMlpIn, sizeof(float) * n * cress::kMlpIn, cudaMemcpyDeviceToHost,
                  m->stream);
  cudaMemcpyAsync(t, m->ty + first * cress::kMlpOut, sizeof(float) * n * cress::kMlpOut, cudaMemcpyDeviceToHost,
                  m->stream);
  return cress::cuda_check(cudaStreamSynchronize(m->stream), "tuple copy");
}

long long cress_mlp_tuple_count(const cress_mlp* h) {
  const Mlp* m = reinterpret_cast<const Mlp*>(h);
  return m ? m->ntup : -1;
}

// Normalisation and envelope from the stored tuples (means, standard
// deviations floored at 1e-6, per-input minimum and maximum).
int cress_mlp_fit_norm(cress_mlp* h) {
  Mlp* m = reinterpret_cast<Mlp*>(h);
  if (!m || m->ntup < 2) return cress::set_error(CRESS_E_STATE, "cress_mlp_fit_norm: fewer than 2 tuples");
  cudaSetDevice(m->device);
  double* acc = nullptr;
  int* mm = nullptr;
  const int C[2] = {cress::kMlpIn, cress::kMlpOut};
  if (cudaMallocAsync(&acc, sizeof(double) * 4 * 16, m->stream) != cudaSuccess ||
      cudaMallocAsync(&mm, sizeof(int) * 4 * 16, m->stream) != cudaSuccess)
    return cress::set_error(CRESS_E_CUDA, "stats alloc");
  cudaMemsetAsync(acc, 0, sizeof(double) * 64, m->stream);
  std::vector<int> init(64);
  for (int i = 0; i < 64; ++i) init[i] = (i % 32) < 16 ? 0x7FFFFFFF : (int)0x80000000;
  cudaMemcpyAsync(mm, init.data(), sizeof(int) * 64, cudaMemcpyHostToDevice, m->stream);
  const float* src[2] = {m->tx, m->ty};
  for (int s = 0; s < 2; ++s)
    cress::k_col_stats<<<592, dim3(8, C[s]), 0, m->stream>>>(src[s], m->ntup, C[s], acc + 32 * s, acc + 32 * s + 16,
                                                             mm + 32 * s, mm + 32 * s + 16);
  cress::k_unord<<<1, 64, 0, m->stream>>>(mm, 64);
  std::vector<double> a(64);
  std::vector<float> b(64);
  cudaMemcpyAsync(a.data(), acc, sizeof(double) * 64, cudaMemcpyDeviceToHost, m->stream);
  cudaMemcpyAsync(b.data(), mm, sizeof(int) * 64, cudaMemcpyDeviceToHost, m->stream);
  int rc = cress::cuda_check(cudaStreamSynchronize(m->stream), "stats");
  cudaFreeAsync(acc, m->stream);
  cudaFreeAsync(mm, m->stream);
  if (rc) return rc;
  const double n = (double)m->ntup;
  std::vector<float> nm(cress::kNormN, 0.f);
  for (int s = 0; s < 2; ++s)
    for (int c = 0; c < C[s]; ++c) {
      const double mu = a[32 * s + c] / n;
      const double var = std::max(a[32 * s + 16 + c] / n - mu * mu, 0.0);
      const float sd = (float)std::max(std::sqrt(var), 1e-6);
      if (s == 0) {
        nm[cress::kNormXmean + c] = (float)mu;
        nm[cress::kNormXstd + c] = sd;
        nm[cress::kNormXmin + c] = b[c];
        nm[cress::kNormXmax + c] = b[16 + c];
      } else {
        nm[cress::kNormYmean + c] = (float)mu;
        nm[cress::kNormYstd + c] = sd;
      }
    }
  return cress_mlp_set_norm(h, nm.data());
}

// `steps` Adam steps on random batches of the stored tuples; losses[s]
// receives each step's training loss (standardized units).
int cress_mlp_train(cress_mlp* h, int steps, int batch, float lr, unsigned long long seed, float* losses) {
  Mlp* m = reinterpret_cast<Mlp*>(h);
  if (!m || steps < 0 || batch <= 0 || batch % 128 || !(lr > 0.f))
    return cress::set_error(CRESS_E_ARG, "cress_mlp_train: bad argument (batch %% 128 == 0)");
  if (m->ntup < batch) return cress::set_error(CRESS_E_STATE, "cress_mlp_train: %lld tuples < batch %d", m->ntup, batch);
  cudaSetDevice(m->device);
  std::vector<int> idx(batch);
  unsigned long long s = seed * 0x9E3779B97F4A7C15ull + 1;
  std::vector<float> lbuf(steps > 0 ? steps : 1);
  for (int it = 0; it < steps; ++it) {
    for (int b = 0; b < batch; ++b) {
      s ^= s << 13; s ^= s >> 7; s ^= s << 17;
      idx[b] = (int)(s % (unsigned long long)m->ntup);
    }
    int rc = m->train_batch(batch, idx.data(), lr, losses ? &lbuf[it] : nullptr);
    if (rc) return rc;
    if (it % 64 == 63 || it == steps - 1)
      if ((rc = m->check_error())) return rc;
  }
  if (losses) std::memcpy(losses, lbuf.data(), sizeof(float) * steps);
  return m->check_error();
}

}  // extern "C"

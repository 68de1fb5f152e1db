// Learned microphysics: per-cell kernels around the MLP (features, tuple
// collection from the plain scheme, tendency application with positivity,
// water conservation and fallback).  Included by micro.cu only (they share
// its Koenig tables and cell loaders).
//
// The MLP replaces the process-rate part of s_coldblk (adjstni, srcblk,
// adjstni: SrcOrig/coldblk.f90:327-425) for one cell: from the thermodynamic
// state and hydrometeors of the past level (and the condensate of the
// future level) it predicts the change of qv, qc, qr, qi, qs, qg, ni, ns,
// ng on the future level over 2*dtb.  Sedimentation (s_fallblk) stays the
// plain scheme.
//
// Inputs (16): T-273.16, ln p, rho, w, log10 of qv..qg (floor 1e-12),
// log10 of ni, ns, ng (floor 1), supersaturation over water and over ice
// (clipped to [-1, 1]), log10 of the future level's total condensate.
// Targets (9): y = sign(d) * log10(1 + |d|/s), s = 1e-9 kg/kg for the
// mixing ratios and 1 /kg for the numbers; inputs and targets are then
// standardized with the training set's means and scales.
#pragma once

namespace cress {
namespace {

constexpr float kTgtScaleQ = 1.e-9f, kTgtScaleN = 1.f;

__device__ __forceinline__ float tgt_scale(int c) { return c < 6 ? kTgtScaleQ : kTgtScaleN; }
__device__ __forceinline__ float tgt_fwd(float d, int c) {
  return copysignf(log10f(1.f + fabsf(d) / tgt_scale(c)), d);
}
__device__ __forceinline__ float tgt_inv(float y, int c) {
  return copysignf(tgt_scale(c) * (exp10f(fminf(fabsf(y), 30.f)) - 1.f), y);
}

// Interior cell n = ((k-1) * ny + (j-2)) * nx + (i-2), k = 1..nk-1.
__device__ __forceinline__ long long cell_index(const Grid& g, long long n, int& k) {
  const long long nx = g.ni - 3, ny = g.nj - 3;
  const long long i = n % nx, j = (n / nx) % ny;
  k = (int)(n / (nx * ny)) + 1;
  return g.at((int)i + 2, (int)j + 2, k);
}

__device__ inline void load_future(const MicroArgs& a, long long id, MCell& c) {
  c.ptpf = a.ptpf[id]; c.qvf = a.qvf[id]; c.qcf = a.qcf[id]; c.qrf = a.qrf[id];
  c.qif = a.qif[id]; c.qsf = a.qsf[id]; c.qgf = a.qgf[id]; c.ncif = a.nif[id];
  c.ncsf = a.nsf[id]; c.ncgf = a.ngf[id];
}

__device__ inline void mlp_features(const MCell& c, float wc, float (&f)[kMlpIn]) {
  const float t = (c.ptbr + c.ptpp) * c.pi;
  const float tcel = t - 273.16f;
  auto lq = [](float q) { return log10f(fmaxf(q, 1.e-12f)); };
  auto ln = [](float n) { return log10f(fmaxf(n, 1.f)); };
  f[0] = tcel;
  f[1] = logf(c.p);
  f[2] = c.rbr;
  f[3] = wc;
  f[4] = lq(c.qvp); f[5] = lq(c.qcp); f[6] = lq(c.qrp); f[7] = lq(c.qip); f[8] = lq(c.qsp); f[9] = lq(c.qgp);
  f[10] = ln(c.ncip); f[11] = ln(c.ncsp); f[12] = ln(c.ncgp);
  const float esw = 610.78f * expf(17.269f * tcel / (t - 35.86f));   // setblk.f90:333
  const float esi = 610.78f * expf(21.875f * tcel / (t - 7.66f));    // setblk.f90:334
  const float qvsw = .622f * esw / (c.p - esw), qvsi = .622f * esi / (c.p - esi);
  f[13] = fminf(fmaxf(c.qvp / qvsw - 1.f, -1.f), 1.f);
  f[14] = fminf(fmaxf(c.qvp / qvsi - 1.f, -1.f), 1.f);
  f[15] = lq(c.qcf + c.qrf + c.qif + c.qsf + c.qgf);
}

// The plain process-rate part on a copy of the cell; d = change of the nine
// future fields (qv..ng) and of theta'.
__device__ inline void plain_source(const MicroArgs& a, MCell c, float (&d)[kMlpOut], float& dpt) {
  const float b[kMlpOut] = {c.qvf, c.qcf, c.qrf, c.qif, c.qsf, c.qgf, c.ncif, c.ncsf, c.ncgf};
  const float pt0 = c.ptpf;
  adjstni_cell(c.rbr, c.rbv, c.qif, c.qsf, c.qgf, c.ncif, c.ncsf, c.ncgf);
  termblk_cell(a.thresq, c);
  srcblk_cell(a.dtb, a.thresq, c);
  adjstni_cell(c.rbr, c.rbv, c.qif, c.qsf, c.qgf, c.ncif, c.ncsf, c.ncgf);
  const float e[kMlpOut] = {c.qvf, c.qcf, c.qrf, c.qif, c.qsf, c.qgf, c.ncif, c.ncsf, c.ncgf};
#pragma unroll
  for (int n = 0; n < kMlpOut; ++n) d[n] = e[n] - b[n];
  dpt = c.ptpf - pt0;
}

__device__ __forceinline__ float w_center(const float* w, long long id, long long pl) {
  return .5f * (__ldg(w + id) + __ldg(w + id + pl));
}

// Tuple collection: every cell whose hash falls in the sample (1 in
// `stride`; cells without any tendency only 1 in stride/keep_zero) writes
// its transformed features and targets.
__global__ void __launch_bounds__(128) k_micro_tuples(const MicroArgs a, const float* w, float* tx, float* ty,
                                                       unsigned long long* count, long long cap, int stride,
                                                       float keep_zero, unsigned long long seed) {
  const Grid g = a.g;
  const long long ncell = (long long)(g.ni - 3) * (g.nj - 3) * (g.nk - 1);
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < ncell;
       n += (long long)gridDim.x * blockDim.x) {
    unsigned long long h = (unsigned long long)n * 0x9E3779B97F4A7C15ull + seed;
    h ^= h >> 29; h *= 0xBF58476D1CE4E5B9ull; h ^= h >> 32;
    if (h % (unsigned long long)stride) continue;
    int k;
    const long long id = cell_index(g, n, k);
    MCell c;
    load_cell(a, id, k, c);
    load_future(a, id, c);
    float f[kMlpIn], d[kMlpOut], dpt;
    mlp_features(c, w_center(w, id, g.plane), f);
    plain_source(a, c, d, dpt);
    bool any = false;
#pragma unroll
    for (int m = 0; m < kMlpOut; ++m) any |= d[m] != 0.f;
    if (!any && (float)((h >> 40) & 0xFFFF) >= keep_zero * 65536.f) continue;
    const unsigned long long slot = atomicAdd(count, 1ull);
    if ((long long)slot >= cap) continue;
#pragma unroll
    for (int m = 0; m < kMlpIn; ++m) tx[slot * kMlpIn + m] = f[m];
#pragma unroll
    for (int m = 0; m < kMlpOut; ++m) ty[slot * kMlpOut + m] = tgt_fwd(d[m], m);
  }
}

// Features of cells [n0, n0 + cnt): standardized bf16 rows (padded to 64
// columns), the envelope flag, and the sedimentation CFL minimum of the
// past level's fall speeds (as k_micro_src).
__global__ void __launch_bounds__(128) k_mlp_features(const MicroArgs a, const float* w, long long n0, int cnt,
                                                       int rows, const float* norm, bf16* xb,
                                                       unsigned char* out_env) {
  const Grid g = a.g;
  const long long ncell = (long long)(g.ni - 3) * (g.nj - 3) * (g.nk - 1);
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  float lim = 3.0e38f;
  if (r < rows) {
    float f[kMlpIn];
    bool inside = true;
    if (r < cnt && n0 + r < ncell) {
      int k;
      const long long id = cell_index(g, n0 + r, k);
      MCell c;
      load_cell(a, id, k, c);
      load_future(a, id, c);
      mlp_features(c, w_center(w, id, g.plane), f);
      termblk_cell(a.thresq, c);
      store_speeds(a, id, c);
      const float dzjcb = a.dz * __ldg(a.col + C_JCB * (g.nk + 1) + k);
      lim = fminf(lim, dzjcb / (c.ucq + 1.e-20f));
      lim = fminf(lim, dzjcb / (c.urq + 1.e-20f));
      lim = fminf(lim, dzjcb / (c.uiq + 1.e-20f));
      lim = fminf(lim, dzjcb / (c.usq + 1.e-20f));
      lim = fminf(lim, dzjcb / (c.ugq + 1.e-20f));
#pragma unroll
      for (int m = 0; m < kMlpIn; ++m) {
        const float lo = norm[kNormXmin + m], hi = norm[kNormXmax + m], mg = .05f * (hi - lo);
        inside &= f[m] >= lo - mg && f[m] <= hi + mg;
      }
    } else {
#pragma unroll
      for (int m = 0; m < kMlpIn; ++m) f[m] = norm[kNormXmean + m];
    }
    uint32_t wds[32];
#pragma unroll
    for (int m = 0; m < 32; ++m) {
      float v0 = 0.f, v1 = 0.f;
      if (2 * m < kMlpIn) v0 = (f[2 * m] - norm[kNormXmean + 2 * m]) / norm[kNormXstd + 2 * m];
      if (2 * m + 1 < kMlpIn) v1 = (f[2 * m + 1] - norm[kNormXmean + 2 * m + 1]) / norm[kNormXstd + 2 * m + 1];
      const __nv_bfloat162 hv = __floats2bfloat162_rn(v0, v1);
      wds[m] = *reinterpret_cast<const uint32_t*>(&hv);
    }
    uint4* dst = reinterpret_cast<uint4*>(xb + (size_t)r * kMlpK1);
#pragma unroll
    for (int q = 0; q < 8; ++q) dst[q] = make_uint4(wds[4 * q], wds[4 * q + 1], wds[4 * q + 2], wds[4 * q + 3]);
    out_env[r] = inside ? 1 : 0;
  }
  for (int o = 16; o > 0; o >>= 1) lim = fminf(lim, __shfl_xor_sync(0xffffffffu, lim, o));
  if ((threadIdx.x & 31) == 0 && lim < 3.0e38f) atomicMin(a.dtp_bits, __float_as_int(lim));
}

struct ApplyArgs {
  const float* y;          // [rows][64] network outputs (standardized)
  const unsigned char* env;
  const float* norm;
  long long n0;
  int cnt;
  float resid_tol;         // relative tolerance of the water-budget residual
  int* fb_list;            // fallback cells (interior cell indices)
  int* fb_count;
  int fb_cap;
  unsigned long long* stats;   // [0] cells done by the MLP, [1] fallbacks
};

// Apply the network's outputs ys (standardized) for interior cell n to the
// future level, with positivity and water conservation: hydrometeor losses
// are capped at what is present, vapour closes the water budget (the
// network's own vapour change must agree within resid_tol), gains shrink
// if vapour would go negative, theta' follows from the latent heats (lv,
// lf at the cell's temperature, as in srcblk) and adjstni keeps the
// numbers consistent.  Returns false (nothing written) when the cell must
// run the plain process rates instead.
__device__ inline bool mlp_apply_cell(const MicroArgs& a, long long n, const float* ys, bool ok, const float* norm,
                                      float resid_tol) {
  float d[kMlpOut];
#pragma unroll
  for (int m = 0; m < kMlpOut; ++m) {
    const float yv = ys[m] * norm[kNormYstd + m] + norm[kNormYmean + m];
    d[m] = tgt_inv(yv, m);
    ok &= isfinite(d[m]);
  }
  if (!ok) return false;
  int k;
  const long long id = cell_index(a.g, n, k);
  MCell c;
  load_cell(a, id, k, c);
  load_future(a, id, c);
  float q[6] = {c.qvf, c.qcf, c.qrf, c.qif, c.qsf, c.qgf};
  float gain = 0.f, loss = 0.f;
#pragma unroll
  for (int m = 1; m < 6; ++m) {
    d[m] = fmaxf(d[m], -q[m]);
    if (d[m] > 0.f) gain += d[m]; else loss -= d[m];
  }
  const float dqv_pred = d[0];
  if (q[0] + loss - gain < 0.f && gain > 0.f) {
    const float s = (q[0] + loss) / gain;
#pragma unroll
    for (int m = 1; m < 6; ++m)
      if (d[m] > 0.f) d[m] *= s;
    gain = q[0] + loss;
  }
  d[0] = loss - gain;
  const float scale = fabsf(dqv_pred) + gain + loss;
  if (fabsf(dqv_pred - d[0]) > resid_tol * scale + 1.e-10f) return false;
  const float t = (c.ptbr + c.ptpp) * c.pi;
  const float tcel = t - 273.16f;
  const float lv = 2.50078e6f * expf((.167f + 3.67e-4f * t) * logf(273.16f / t));   // as srcblk
  const float lf = 3.34e5f + (4.218e3f - 2.106e3f) * tcel;
  const float cppiv = 1.f / (1004.f * c.pi);
  a.ptpf[id] = c.ptpf + (lv * (-d[0]) + lf * (d[3] + d[4] + d[5])) * cppiv;
  a.qvf[id] = q[0] + d[0];
  a.qcf[id] = q[1] + d[1];
  a.qrf[id] = q[2] + d[2];
  const float qi = q[3] + d[3], qs = q[4] + d[4], qg = q[5] + d[5];
  float nci = fmaxf(c.ncif + d[6], 0.f), ncs = fmaxf(c.ncsf + d[7], 0.f), ncg = fmaxf(c.ncgf + d[8], 0.f);
  adjstni_cell(c.rbr, c.rbv, qi, qs, qg, nci, ncs, ncg);
  a.qif[id] = qi; a.qsf[id] = qs; a.qgf[id] = qg;
  a.nif[id] = nci; a.nsf[id] = ncs; a.ngf[id] = ncg;
  return true;
}

// Apply one chunk's network outputs; cells outside the envelope or failing
// the residual check go to the fallback list.
__global__ void __launch_bounds__(128) k_mlp_apply(const MicroArgs a, const ApplyArgs p) {
  const Grid g = a.g;
  const long long ncell = (long long)(g.ni - 3) * (g.nj - 3) * (g.nk - 1);
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = p.n0 + r;
  bool used = false, fb = false;
  if (r < p.cnt && n < ncell) {
    used = mlp_apply_cell(a, n, p.y + (size_t)r * kMlpN4, p.env[r] != 0, p.norm, p.resid_tol);
    fb = !used;
  }
  // one set of atomics per warp (counts, and the fallback cells' slots)
  const unsigned full = 0xffffffffu, lane = threadIdx.x & 31u;
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
    if (slot < p.fb_cap) p.fb_list[slot] = (int)(n - p.n0);   // relative to the chunk
  }
}

// The plain process-rate part on the listed cells of one chunk.
__global__ void __launch_bounds__(128) k_micro_src_list(const MicroArgs a, long long n0, const int* list,
                                                         const int* count, int cap) {
  const int cnt = min(*count, cap);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
    int k;
    const long long id = cell_index(a.g, n0 + list[t], k);
    MCell c;
    load_cell(a, id, k, c);
    load_future(a, id, c);
    adjstni_cell(c.rbr, c.rbv, c.qif, c.qsf, c.qgf, c.ncif, c.ncsf, c.ncgf);
    termblk_cell(a.thresq, c);
    srcblk_cell(a.dtb, a.thresq, c);
    adjstni_cell(c.rbr, c.rbv, c.qif, c.qsf, c.qgf, c.ncif, c.ncsf, c.ncgf);
    a.ptpf[id] = c.ptpf; a.qvf[id] = c.qvf; a.qcf[id] = c.qcf; a.qrf[id] = c.qrf;
    a.qif[id] = c.qif; a.qsf[id] = c.qsf; a.qgf[id] = c.qgf; a.nif[id] = c.ncif;
    a.nsf[id] = c.ncsf; a.ngf[id] = c.ncgf;
  }
}

}  // namespace
}  // namespace cress

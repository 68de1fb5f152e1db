// HE-VI substep entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc from inside their time loop: a host
// model whose device arrays all live in a pool it sized up front, or a
// framework whose caching allocator owns the device.  They already hold the
// old and new u, v, w, p' and the four forcings in their own buffers; what
// the substep additionally needs is small per-column data (1-D base-state
// columns, their reciprocals, the elimination factors of the w system and
// an error word).  Here that data lives in one file-scope __device__ array
// of fixed size, so the call allocates nothing; the kernel is the same
// k_hevi_substep the context API launches.
//
// Limits and sharing:
//   * nk <= kNoAllocMaxNk (256 levels); larger grids are rejected.
//   * The array is one per device and holds its contents between calls.
//     Each call rewrites all of it (the error word is cleared), so no state
//     carries over, but two calls whose kernels overlap on the GPU (e.g. on
//     different streams) race on it: serialize them.
//   * The first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture begins.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cmath>
#include <cstring>
#include <mutex>
#include "../../include/cress_b200.h"
#include "common.cuh"
#include "ctx.h"
#include "hevi.cuh"

namespace cress {
namespace {

constexpr int kNoAllocMaxNk = 256;
constexpr int kMaxDevices = 64;

struct NoAllocScratch {
  double aa[kNoAllocMaxNk + 2];                 // 1/(b_k - a_k c'_{k-1})
  double cp[kNoAllocMaxNk + 2];                 // c'_k
  float rr[kNoAllocMaxNk + 2];                  // a_k
  float col[C_NFIELDS * (kNoAllocMaxNk + 1)];   // 1-D base columns
  int err;                                      // bounded-wait failure flag
};

// The scratch: a fixed device array, resident on every GPU that loads the
// library until the process exits.
static __device__ __align__(256) unsigned char g_hevi_scratch[sizeof(NoAllocScratch)];

std::mutex g_mu;
void* g_scratch_dev[kMaxDevices];  // device address of g_hevi_scratch per device
bool g_ready[kMaxDevices];

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encoder() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

int encode(EncodeTiledFn fn, const Grid& g, const float* buf, int rows, CUtensorMap* m) {
  cuuint64_t dims[3] = {(cuuint64_t)g.px, (cuuint64_t)g.py, (cuuint64_t)g.nk};
  cuuint64_t strides[2] = {(cuuint64_t)g.px * 4, (cuuint64_t)g.plane * 4};
  cuuint32_t box[3] = {(cuuint32_t)kHeviBoxX, (cuuint32_t)rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(buf), dims, strides, box,
                  estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? CRESS_OK : set_error(CRESS_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
}

// Device address of the scratch on the current device (set up once).
int scratch_address(int dev, NoAllocScratch** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ready[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_hevi_scratch);
    if (e != cudaSuccess) return cuda_check(e, "cudaGetSymbolAddress(hevi scratch)");
    g_scratch_dev[dev] = p;
    g_ready[dev] = true;
  }
  *out = reinterpret_cast<NoAllocScratch*>(g_scratch_dev[dev]);
  return CRESS_OK;
}

}  // namespace
}  // namespace cress

using namespace cress;

extern "C" int cress_hevi_substep_noalloc(const cress_cfg* cfg, float dts,
                                          const float* const* base3d, const float* u_old,
                                          const float* v_old, const float* w_old,
                                          const float* p_old, const float* ufrc, const float* vfrc,
                                          const float* wfrc, const float* pfrc, float* u_new,
                                          float* v_new, float* w_new, float* p_new, void* stream) {
  if (!cfg || !base3d) return set_error(CRESS_E_ARG, "cress_hevi_substep_noalloc: null argument");
  const float* dev_in[8] = {u_old, v_old, w_old, p_old, ufrc, vfrc, wfrc, pfrc};
  float* dev_out[4] = {u_new, v_new, w_new, p_new};
  for (auto p : dev_in)
    if (!p || (reinterpret_cast<uintptr_t>(p) & 15))
      return set_error(CRESS_E_ARG, "cress_hevi_substep_noalloc: input buffer null or not 16-byte aligned");
  for (auto p : dev_out)
    if (!p || (reinterpret_cast<uintptr_t>(p) & 15))
      return set_error(CRESS_E_ARG, "cress_hevi_substep_noalloc: output buffer null or not 16-byte aligned");
  for (int n = 0; n < CRESS_B_N; ++n)
    if (!base3d[n]) return set_error(CRESS_E_ARG, "cress_hevi_substep_noalloc: base array %d is null", n);
  const int ni = cfg->ni, nj = cfg->nj, nk = cfg->nk;
  if (ni < 8 || nj < 8 || nk < 8)
    return set_error(CRESS_E_ARG, "cress_hevi_substep_noalloc: dims too small (%d,%d,%d)", ni, nj, nk);
  if (nk > kNoAllocMaxNk)
    return set_error(CRESS_E_ARG,
                     "cress_hevi_substep_noalloc: nk=%d exceeds the %d levels its fixed device scratch holds",
                     nk, kNoAllocMaxNk);
  if (cfg->impopt != 1 || cfg->gwmopt != 0 || cfg->bbc != 2 || cfg->tbc != 2 ||
      !(cfg->wbc == -1 && cfg->ebc == -1 && cfg->sbc == -1 && cfg->nbc == -1))
    return set_error(CRESS_E_UNSUPPORTED,
                     "cress_hevi_substep_noalloc: needs impopt=1, gwmopt=0, periodic sides, bbc=tbc=2");
  if (cfg->dx <= 0.f || cfg->dy <= 0.f || cfg->dz <= 0.f)
    return set_error(CRESS_E_ARG, "cress_hevi_substep_noalloc: non-positive grid spacing");
  int dev = 0;
  int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  if (dev < 0 || dev >= kMaxDevices) return set_error(CRESS_E_ARG, "device index %d out of range", dev);
  NoAllocScratch* sd = nullptr;
  if ((rc = scratch_address(dev, &sd))) return rc;
  EncodeTiledFn fn = encoder();
  if (!fn) return set_error(CRESS_E_CUDA, "cuTensorMapEncodeTiled entry point unavailable");

  // Host image of the scratch, built in a static per-thread buffer.
  static thread_local NoAllocScratch h;
  std::memset(&h, 0, sizeof h);
  const int ncol = nk + 1;
  auto at = [&](const float* a, int i, int j, int k) {
    return a[(size_t)i + (size_t)(ni + 2) * ((size_t)j + (size_t)(nj + 2) * (size_t)(k - 1))];
  };
  const int map[CRESS_B_N] = {C_JCB, C_JCB8U, C_JCB8V, C_JCB8W, C_RBR, C_PTBR,
                              C_RST, C_RST8U, C_RST8V, C_RST8W, C_RCSQ};
  const int ic = ni / 2, jc = nj / 2;
  for (int n = 0; n < CRESS_B_N; ++n)
    for (int k = 1; k <= nk; ++k) {
      const float v = at(base3d[n], ic, jc, k);
      h.col[map[n] * ncol + k] = v;
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          const float x = at(base3d[n], i, j, k);
          if (x != v && !(std::isnan(x) && std::isnan(v)))
            return set_error(CRESS_E_NONUNIFORM, "base array %d varies horizontally at (%d,%d,%d)", n, i, j, k);
        }
    }
  const int inv_src[6] = {C_RST8U, C_RST8V, C_JCB, C_RCSQ, C_RST8W, C_JCB8W};
  const int inv_dst[6] = {C_IRST8U, C_IRST8V, C_IJCB, C_IRCSQ, C_IRST8W, C_IJCB8W};
  for (int n = 0; n < 6; ++n)
    for (int k = 1; k <= nk; ++k) {
      const float v = h.col[inv_src[n] * ncol + k];
      h.col[inv_dst[n] * ncol + k] = (v != 0.f) ? 1.f / v : 0.f;
    }
  // w-system coefficients (stepwi.f90:308-416) and Thomas factors
  // (gaussel.f90:189-240), as the context API forms them.
  const float g = 9.8f;
  const float dziv = 1.f / cfg->dz, weicoe = cfg->weicoe, g05 = .5f * g;
  const float sbsqzi = dts * dts * weicoe * weicoe * dziv;
  const float sbsqg5 = .5f * g * dts * dts * weicoe * weicoe;
  float fwc[kNoAllocMaxNk + 2] = {0}, wcc[kNoAllocMaxNk + 2] = {0}, ss[kNoAllocMaxNk + 2] = {0},
        tt[kNoAllocMaxNk + 2] = {0};
  auto C = [&](int f, int k) { return h.col[f * ncol + k]; };
  for (int k = 2; k <= nk - 2; ++k) {
    const float t1 = g05 * C(C_RBR, k) / C(C_RCSQ, k), t2 = dziv / C(C_JCB, k);
    fwc[k] = t1 + t2;
    wcc[k] = t1 - t2;
  }
  for (int k = 3; k <= nk - 2; ++k) {
    if (cfg->buyopt == 0) {
      const float a = sbsqzi / C(C_RST8W, k), mm = a * C(C_RCSQ, k - 1), nn = a * C(C_RCSQ, k);
      h.rr[k] = -mm * fwc[k - 1];
      ss[k] = 1.f + (nn * fwc[k] - mm * wcc[k - 1]);
      tt[k] = nn * wcc[k];
    } else {
      const float rstiv = 1.f / C(C_RST8W, k), a = rstiv * sbsqzi, b = rstiv * sbsqg5;
      const float mm = b * C(C_RST, k - 1) - a * C(C_RCSQ, k - 1);
      const float nn = b * C(C_RST, k) + a * C(C_RCSQ, k);
      h.rr[k] = mm * fwc[k - 1];
      ss[k] = 1.f + (mm * wcc[k - 1] + nn * fwc[k]);
      tt[k] = nn * wcc[k];
    }
  }
  const int ks = 3, ke = nk - 2;
  h.aa[ks] = 1.0 / (double)ss[ks];
  h.cp[ks] = (double)tt[ks] * h.aa[ks];
  for (int k = ks + 1; k <= ke - 1; ++k) {
    h.aa[k] = 1.0 / ((double)ss[k] - (double)h.rr[k] * h.cp[k - 1]);
    h.cp[k] = (double)tt[k] * h.aa[k];
  }
  h.aa[ke] = 1.0 / ((double)ss[ke] - (double)h.rr[ke] * h.cp[ke - 1]);
  h.err = 0;

  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if ((rc = cuda_check(cudaMemcpyAsync(sd, &h, sizeof h, cudaMemcpyHostToDevice, st), "copy to hevi scratch")))
    return rc;

  const Grid gr = make_grid(ni, nj, nk);
  const int tile = 0;
  const int TY = hevi_tile_rows(tile);
  HeviMaps maps;
  if ((rc = encode(fn, gr, u_old, TY + 2, &maps.u)) || (rc = encode(fn, gr, v_old, TY + 3, &maps.v)) ||
      (rc = encode(fn, gr, w_old, TY + 2, &maps.w)) || (rc = encode(fn, gr, p_old, TY + 2, &maps.p)) ||
      (rc = encode(fn, gr, ufrc, TY, &maps.uf)) || (rc = encode(fn, gr, vfrc, TY + 1, &maps.vf)) ||
      (rc = encode(fn, gr, wfrc, TY, &maps.wf)) || (rc = encode(fn, gr, pfrc, TY, &maps.pf)))
    return rc;
  HeviArgs a{};
  a.g = gr;
  a.u_old = u_old; a.v_old = v_old; a.p_old = p_old;
  a.u_new = u_new; a.v_new = v_new; a.w_new = w_new; a.p_new = p_new;
  a.col = sd->col;
  a.thom_rr = sd->rr; a.thom_aa = sd->aa; a.thom_cp = sd->cp;
  a.err = &sd->err;
  a.dts = dts;
  a.dxiv = 1.f / cfg->dx; a.dyiv = 1.f / cfg->dy; a.dziv = dziv;
  a.divch = 0.05f / dts * cfg->dx * cfg->dy;   // pgrad.f90:253 (divndc = 0.05)
  a.divcv = 0.05f / dts * cfg->dz * cfg->dz;   // pgrad.f90:254
  a.weicoe = weicoe;
  a.dtdzw = dts * dziv * weicoe;
  a.dtw = dts * weicoe;
  a.g05 = g05;
  a.g05n = -.5f * g;
  a.divopt = cfg->divopt; a.buyopt = cfg->buyopt; a.sthopt = cfg->sthopt; a.bbc = cfg->bbc;
  if ((rc = launch_hevi_substep(a, maps, tile, st)))
    return set_error(rc, "cress_hevi_substep_noalloc: launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  int err = 0;
  if ((rc = cuda_check(cudaMemcpyAsync(&err, &sd->err, sizeof(int), cudaMemcpyDeviceToHost, st), "read error word")) ||
      (rc = cuda_check(cudaStreamSynchronize(st), "cress_hevi_substep_noalloc sync")))
    return rc;
  if (err) return set_error(CRESS_E_TIMEOUT, "cress_hevi_substep_noalloc: a bounded device-side wait gave up");
  return CRESS_OK;
}

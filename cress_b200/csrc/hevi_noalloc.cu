// HE-VI substep entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc from inside their time loop: a host
// model whose device arrays all live in a pool it sized up front, or a
// framework whose caching allocator owns the device.  They already hold the
// old and new u, v, w, p' and the four forcings in their own buffers; what
// the substep additionally needs is small per-column data (1-D base-state
// columns, their reciprocals, the elimination factors of the w system and
// an error word).  Here that data lives in one file-scope __device__ array
// of fixed size, so the call allocates nothing.  The kernel is the one the
// context API launches for the same HE-VI tile (cfg->tile 0..10; tile 0,
// the default, is k_hevi2); tile 11 reads a level table this entry point
// does not hold and is rejected.
//
// Limits and sharing:
//   * nk <= kNoAllocMaxNk (256 levels); larger grids are rejected.
//   * The array is one per device and holds its contents between calls.
//     A call rewrites it whenever its parameters differ from the previous
//     call's on that device and always clears the error word, so no state
//     carries over; but two calls whose kernels overlap on the GPU (e.g. on
//     different streams) race on it: serialize them.
//   * The horizontal-uniformity scan of the 11 base arrays (every point,
//     as cress_set_base3d does) and the column and factor set-up run only
//     when the call's parameters change: dims, spacing, dts, weicoe, buyopt,
//     the base-array pointers, or any value of the base arrays' centre
//     column.  A caller that changes base values off the centre column in
//     place, behind the same pointers, is not re-scanned.
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
#include "wsystem.h"

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

// What the device array of one GPU was last filled from: the parameters the
// set-up depends on, the base arrays' centre columns and the host image.
struct SetupKey {
  int ni = 0, nj = 0, nk = 0, buyopt = -1;
  float dx = 0.f, dy = 0.f, dz = 0.f, dts = 0.f, weicoe = 0.f;
  const float* base[CRESS_B_N] = {};
  bool operator==(const SetupKey& o) const {
    auto same = [](float x, float y) { return std::memcmp(&x, &y, sizeof x) == 0; };
    if (ni != o.ni || nj != o.nj || nk != o.nk || buyopt != o.buyopt || !same(dx, o.dx) || !same(dy, o.dy) ||
        !same(dz, o.dz) || !same(dts, o.dts) || !same(weicoe, o.weicoe))
      return false;
    for (int n = 0; n < CRESS_B_N; ++n)
      if (base[n] != o.base[n]) return false;
    return true;
  }
};
struct DeviceSetup {
  bool valid = false;
  SetupKey key;
  float centre[CRESS_B_N * (kNoAllocMaxNk + 1)];
  NoAllocScratch image;
};
DeviceSetup* g_setup[kMaxDevices];   // host memory, made on a device's first call

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

// Device address of the scratch on the current device (set up once; the
// caller holds g_mu).
int scratch_address(int dev, NoAllocScratch** out) {
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
  if (cfg->tile < 0 || cfg->tile > 10)
    return set_error(CRESS_E_UNSUPPORTED,
                     "cress_hevi_substep_noalloc: tile %d (tiles 0-10; tile 11 needs a level table)", cfg->tile);
  EncodeTiledFn fn = encoder();
  if (!fn) return set_error(CRESS_E_CUDA, "cuTensorMapEncodeTiled entry point unavailable");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);

  std::lock_guard<std::mutex> lk(g_mu);
  NoAllocScratch* sd = nullptr;
  if ((rc = scratch_address(dev, &sd))) return rc;
  if (!g_setup[dev]) g_setup[dev] = new DeviceSetup();
  DeviceSetup& ds = *g_setup[dev];
  SetupKey key;
  key.ni = ni; key.nj = nj; key.nk = nk; key.buyopt = cfg->buyopt;
  key.dx = cfg->dx; key.dy = cfg->dy; key.dz = cfg->dz; key.dts = dts; key.weicoe = cfg->weicoe;
  for (int n = 0; n < CRESS_B_N; ++n) key.base[n] = base3d[n];
  // the centre column of every base array (a cheap check for values
  // changed in place behind the same pointers)
  const int ic = ni / 2, jc = nj / 2;
  bool same = ds.valid && ds.key == key;
  for (int n = 0; n < CRESS_B_N; ++n)
    for (int k = 1; k <= nk; ++k) {
      const float v = base3d[n][(size_t)ic + (size_t)(ni + 2) * ((size_t)jc + (size_t)(nj + 2) * (size_t)(k - 1))];
      float& c = ds.centre[n * (kNoAllocMaxNk + 1) + k];
      if (same && std::memcmp(&c, &v, sizeof v) != 0) same = false;
      c = v;
    }
  if (same) {
    // the device array already holds this set-up: clear the error word only
    if ((rc = cuda_check(cudaMemsetAsync(&sd->err, 0, sizeof(int), st), "clear error word"))) return rc;
  } else {
    ds.valid = false;
    NoAllocScratch& h = ds.image;
    std::memset(&h, 0, sizeof h);
    const NonUniform bad = base_columns(base3d, ni, nj, nk, h.col);
    if (bad.n >= 0)
      return set_error(CRESS_E_NONUNIFORM, "base array %d varies horizontally at (%d,%d,%d)", bad.n, bad.i,
                       bad.j, bad.k);
    float work[4 * (kNoAllocMaxNk + 2)];
    w_system_factors(h.col, nk, cfg->dz, cfg->weicoe, cfg->buyopt, dts, h.rr, h.aa, h.cp, work);
    h.err = 0;
    if ((rc = cuda_check(cudaMemcpyAsync(sd, &h, sizeof h, cudaMemcpyHostToDevice, st), "copy to hevi scratch")))
      return rc;
    ds.key = key;
    ds.valid = true;
  }

  const Grid gr = make_grid(ni, nj, nk);
  const int tile = cfg->tile;
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
  const float dziv = 1.f / cfg->dz, weicoe = cfg->weicoe;
  a.dxiv = 1.f / cfg->dx; a.dyiv = 1.f / cfg->dy; a.dziv = dziv;
  a.divch = kDivndc / dts * cfg->dx * cfg->dy;   // pgrad.f90:253
  a.divcv = kDivndc / dts * cfg->dz * cfg->dz;   // pgrad.f90:254
  a.weicoe = weicoe;
  a.dtdzw = dts * dziv * weicoe;
  a.dtw = dts * weicoe;
  a.g05 = .5f * kG;
  a.g05n = -.5f * kG;
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

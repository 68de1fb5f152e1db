// C-ABI implementation: contexts, device-resident state, host syncs and the
// small-step driver.  Declarations and the reference interface each entry
// point replaces are in include/cress_b200.h.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#include "../../include/cress_b200.h"
#include "common.cuh"
#include "ctx.h"
#include "diag.cuh"
#include "hevi.cuh"
#include "forcing.cuh"
#include "openbc.cuh"
#include "tke.cuh"
#include "micro.cuh"
#include "mlp_impl.cuh"
#include "wsystem.h"

namespace cress {

thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return CRESS_OK;
  return set_error(CRESS_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

float* Ctx::alloc_field() {
  float* p = nullptr;
  if (cudaMalloc(&p, sizeof(float) * (size_t)g.count()) != cudaSuccess) return nullptr;
  cudaMemsetAsync(p, 0, sizeof(float) * (size_t)g.count(), stream);
  owned.push_back(p);
  return p;
}

void Ctx::free_learned() {
  for (void* p : lb_owned) cudaFree(p);
  lb_owned.clear();
  lb = LearnedBuffers{};
  mlp = nullptr;
}

std::vector<float*> Ctx::pointer_state() const {
  std::vector<float*> s;
  for (int f = 0; f < CRESS_NFIELD; ++f) {
    for (int l = 0; l < 4; ++l) s.push_back(lev[f][l]);
    s.push_back(spare[f]);
  }
  return s;
}

void Ctx::set_pointer_state(const std::vector<float*>& s) {
  size_t n = 0;
  for (int f = 0; f < CRESS_NFIELD; ++f) {
    for (int l = 0; l < 4; ++l) lev[f][l] = s[n++];
    spare[f] = s[n++];
  }
}

void Ctx::free_graphs() {
  for (auto& kv : grec)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  grec.clear();
  gseen.clear();
}

// One large step, replayed from a CUDA graph when this pointer state and
// these parameters were seen before: the first occurrence runs eagerly
// (it fills the host-side caches: elimination factors, tensor maps), the
// second is captured and instantiated, later ones launch the graph and
// move the pointer state on as the eager step would.  Steps that sample
// training tuples (they read a count back on the host) always run eagerly.
int Ctx::step(bool filter, float dtb, int nsstp, float dts) {
  if (!graphs || sampler) return large_step(filter, dtb, nsstp, dts);
  const std::vector<float*> pre = pointer_state();
  std::string key(reinterpret_cast<const char*>(pre.data()), pre.size() * sizeof(float*));
  const struct { int filter, nsstp; float dtb, dts, resid; const void* mlp; int chunk; } p{
      filter ? 1 : 0, nsstp, dtb, dts, resid_tol, mlp, lb.chunk};
  key.append(reinterpret_cast<const char*>(&p), sizeof p);
  auto it = grec.find(key);
  if (it == grec.end()) {
    if (gseen[key]++ == 0) return large_step(filter, dtb, nsstp, dts);
    const long long l0 = launches;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      return large_step(filter, dtb, nsstp, dts);
    }
    const int rc = large_step(filter, dtb, nsstp, dts);
    const cudaError_t e = cudaStreamEndCapture(stream, &graph);
    GraphRec r;
    if (rc || e != cudaSuccess || cudaGraphInstantiate(&r.exec, graph, 0) != cudaSuccess) {
      // nothing ran: restore the pointer state and run eagerly
      cudaGetLastError();
      if (graph) cudaGraphDestroy(graph);
      set_pointer_state(pre);
      launches = l0;
      graphs = false;
      return large_step(filter, dtb, nsstp, dts);
    }
    cudaGraphDestroy(graph);
    r.nlaunch = launches - l0;
    launches = l0;
    r.post = pointer_state();
    it = grec.emplace(key, std::move(r)).first;
  }
  if (cudaGraphLaunch(it->second.exec, stream) != cudaSuccess)
    return set_error(CRESS_E_CUDA, "cudaGraphLaunch: %s", cudaGetErrorString(cudaGetLastError()));
  launches += it->second.nlaunch;
  set_pointer_state(it->second.post);
  return CRESS_OK;
}

Ctx::~Ctx() {
  cudaSetDevice(device);
  if (copy_stream) {
    cudaStreamSynchronize(copy_stream);
    cudaStreamDestroy(copy_stream);
  }
  for (int b = 0; b < 2; ++b) {
    if (ev_out[b]) cudaEventDestroy(ev_out[b]);
    if (ev_done[b]) cudaEventDestroy(ev_done[b]);
  }
  if (err_h) cudaFreeHost(err_h);
  if (in_stream) {
    cudaStreamSynchronize(in_stream);
    cudaStreamDestroy(in_stream);
  }
  for (int l = 0; l < 4; ++l) {
    if (ev_in[l]) cudaEventDestroy(ev_in[l]);
    if (ev_in_free[l]) cudaEventDestroy(ev_in_free[l]);
  }
  free_graphs();
  free_learned();
  if (slab) cress_slab_detach(reinterpret_cast<cress_ctx*>(this));
  if (rec_d) cudaFree(rec_d);
  for (void* p : owned) cudaFree(p);
  if (own_stream) cudaStreamDestroy(own_stream);
}

// Host fields are contiguous (pitch ni+2); device fields have pitch px.
// A strided copy of ~2 KB rows runs far below the link's bandwidth, so a
// field crosses as one contiguous copy into (or out of) a staging buffer
// and a kernel moves it between the two pitches.  Stream order keeps the
// staging buffer's uses apart.
int Ctx::stage() {
  if (stage_d) return CRESS_OK;
  const size_t n = (size_t)(g.ni + 2) * (size_t)(g.nj + 2) * (size_t)g.nk;
  int rc = cuda_check(cudaMalloc(&stage_d, sizeof(float) * n), "cudaMalloc staging buffer");
  if (!rc) owned.push_back(stage_d);
  return rc;
}

int Ctx::put_host(float* dst, const float* host) {
  const long long rows = (long long)(g.nj + 2) * g.nk;
  const size_t bytes = sizeof(float) * (size_t)(g.ni + 2) * (size_t)rows;
  int rc;
  if ((rc = stage())) return rc;
  if ((rc = cuda_check(cudaMemcpyAsync(stage_d, host, bytes, cudaMemcpyHostToDevice, stream), "host->device copy")))
    return rc;
  ++launches;
  return launch_repitch(stage_d, g.ni + 2, dst, g.px, g.ni + 2, rows, stream);
}

int Ctx::get_host(float* host, const float* src) {
  const long long rows = (long long)(g.nj + 2) * g.nk;
  const size_t bytes = sizeof(float) * (size_t)(g.ni + 2) * (size_t)rows;
  int rc;
  if ((rc = stage())) return rc;
  if ((rc = launch_repitch(src, g.px, stage_d, g.ni + 2, g.ni + 2, rows, stream))) return rc;
  ++launches;
  return cuda_check(cudaMemcpyAsync(host, stage_d, bytes, cudaMemcpyDeviceToHost, stream), "device->host copy");
}

// Asynchronous read-back of whole fields of one time level: the fields
// are repitched on the context's stream into one host-layout buffer each
// (two sets, used in turn), then copied to the host on a second stream,
// with the device error word as the work before the read-back left it.
// A read-back's repitch waits on the device for the copies of the
// read-back two before it, the last user of its set; cress_wait_fields
// waits for them on the host without waiting for the context's stream.
int Ctx::get_async(int level, int n, const int* fields, float* const* host) {
  int rc;
  if (!copy_stream) {
    if ((rc = cuda_check(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking), "copy stream")) ||
        (rc = cuda_check(cudaHostAlloc(&err_h, 2 * sizeof(int), cudaHostAllocDefault), "cudaHostAlloc error words")))
      return rc;
    for (int b = 0; b < 2; ++b)
      if ((rc = cuda_check(cudaEventCreateWithFlags(&ev_out[b], cudaEventDisableTiming), "event")) ||
          (rc = cuda_check(cudaEventCreateWithFlags(&ev_done[b], cudaEventDisableTiming), "event")))
        return rc;
  }
  const long long rows = (long long)(g.nj + 2) * g.nk;
  const size_t bytes = sizeof(float) * (size_t)(g.ni + 2) * (size_t)rows;
  const int b = (int)(out_issued & 1);
  if (out_issued >= 2 && (rc = cuda_check(cudaStreamWaitEvent(stream, ev_done[b], 0), "wait earlier read-back")))
    return rc;
  for (int q = 0; q < n; ++q) {
    float*& st = stage_out[fields[q]][b];
    if (!st) {
      if ((rc = cuda_check(cudaMalloc(&st, bytes), "cudaMalloc read-back buffer"))) return rc;
      owned.push_back(st);
    }
    if ((rc = launch_repitch(lev[fields[q]][level], g.px, st, g.ni + 2, g.ni + 2, rows, stream))) return rc;
    ++launches;
  }
  if ((rc = cuda_check(cudaEventRecord(ev_out[b], stream), "record read-back")) ||
      (rc = cuda_check(cudaStreamWaitEvent(copy_stream, ev_out[b], 0), "order read-back")) ||
      (rc = cuda_check(cudaMemcpyAsync(&err_h[b], err_d, sizeof(int), cudaMemcpyDeviceToHost, copy_stream),
                       "read error word")))
    return rc;
  for (int q = 0; q < n; ++q)
    if ((rc = cuda_check(cudaMemcpyAsync(host[q], stage_out[fields[q]][b], bytes, cudaMemcpyDeviceToHost, copy_stream),
                         "device->host copy")))
      return rc;
  if ((rc = cuda_check(cudaEventRecord(ev_done[b], copy_stream), "record read-back done"))) return rc;
  ++out_issued;
  return CRESS_OK;
}

// Asynchronous input of whole fields of one time level: contiguous
// host->device copies on in_stream, each into its own staging buffer, then
// the repitch kernels on the context's stream, so the copies overlap the
// work already queued there (the previous step) and the copy engine is not
// held up by the repitch of the field before.
int Ctx::put_async(int level, int n, const int* fields, const float* const* host) {
  int rc;
  if (!in_stream && (rc = cuda_check(cudaStreamCreateWithFlags(&in_stream, cudaStreamNonBlocking), "input stream")))
    return rc;
  if (!ev_in[level] &&
      ((rc = cuda_check(cudaEventCreateWithFlags(&ev_in[level], cudaEventDisableTiming), "event")) ||
       (rc = cuda_check(cudaEventCreateWithFlags(&ev_in_free[level], cudaEventDisableTiming), "event"))))
    return rc;
  const long long rows = (long long)(g.nj + 2) * g.nk;
  const size_t bytes = sizeof(float) * (size_t)(g.ni + 2) * (size_t)rows;
  if (in_used[level] && (rc = cuda_check(cudaStreamWaitEvent(in_stream, ev_in_free[level], 0), "order input copies")))
    return rc;
  for (int q = 0; q < n; ++q) {
    float*& st = stage_in[fields[q]][level];
    if (!st) {
      if ((rc = cuda_check(cudaMalloc(&st, bytes), "cudaMalloc input buffer"))) return rc;
      owned.push_back(st);
    }
    if ((rc = cuda_check(cudaMemcpyAsync(st, host[q], bytes, cudaMemcpyHostToDevice, in_stream), "host->device copy")))
      return rc;
  }
  if ((rc = cuda_check(cudaEventRecord(ev_in[level], in_stream), "record input copies")) ||
      (rc = cuda_check(cudaStreamWaitEvent(stream, ev_in[level], 0), "wait input copies")))
    return rc;
  for (int q = 0; q < n; ++q) {
    const int f = fields[q];
    if ((rc = launch_repitch(stage_in[f][level], g.ni + 2, lev[f][level], g.px, g.ni + 2, rows, stream))) return rc;
    ++launches;
  }
  if ((rc = cuda_check(cudaEventRecord(ev_in_free[level], stream), "record input repitch"))) return rc;
  in_used[level] = true;
  return CRESS_OK;
}

// Read-backs complete in issue order (one copy stream).  A nonzero error
// word in a completed read-back (a bounded device-side wait gave up in the
// work before it) is reported once and the word cleared.
int Ctx::wait_async(int keep) {
  bool failed = false;
  while (out_issued - out_waited > keep) {
    const int b = (int)(out_waited & 1);
    const int rc = cuda_check(cudaEventSynchronize(ev_done[b]), "wait read-back");
    if (rc) return rc;
    failed = failed || err_h[b] != 0;
    ++out_waited;
  }
  if (failed) {
    cudaMemsetAsync(err_d, 0, sizeof(int), stream);
    return set_error(CRESS_E_TIMEOUT, "a bounded device-side wait gave up (TMA staging did not complete)");
  }
  return CRESS_OK;
}

// Elimination factors of the w system for one dts (w_system_factors,
// wsystem.h: s_stepwi's coefficients and s_gaussel's factors), uploaded
// once per distinct dts.
int Ctx::thomas_for(float dts, const ThomasSet** out) {
  uint32_t key;
  std::memcpy(&key, &dts, 4);
  auto it = thomas.find(key);
  if (it != thomas.end()) { *out = &it->second; return CRESS_OK; }
  const int nk = g.nk;
  std::vector<float> rr(nk + 2), work(4 * (nk + 2));
  std::vector<double> cp(nk + 2), aa(nk + 2);
  w_system_factors(col_h.data(), nk, cfg.dz, cfg.weicoe, cfg.buyopt, dts, rr.data(), aa.data(), cp.data(),
                   work.data());
  std::vector<HeviLevel> rows(nk + 1);
  hevi_level_rows(col_h.data(), nk, rr.data(), aa.data(), cp.data(), rows.data());
  std::vector<HeviLevel1> rows1(nk + 1);
  hevi_level_rows1(col_h.data(), nk, rr.data(), aa.data(), cp.data(), rows1.data());
  ThomasSet t;
  if (cudaMalloc(&t.rr, sizeof(float) * (nk + 2)) != cudaSuccess ||
      cudaMalloc(&t.aa, sizeof(double) * (nk + 2)) != cudaSuccess ||
      cudaMalloc(&t.cp, sizeof(double) * (nk + 2)) != cudaSuccess ||
      cudaMalloc(&t.lvl3, sizeof(HeviLevel) * (nk + 1)) != cudaSuccess ||
      cudaMalloc(&t.lvl4, sizeof(HeviLevel1) * (nk + 1)) != cudaSuccess)
    return set_error(CRESS_E_CUDA, "cudaMalloc (tridiagonal factors) failed");
  owned.push_back(t.rr); owned.push_back(t.aa); owned.push_back(t.cp); owned.push_back(t.lvl3);
  owned.push_back(t.lvl4);
  int rc;
  if ((rc = cuda_check(cudaMemcpyAsync(t.rr, rr.data(), sizeof(float) * (nk + 2), cudaMemcpyHostToDevice, stream), "copy rr")) ||
      (rc = cuda_check(cudaMemcpyAsync(t.aa, aa.data(), sizeof(double) * (nk + 2), cudaMemcpyHostToDevice, stream), "copy aa")) ||
      (rc = cuda_check(cudaMemcpyAsync(t.cp, cp.data(), sizeof(double) * (nk + 2), cudaMemcpyHostToDevice, stream), "copy cp")) ||
      (rc = cuda_check(cudaMemcpyAsync(t.lvl3, rows.data(), sizeof(HeviLevel) * (nk + 1), cudaMemcpyHostToDevice,
                                       stream), "copy level table")) ||
      (rc = cuda_check(cudaMemcpyAsync(t.lvl4, rows1.data(), sizeof(HeviLevel1) * (nk + 1),
                                       cudaMemcpyHostToDevice, stream), "copy level table")))
    return rc;
  // The host vectors above are freed on return; make the copies complete.
  if ((rc = cuda_check(cudaStreamSynchronize(stream), "sync after factor upload"))) return rc;
  auto res = thomas.emplace(key, t);
  *out = &res.first->second;
  return CRESS_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link-time dependency on libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
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

// 3-D tensor map (x = i, y = j, z = k-1) over one field buffer with a box
// of kHeviBoxX x rows x 1, cached per (buffer, rows).
int Ctx::tmap(const float* buf, int rows, CUtensorMap* out) {
  auto key = std::make_pair(reinterpret_cast<const void*>(buf), rows);
  auto it = tmaps.find(key);
  if (it != tmaps.end()) { *out = it->second; return CRESS_OK; }
  EncodeTiledFn fn = encode_fn();
  if (!fn) return set_error(CRESS_E_CUDA, "cuTensorMapEncodeTiled entry point unavailable");
  CUtensorMap m;
  cuuint64_t dims[3] = {(cuuint64_t)g.px, (cuuint64_t)g.py, (cuuint64_t)g.nk};
  cuuint64_t strides[2] = {(cuuint64_t)g.px * 4, (cuuint64_t)g.plane * 4};
  cuuint32_t box[3] = {(cuuint32_t)kHeviBoxX, (cuuint32_t)rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(buf), dims, strides, box,
                  estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(CRESS_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  tmaps.emplace(key, m);
  *out = m;
  return CRESS_OK;
}

// The level table of the large-step kernels for a step of 2*dtb = dtb2
// (forcing.cuh: columns, reciprocals, derived quotients), formed on the
// host with the same IEEE operations the device would use and kept per
// distinct dtb2 (the half first step and the regular one).
int Ctx::level_table(float dtb2, const float** out) {
  uint32_t key;
  std::memcpy(&key, &dtb2, 4);
  auto it = level_tables.find(key);
  if (it != level_tables.end()) { *out = it->second; return CRESS_OK; }
  const int nk = g.nk, nc = nk + 1;
  auto B = [&](int f, int kk) { return col_h[(size_t)f * nc + kk]; };
  std::vector<float> t((size_t)nc * kLevelStride, 0.f);
  for (int kk = 0; kk < nc; ++kk)
    for (int f = 0; f < D_NFIELDS; ++f) t[(size_t)kk * kLevelStride + f] = level_value(f, kk, B, dtb2);
  float* d = nullptr;
  int rc;
  if ((rc = cuda_check(cudaMalloc(&d, sizeof(float) * t.size()), "cudaMalloc level table"))) return rc;
  owned.push_back(d);
  if ((rc = cuda_check(cudaMemcpyAsync(d, t.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice, stream),
                       "copy level table")) ||
      (rc = cuda_check(cudaStreamSynchronize(stream), "sync level table")))
    return rc;
  level_tables.emplace(key, d);
  *out = d;
  return CRESS_OK;
}

int Ctx::small_steps(int nsstp, float dts) { return small_steps(nsstp, dts, nullptr); }

int Ctx::small_steps(int nsstp, float dts, std::vector<HeviJob>* jobs) {
  if (!base_set) return set_error(CRESS_E_STATE, "cress_small_steps: base state not set");
  if (jobs && (cfg.impopt != 1 || (cfg.tile != 0 && cfg.tile != 13) || g.openx))
    return set_error(CRESS_E_UNSUPPORTED, "ensemble small steps need impopt=1, tile 0 or 13 and periodic x");
  if (g.openx && cfg.tile != 0 && cfg.tile != 11 && cfg.tile != 12 && cfg.tile != 13)
    return set_error(CRESS_E_UNSUPPORTED, "open x boundaries run the HE-VI tiles 0, 11, 12 and 13");
  if (nsstp < 1) return set_error(CRESS_E_ARG, "cress_small_steps: nsstp=%d", nsstp);
  const bool heve = cfg.impopt == 0;
  const ThomasSet* th = nullptr;
  int rc = heve ? CRESS_OK : thomas_for(dts, &th);
  if (rc) return rc;
  HeviArgs a{};
  a.g = g;
  a.col = col_d;
  if (level_tables.empty()) {   // any level table serves: the small step reads only its columns
    const float* t = nullptr;
    if ((rc = level_table(0.f, &t))) return rc;
  }
  a.lvl = level_tables.begin()->second;
  if (th) { a.thom_rr = th->rr; a.thom_aa = th->aa; a.thom_cp = th->cp; a.lvl3 = th->lvl3; a.lvl4 = th->lvl4; }
  a.err = err_d;
  a.dts = dts;
  a.dxiv = 1.f / cfg.dx; a.dyiv = 1.f / cfg.dy; a.dziv = 1.f / cfg.dz;
  a.divch = kDivndc / dts * cfg.dx * cfg.dy;     // pgrad.f90:253
  a.divcv = kDivndc / dts * cfg.dz * cfg.dz;     // pgrad.f90:254
  a.weicoe = cfg.weicoe;
  a.dtdzw = dts * a.dziv * cfg.weicoe;           // pgradiv.f90:135
  a.dtw = dts * cfg.weicoe;                      // buoywsi.f90:153
  a.g05 = .5f * kG;
  a.g05n = -.5f * kG;
  a.divopt = cfg.divopt; a.buyopt = cfg.buyopt; a.sthopt = cfg.sthopt; a.bbc = cfg.bbc;
  a.spin = spin_limit;
  const int TY = hevi_tile_rows(heve ? 0 : cfg.tile);
  HeviMaps maps;
  if ((rc = tmap(lev[CRESS_U][CRESS_FORCING], TY, &maps.uf)) ||
      (rc = tmap(lev[CRESS_V][CRESS_FORCING], TY + 1, &maps.vf)) ||
      (rc = tmap(lev[CRESS_W][CRESS_FORCING], TY, &maps.wf)) ||
      (rc = tmap(lev[CRESS_PP][CRESS_FORCING], TY, &maps.pf)))
    return rc;
  const int F[4] = {CRESS_U, CRESS_V, CRESS_W, CRESS_PP};
  // Substep 1 reads the past level directly (smalldrv.f90:343-346 copies it
  // into the future arrays first); later substeps ping-pong between the
  // future buffer and a spare, so halo reads see old values only.
  float* olds[4];
  float* news[4];
  for (int n = 0; n < 4; ++n) { olds[n] = lev[F[n]][CRESS_PAST]; news[n] = lev[F[n]][CRESS_FUTURE]; }
  for (int s = 0; s < nsstp; ++s) {
    a.u_old = olds[0]; a.v_old = olds[1]; a.p_old = olds[3];
    a.u_new = news[0]; a.v_new = news[1]; a.w_new = news[2]; a.p_new = news[3];
    if ((rc = tmap(olds[0], TY + 2, &maps.u)) || (rc = tmap(olds[1], TY + 3, &maps.v)) ||
        (rc = tmap(olds[2], TY + 2, &maps.w)) || (rc = tmap(olds[3], TY + 2, &maps.p)))
      return rc;
    if (jobs) {
      HeviJob jb;
      std::memset(&jb, 0, sizeof jb);
      jb.maps = maps;
      jb.args = a;
      jobs->push_back(jb);
      rc = CRESS_OK;
    } else if (heve) {
      // the first substep forms the contravariant w of levels 2 and nk-1
      // from the past w (phy2cnt before the loop, smalldrv.f90:358)
      a.wc_from_w = s == 0;
      a.wc_old = wcside[s & 1];
      a.wc_new = wcside[(s + 1) & 1];
      rc = launch_heve_substep(a, maps, stream);
      ++launches;
    } else {
      rc = launch_hevi_substep(a, maps, cfg.tile, stream);
      ++launches;
      if (!rc && g.openx) {   // the boundary columns of this substep (stepuv/stepwi/steppi rbc*)
        RbcSmallArgs r{};
        r.g = g;
        r.cp = rad_d;
        r.col = col_d;
        r.u_old = olds[0]; r.v_old = olds[1]; r.w_old = olds[2]; r.p_old = olds[3];
        r.u_new = news[0]; r.v_new = news[1]; r.w_new = news[2]; r.p_new = news[3];
        r.sthopt = cfg.sthopt;
        r.bbc = cfg.bbc;
        rc = launch_rbc_small(r, stream);
        ++launches;
      }
    }
    if (rc) return set_error(rc, "small-step launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    if (slab) {   // y slab: the new level's ghost rows from the neighbours (shiftsx after each substep)
      const int stag[4] = {STAG_U, STAG_V, STAG_S, STAG_S};
      if ((rc = slab->exchange(this, 4, news, stag))) return rc;
    }
    for (int n = 0; n < 4; ++n) {
      float* t = news[n];
      news[n] = (s == 0) ? spare[F[n]] : olds[n];
      olds[n] = t;
    }
  }
  // olds[] now hold the result; make it the future level.
  for (int n = 0; n < 4; ++n) {
    if (olds[n] != lev[F[n]][CRESS_FUTURE]) {
      spare[F[n]] = lev[F[n]][CRESS_FUTURE];
      lev[F[n]][CRESS_FUTURE] = olds[n];
    }
  }
  return CRESS_OK;
}

// One large step on the device-resident state in s_intgdrv's order
// (SrcOrig/intgdrv.f90:832-1119): forcing (moist buoyancy when cphopt=3),
// small steps, the theta' step (inside k_force), the moist scalar steps,
// s_cloudphy, s_timeflt (not at ctime=0), s_satadjst on t and t+dt,
// periodic ghost planes, swp2nxt.
int Ctx::large_step(bool filter, float dtb, int nsstp, float dts, int phase) {
  if (!base_set || !large_set)
    return set_error(CRESS_E_STATE, "cress_large_step: base state (set_base3d, set_base_large) not set");
  if (!(cfg.advopt == 2 || cfg.advopt == 3) || cfg.tubopt < 0 || cfg.tubopt > 2 ||
      !(cfg.cphopt == 0 || cfg.cphopt == 3) ||
      !(cfg.smtopt == 0 || cfg.smtopt % 10 == 2 || cfg.smtopt % 10 == 3) ||
      !(cfg.vspopt == 0 || cfg.vspopt == 2) || !(cfg.coropt == 0 || cfg.coropt == 1))
    return set_error(CRESS_E_UNSUPPORTED,
                     "cress_large_step: needs advopt 2/3, tubopt 0/1/2, cphopt 0/3, smtopt 0/2/3, vspopt 0/2, coropt 0/1");
  const bool tke = cfg.tubopt == 2;
  const bool moist = cfg.cphopt == 3;
  if (moist && !moist_set) return set_error(CRESS_E_STATE, "cress_large_step: moist base state not set");
  const int N = CRESS_NOW, P = CRESS_PAST, F = CRESS_FUTURE;
  ForceArgs f{};
  f.g = g;
  f.col = col_d;
  f.u = lev[CRESS_U][N]; f.v = lev[CRESS_V][N]; f.w = lev[CRESS_W][N];
  f.pp = lev[CRESS_PP][N]; f.ptp = lev[CRESS_PTP][N];
  f.up = lev[CRESS_U][P]; f.vp = lev[CRESS_V][P]; f.wp = lev[CRESS_W][P];
  f.ppp = lev[CRESS_PP][P]; f.ptpp = lev[CRESS_PTP][P];
  f.ufrc = lev[CRESS_U][CRESS_FORCING]; f.vfrc = lev[CRESS_V][CRESS_FORCING];
  f.wfrc = lev[CRESS_W][CRESS_FORCING]; f.pfrc = lev[CRESS_PP][CRESS_FORCING];
  f.ptpf = lev[CRESS_PTP][F];
  f.dxiv = 1.f / cfg.dx; f.dyiv = 1.f / cfg.dy; f.dziv = 1.f / cfg.dz;
  f.smhcoe = cfg.smhcoe; f.smvcoe = cfg.smvcoe;
  f.fc = cfg.fc;
  f.dtb2 = 2.f * dtb;
  int rc;
  if ((rc = level_table(f.dtb2, &f.lvl))) return rc;
  f.smtopt = cfg.smtopt; f.vspopt = cfg.vspopt; f.coropt = cfg.coropt; f.sthopt = cfg.sthopt;
  f.advopt = cfg.advopt;
  f.ksp0 = ksp0;
  auto on = [&](int n) { return cfg.vspvar[n] == 'o' ? 1 : 0; };
  f.vsp_u = on(0); f.vsp_v = on(1); f.vsp_w = on(2); f.vsp_p = on(3); f.vsp_pt = on(4);
  if (moist) {
    f.qv = lev[CRESS_QV][N]; f.qc = lev[CRESS_QC][N]; f.qr = lev[CRESS_QR][N];
    f.qi = lev[CRESS_QI][N]; f.qs = lev[CRESS_QS][N]; f.qg = lev[CRESS_QG][N];
  }
  const float cpriv = 3.f;   // min(1/prnum, 3) with prnum = 0.33 (eddyvis.f90:219-222)
  if (cfg.tubopt >= 1) {
    f.rkv = rkv_d;
    // the theta' mixing stages the eddy viscosity (Smagorinsky) or the
    // scalar diffusivity the TKE closure's s_eddydif leaves
    f.rks = tke ? rks_d : rkv_d;
    f.kdiv = tke ? 1 : 0;
    f.cpriv = cpriv;
  }
  if (cfg.tubopt >= 1 && phase != 2) {
    // s_turbdrv up to s_eddyvis on the past level (forceuvw.f90:423-431);
    // with the TKE closure also the per-point terms of s_forcetke
    TurbArgs t{};
    t.g = g;
    t.col = col_d;
    t.lvl = f.lvl;
    t.up = lev[CRESS_U][P]; t.vp = lev[CRESS_V][P]; t.wp = lev[CRESS_W][P];
    t.ptpp = lev[CRESS_PTP][P]; t.ppp = lev[CRESS_PP][P];
    if (moist) {
      t.qvp = lev[CRESS_QV][P]; t.qcp = lev[CRESS_QC][P]; t.qrp = lev[CRESS_QR][P];
      t.qip = lev[CRESS_QI][P]; t.qsp = lev[CRESS_QS][P]; t.qgp = lev[CRESS_QG][P];
    }
    t.rkv = rkv_d;
    t.dxiv = f.dxiv; t.dyiv = f.dyiv; t.dziv = f.dziv;
    t.ds3 = cfg.dx * cfg.dy * cfg.dz;
    t.ckmax = .125f / dtb;
    t.cpriv = cpriv;
    t.thresq = cfg.thresq;
    if (tke) {
      t.tkep = lev[CRESS_TKE][P];
      t.rks = rks_d; t.nsq = nsq_d; t.shr = shr_d; t.dsp = dsp_d;
      t.ds308 = .125f * cfg.dx * cfg.dy * cfg.dz;   // disptke.f90:176
    }
    if ((rc = launch_turb_visc(t, stream))) return set_error(rc, "eddy viscosity launch failed");
    ++launches;
  }
  f.err = err_d;
  if (phase != 2) {
    const float* bufs[FB_NONE] = {lev[CRESS_U][N], lev[CRESS_V][N], lev[CRESS_W][N], lev[CRESS_PP][N],
                                  lev[CRESS_PTP][N], lev[CRESS_U][P], lev[CRESS_V][P], lev[CRESS_W][P],
                                  lev[CRESS_PP][P], lev[CRESS_PTP][P], f.rkv};
    ForceMaps fm;
    for (int sg = 0; sg < 2; ++sg)
      for (int q = 0; q < force_nslots(sg, f.rkv != nullptr); ++q) {
        const int b = force_slot_buf(sg, q);
        const float* buf = (sg == 1 && b == FB_RKV) ? f.rks : bufs[b];   // the theta' mixing's field
        if ((rc = tmap(buf, force_slot_rows(sg, q), &fm.m[sg][q]))) return rc;
      }
    rc = launch_force(f, fm, stream);
    launches += 2;
    if (rc) return set_error(rc, "forcing launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  if (phase == 1) return CRESS_OK;   // an ensemble runs the small steps of all members next
  if (phase == 0 && (rc = small_steps(nsstp, dts))) return rc;
  if (tke) {   // s_forcetke and the TKE part of s_steps (forcetke.f90:269-354, steps.f90:999-1014)
    TkeArgs t{};
    t.g = g;
    t.lvl = f.lvl;
    t.rks = rks_d; t.nsq = nsq_d; t.shr = shr_d; t.dsp = dsp_d;
    t.tkef = lev[CRESS_TKE][F];
    t.dxiv = f.dxiv; t.dyiv = f.dyiv; t.dziv = f.dziv;
    t.smhcoe = cfg.smhcoe; t.smvcoe = cfg.smvcoe;
    t.smtopt = cfg.smtopt; t.vspopt = cfg.vspopt; t.sthopt = cfg.sthopt; t.ksp0 = ksp0;
    t.advopt = cfg.advopt;
    t.vsp_tke = on(9);
    t.err = err_d;
    TkeMaps tm;
    if ((rc = tmap(lev[CRESS_TKE][N], TkeRows::s, &tm.s)) || (rc = tmap(lev[CRESS_TKE][P], TkeRows::s, &tm.sp)) ||
        (rc = tmap(lev[CRESS_U][N], TkeRows::u, &tm.u)) || (rc = tmap(lev[CRESS_V][N], TkeRows::v, &tm.v)) ||
        (rc = tmap(lev[CRESS_W][N], TkeRows::w, &tm.w)) || (rc = tmap(rkv_d, TkeRows::r, &tm.rkv)))
      return rc;
    if ((rc = launch_tke(t, tm, stream))) return set_error(rc, "TKE launch failed");
    ++launches;
  }
  if (moist) {
    MoistScalarArgs m{};
    m.g = g;
    m.col = col_d;
    m.u = lev[CRESS_U][N]; m.v = lev[CRESS_V][N]; m.w = lev[CRESS_W][N];
    for (int n = 0; n < kMoistN; ++n) {
      m.s[n] = lev[CRESS_QV + n][N];
      m.sp[n] = lev[CRESS_QV + n][P];
      m.sf[n] = lev[CRESS_QV + n][F];
    }
    m.dxiv = f.dxiv; m.dyiv = f.dyiv; m.dziv = f.dziv;
    m.smhcoe = cfg.smhcoe; m.smvcoe = cfg.smvcoe; m.dtb2 = f.dtb2;
    m.smtopt = cfg.smtopt; m.vspopt = cfg.vspopt; m.sthopt = cfg.sthopt; m.ksp0 = ksp0;
    m.advopt = cfg.advopt;
    m.vsp_qv = on(5); m.vsp_q = on(6);
    m.rkv = f.rks; m.cpriv = cpriv; m.kdiv = f.kdiv;
    m.err = err_d;
    m.lvl = f.lvl;
    MoistMaps mm;
    for (int n = 0; n < kMoistN; ++n)
      if ((rc = tmap(m.s[n], ScalarRows::s, &mm.s[n])) || (rc = tmap(m.sp[n], ScalarRows::s, &mm.sp[n]))) return rc;
    if ((rc = tmap(m.u, ScalarRows::u, &mm.u)) || (rc = tmap(m.v, ScalarRows::v, &mm.v)) ||
        (rc = tmap(m.w, ScalarRows::w, &mm.w)))
      return rc;
    if (m.rkv && (rc = tmap(m.rkv, ScalarRows::r, &mm.rkv))) return rc;
    if (!m.rkv) mm.rkv = mm.w;
    if ((rc = launch_moist_scalars(m, mm, stream))) return set_error(rc, "moist scalar launch failed");
    ++launches;
  }
  if (g.openx) {   // the leapfrog scalars' boundary columns (steps.f90:1024-1260)
    RbcLeapArgs r{};
    r.g = g;
    r.cp = rad_d;
    auto add = [&](int fld, int var, int kind) {
      r.s[r.n] = lev[fld][N]; r.sp[r.n] = lev[fld][P]; r.sf[r.n] = lev[fld][F];
      r.var[r.n] = var; r.kind[r.n] = kind;
      ++r.n;
    };
    add(CRESS_PTP, RAD_PT, 0);
    if (moist)
      for (int n = 0; n < kMoistN; ++n) add(CRESS_QV + n, RAD_QV + n, n == 0 ? 1 : n < 6 ? 2 : 3);
    if ((rc = launch_rbc_leapfrog(r, stream))) return set_error(rc, "open-boundary scalar launch failed");
    ++launches;
  }
  // the final adjstni of cloudphy runs inside the moist post kernel below
  if (moist && (rc = cloudphy(dtb, cfg.thresq, true))) return rc;
  if (filter) {
    FilterArgs t{};
    t.g = g;
    t.u = lev[CRESS_U][N]; t.v = lev[CRESS_V][N]; t.w = lev[CRESS_W][N];
    t.pp = lev[CRESS_PP][N]; t.ptp = lev[CRESS_PTP][N];
    t.uf = lev[CRESS_U][F]; t.vf = lev[CRESS_V][F]; t.wf = lev[CRESS_W][F];
    t.ppf = lev[CRESS_PP][F]; t.ptpf = lev[CRESS_PTP][F];
    t.up = lev[CRESS_U][P]; t.vp = lev[CRESS_V][P]; t.wp = lev[CRESS_W][P];
    t.ppp = lev[CRESS_PP][P]; t.ptpp = lev[CRESS_PTP][P];
    t.filcoe = cfg.filcoe;
    if (tke) { t.tke = lev[CRESS_TKE][N]; t.tkef = lev[CRESS_TKE][F]; t.tkep = lev[CRESS_TKE][P]; }
    if ((rc = launch_timeflt(t, stream))) return set_error(rc, "timeflt launch failed");
    ++launches;
  }
  if (moist) {
    MoistPostArgs m{};
    m.g = g;
    m.col = col_d;
    for (int n = 0; n < kMoistN; ++n) {
      m.c[n] = lev[CRESS_QV + n][N];
      m.f[n] = lev[CRESS_QV + n][F];
      m.p[n] = lev[CRESS_QV + n][P];
    }
    m.ptpc = lev[CRESS_PTP][N]; m.ppc = lev[CRESS_PP][N];
    m.ptpf = lev[CRESS_PTP][F]; m.ppf = lev[CRESS_PP][F];
    m.filcoe = cfg.filcoe; m.thresq = cfg.thresq; m.filter = filter ? 1 : 0;
    m.adjstni = 1;
    if ((rc = launch_moist_post(m, stream))) return set_error(rc, "moist filter/adjustment launch failed");
    ++launches;
  }
  HaloArgs h{};
  h.g = g;
  // the rotated fields: u, v, w, p', theta' (RadVar order), the moist
  // species, the TKE
  int nrot = moist ? 5 + kMoistN : 5;
  int F5[5 + kMoistN + 1] = {CRESS_U, CRESS_V, CRESS_W, CRESS_PP, CRESS_PTP};
  int S5[5 + kMoistN + 1] = {STAG_U, STAG_V, STAG_S, STAG_S, STAG_S};
  for (int n = 0; n < kMoistN; ++n) { F5[5 + n] = CRESS_QV + n; S5[5 + n] = STAG_S; }
  if (tke) { F5[nrot] = CRESS_TKE; S5[nrot] = STAG_S; ++nrot; }
  for (int lvl : {N, F})
    for (int n = 0; n < nrot; ++n) {
      h.f[h.n] = lev[F5[n]][lvl];
      h.stag[h.n] = S5[n];
      ++h.n;
    }
  if ((rc = launch_halo(h, stream))) return set_error(rc, "halo launch failed");
  ++launches;
  if (slab && (rc = slab->exchange(this, h.n, h.f, h.stag))) return rc;   // y ghosts of t and t+dt
  if (g.openx) {   // s_phasev from the filtered present, past and future levels (intgdrv.f90:1023)
    PhaseArgs ph{};
    ph.g = g;
    ph.cp = rad_d;
    ph.obc = cfg.wbc;
    ph.gwave = cfg.gwave;
    ph.dxiv = 1.f / cfg.dx;
    ph.dtb = dtb;
    ph.dts = dts;
    for (int n = 0; n < nrot; ++n) {
      ph.s[n] = lev[F5[n]][N]; ph.sp[n] = lev[F5[n]][P]; ph.sf[n] = lev[F5[n]][F];
      ph.var[n] = n;   // the rotation list is in RadVar order
    }
    ph.n = nrot;
    if ((rc = launch_phase(ph, stream))) return set_error(rc, "phase-speed launch failed");
    ++launches;
  }
  // swp2nxt: past <- t, t <- t+dt (pointer rotation)
  for (int n = 0; n < nrot; ++n) {
    float* p = lev[F5[n]][P];
    lev[F5[n]][P] = lev[F5[n]][N];
    lev[F5[n]][N] = lev[F5[n]][F];
    lev[F5[n]][F] = p;
  }
  return CRESS_OK;
}

// s_cloudphy for cphopt=3 on the device-resident past and future levels.
int Ctx::cloudphy(float dtb, float thresq, bool defer_adjstni) {
  if (cfg.cphopt != 3 || !prec_d) return set_error(CRESS_E_STATE, "cress_cloudphy: context is not cphopt=3");
  if (!base_set || !moist_set) return set_error(CRESS_E_STATE, "cress_cloudphy: base state not set");
  MicroArgs m{};
  m.g = g;
  m.col = col_d;
  const int P = CRESS_PAST, F = CRESS_FUTURE;
  m.ptpp = lev[CRESS_PTP][P]; m.qvp = lev[CRESS_QV][P]; m.qcp = lev[CRESS_QC][P]; m.qrp = lev[CRESS_QR][P];
  m.qip = lev[CRESS_QI][P]; m.qsp = lev[CRESS_QS][P]; m.qgp = lev[CRESS_QG][P]; m.nip = lev[CRESS_NI][P];
  m.nsp = lev[CRESS_NS][P]; m.ngp = lev[CRESS_NG][P]; m.ppp = lev[CRESS_PP][P];
  m.ptpf = lev[CRESS_PTP][F]; m.qvf = lev[CRESS_QV][F]; m.qcf = lev[CRESS_QC][F]; m.qrf = lev[CRESS_QR][F];
  m.qif = lev[CRESS_QI][F]; m.qsf = lev[CRESS_QS][F]; m.qgf = lev[CRESS_QG][F]; m.nif = lev[CRESS_NI][F];
  m.nsf = lev[CRESS_NS][F]; m.ngf = lev[CRESS_NG][F];
  m.prec = prec_d;
  m.uspd = uspd_d;
  m.dtp_bits = dtp_d;
  m.dtb = 2.f * dtb;        // cloudphy.f90:282
  m.dz = cfg.dz;
  m.thresq = thresq;
  m.defer_adjstni = defer_adjstni ? 1 : 0;
  int rc;
  if (sampler) {
    // tuples of the plain scheme on this step's state (before it changes)
    const long long room = sampler->tcap - sampler->ntup;
    if (room > 0) {
      cudaMemsetAsync(count_d, 0, sizeof(unsigned long long), stream);
      if ((rc = launch_collect_tuples(m, lev[CRESS_W][CRESS_NOW], sampler, sample_stride, sample_keep_zero,
                                      sample_seed++, count_d, stream)))
        return set_error(rc, "tuple sampling launch failed");
      ++launches;
      unsigned long long got = 0;
      cudaMemcpyAsync(&got, count_d, sizeof(got), cudaMemcpyDeviceToHost, stream);
      if ((rc = cuda_check(cudaStreamSynchronize(stream), "tuple sampling"))) return rc;
      const long long add = (long long)got < room ? (long long)got : room;
      sampler->ntup += add;
      sampled += add;
    }
  }
  if (mlp) {
    rc = lb.fused ? launch_cloudphy_fused(m, lev[CRESS_W][CRESS_NOW], mlp, lb, resid_tol, stream, &launches)
                  : launch_cloudphy_learned(m, lev[CRESS_W][CRESS_NOW], mlp, lb, resid_tol, stream, &launches);
    if (rc) return set_error(rc, "learned cloudphy failed: %s", cudaGetErrorString(cudaGetLastError()));
    return CRESS_OK;
  }
  if (slab) {   // the sub-step minimum over all ranks between the halves (chkfall.f90:88)
    if ((rc = launch_cloudphy_src(m, stream))) return set_error(rc, "cloudphy launch failed");
    if ((rc = slab->min_word(this, dtp_d))) return rc;
    rc = launch_cloudphy_fall(m, stream);
  } else {
    rc = launch_cloudphy(m, stream);
  }
  launches += defer_adjstni ? 3 : 4;
  if (rc) return set_error(rc, "cloudphy launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  return CRESS_OK;
}

int Ctx::satadjst(int level, float thresq) {
  if (cfg.cphopt != 3) return set_error(CRESS_E_STATE, "cress_satadjst: context is not cphopt=3");
  if (!base_set || !moist_set) return set_error(CRESS_E_STATE, "cress_satadjst: base state not set");
  SatArgs s{};
  s.g = g;
  s.col = col_d;
  s.pp = lev[CRESS_PP][level];
  s.ptp = lev[CRESS_PTP][level]; s.qv = lev[CRESS_QV][level]; s.qc = lev[CRESS_QC][level];
  s.qi = lev[CRESS_QI][level]; s.ni = lev[CRESS_NI][level];
  s.thresq = thresq;
  int rc = launch_satadjst(s, stream);
  ++launches;
  if (rc) return set_error(rc, "satadjst launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  return CRESS_OK;
}

// Read and clear the device error word (bounded-wait failures).
int Ctx::check_device_error() {
  int h = 0;
  int rc = cuda_check(cudaMemcpyAsync(&h, err_d, sizeof(int), cudaMemcpyDeviceToHost, stream), "read error word");
  if (rc) return rc;
  if ((rc = cuda_check(cudaStreamSynchronize(stream), "sync"))) return rc;
  if (h) {
    cudaMemsetAsync(err_d, 0, sizeof(int), stream);
    return set_error(CRESS_E_TIMEOUT, "a bounded device-side wait gave up (TMA staging did not complete)");
  }
  return CRESS_OK;
}

// Domain diagnostics of one time level (diag.cu): out[0..2] FP64 water,
// precipitated water and mass (kg), out[3..6] max |u|, |v|, |w|, |theta'|,
// out[7] the number of non-finite values.
int Ctx::diagnostics(int level, double* out) {
  if (level < CRESS_PAST || level > CRESS_FUTURE)
    return set_error(CRESS_E_ARG, "cress_diagnostics: level %d (0..2)", level);
  if (!base_set) return set_error(CRESS_E_STATE, "cress_diagnostics: base state not set");
  int rc;
  if (!diag_d) {
    if ((rc = cuda_check(cudaMalloc(&diag_d, sizeof(DiagAcc)), "cudaMalloc diagnostics"))) return rc;
    owned.push_back(diag_d);
  }
  DiagArgs a{};
  a.g = g;
  a.col = col_d;
  a.u = lev[CRESS_U][level]; a.v = lev[CRESS_V][level]; a.w = lev[CRESS_W][level];
  a.pp = lev[CRESS_PP][level]; a.ptp = lev[CRESS_PTP][level];
  if (cfg.cphopt == 3) {
    for (int n = 0; n < 6; ++n) a.q[n] = lev[CRESS_QV + n][level];
    for (int n = 0; n < 3; ++n) a.n[n] = lev[CRESS_NI + n][level];
    a.prec = prec_d;
  }
  a.dv = (double)cfg.dx * (double)cfg.dy * (double)cfg.dz;
  a.dxdy = (double)cfg.dx * (double)cfg.dy;
  a.acc = static_cast<DiagAcc*>(diag_d);
  if ((rc = cuda_check(cudaMemsetAsync(diag_d, 0, sizeof(DiagAcc), stream), "clear diagnostics"))) return rc;
  if ((rc = launch_diag(a, stream))) return set_error(rc, "diagnostics launch failed");
  DiagAcc h{};
  if ((rc = cuda_check(cudaMemcpyAsync(&h, diag_d, sizeof h, cudaMemcpyDeviceToHost, stream), "read diagnostics")) ||
      (rc = cuda_check(cudaStreamSynchronize(stream), "sync")))
    return rc;
  for (int n = 0; n < 3; ++n) out[n] = h.sum[n];
  for (int n = 0; n < 4; ++n) {
    float f;
    std::memcpy(&f, &h.maxbits[n], 4);
    out[3 + n] = f;
  }
  out[7] = (double)h.nonfinite;
  if (h.nonfinite)
    return set_error(CRESS_E_NONFINITE, "%llu non-finite values in time level %d", h.nonfinite, level);
  return CRESS_OK;
}

// Time every HE-VI tile variant over `reps` small-step loops of nsstp
// substeps on the current state (the loop writes only the future level and
// its spare, so the state the next large step starts from is untouched),
// keep the fastest as cfg.tile and drop graphs captured with another tile.
int Ctx::autotune(int nsstp, float dts, int reps, int* best, float* ms) {
  if (nsstp < 1 || reps < 1) return set_error(CRESS_E_ARG, "cress_autotune: nsstp=%d reps=%d", nsstp, reps);
  if (cfg.impopt == 0) return set_error(CRESS_E_UNSUPPORTED, "cress_autotune: the HE-VE step has one tile shape");
  if (slab) return set_error(CRESS_E_UNSUPPORTED, "cress_autotune: a y-slab rank steps with the other ranks");
  const int keep = cfg.tile;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    return set_error(CRESS_E_CUDA, "cudaEventCreate failed");
  float best_ms = 0.f;
  int best_tile = -1, rc = CRESS_OK;
  for (int t = 0; t < CRESS_NTILES; ++t) {
    cfg.tile = t;
    if (ms) ms[t] = -1.f;
    rc = small_steps(nsstp, dts);   // warm-up; a shape the grid cannot use is skipped
    if (rc == CRESS_E_UNSUPPORTED) { rc = CRESS_OK; continue; }
    if (rc) break;
    cudaEventRecord(e0, stream);
    for (int r = 0; r < reps && !rc; ++r) rc = small_steps(nsstp, dts);
    cudaEventRecord(e1, stream);
    if (rc) break;
    if ((rc = cuda_check(cudaEventSynchronize(e1), "autotune sync"))) break;
    if ((rc = check_device_error())) break;
    float t_ms = 0.f;
    cudaEventElapsedTime(&t_ms, e0, e1);
    t_ms /= (float)(reps * nsstp);
    if (ms) ms[t] = t_ms;
    if (best_tile < 0 || t_ms < best_ms) { best_ms = t_ms; best_tile = t; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc || best_tile < 0) {
    cfg.tile = keep;
    return rc ? rc : set_error(CRESS_E_UNSUPPORTED, "cress_autotune: no tile shape fits this grid");
  }
  cfg.tile = best_tile;
  free_graphs();
  if (best) *best = best_tile;
  return CRESS_OK;
}

// An ensemble of independent domains on one device and one stream: every
// member runs its own large step, except that the acoustic substeps of all
// members run as one launch per substep (k_hevi2_batch over every
// member's tiles), so small domains fill the GPU together.
// An ensemble step runs each member's work before and after the acoustic
// substeps on the member's own stream (members overlap), and the substeps of
// all members as one launch per substep on the ensemble's stream, joined to
// the members' streams by events.  With graphs on, a step whose pointer
// states and parameters were seen before replays one CUDA graph that holds
// all of it (member streams forked from and joined back to the ensemble's).
struct Ensemble {
  std::vector<Ctx*> members;
  cudaStream_t stream = nullptr;      // the ensemble's own stream
  int device = 0;
  cudaEvent_t fork = nullptr, done = nullptr;
  std::vector<cudaEvent_t> ev;        // one per member
  HeviJob* jobs_d = nullptr;          // eager steps: nsstp x members jobs
  HeviJob* jobs_h = nullptr;          // pinned staging
  size_t cap = 0;
  cudaEvent_t staged = nullptr;       // the last copy out of jobs_h has completed
  long long launches = 0;
  bool graphs = true;
  int tile = 0;                       // the batched acoustic kernel: tile 0's or tile 13's
  struct Rec {
    cudaGraphExec_t exec = nullptr;
    HeviJob* jobs_d = nullptr;        // this graph's job table and its pinned source
    HeviJob* jobs_h = nullptr;
    long long nlaunch = 0;
    std::vector<long long> member_launches;
    std::vector<std::vector<float*>> post;
  };
  std::map<std::string, Rec> grec;
  std::map<std::string, int> gseen;
  void free_graphs() {
    for (auto& kv : grec) {
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
      if (kv.second.jobs_d) cudaFree(kv.second.jobs_d);
      if (kv.second.jobs_h) cudaFreeHost(kv.second.jobs_h);
    }
    grec.clear();
    gseen.clear();
  }
  ~Ensemble() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    free_graphs();
    if (staged) { cudaEventSynchronize(staged); cudaEventDestroy(staged); }
    for (cudaEvent_t x : ev) cudaEventDestroy(x);
    if (fork) cudaEventDestroy(fork);
    if (done) cudaEventDestroy(done);
    if (jobs_d) cudaFree(jobs_d);
    if (jobs_h) cudaFreeHost(jobs_h);
    if (stream) cudaStreamDestroy(stream);
  }
  int large_step(long long ctime, float dtb, int nsstp, float dts, HeviJob* jd, HeviJob* jh, bool eager);
  int step(long long ctime, float dtb, int nsstp, float dts);
  int set_tile(int t);
  int batch(const HeviJob* jd, int nblocks, int nk_max) {
    const cress_cfg& c0 = members[0]->cfg;
    const int n = (int)members.size();
    return tile == 13 ? launch_hevi4_batch(jd, n, nblocks, nk_max, c0.divopt, c0.sthopt != 0, c0.buyopt == 1, stream)
                      : launch_hevi_batch(jd, n, nblocks, nk_max, c0.divopt, c0.sthopt != 0, c0.buyopt == 1, stream);
  }
  int jobs_for(int nsstp, float dts, HeviJob* jh, int* nblocks, int* nk_max);
  int autotune(int nsstp, float dts, int reps, int* best, float* ms);
};

// One ensemble step issued on the streams (eager, or inside a capture that
// began on `stream`).  jd/jh: job table on the device and its pinned source.
int Ensemble::large_step(long long ctime, float dtb, int nsstp, float dts, HeviJob* jd, HeviJob* jh,
                         bool eager) {
  const bool filter = ctime != 0;
  const int n = (int)members.size();
  int rc;
  cudaEventRecord(fork, stream);
  for (int m = 0; m < n; ++m) {
    Ctx* c = members[m];
    cudaStreamWaitEvent(c->stream, fork, 0);
    if ((rc = c->large_step(filter, dtb, nsstp, dts, 1))) return rc;
  }
  const size_t need = (size_t)nsstp * n;
  if (eager) cudaEventSynchronize(staged);   // the previous step's copy has left the staging buffer
  int nblocks = 0, nk_max = 0;
  if ((rc = jobs_for(nsstp, dts, jh, &nblocks, &nk_max))) return rc;
  for (int m = 0; m < n; ++m) {
    cudaEventRecord(ev[m], members[m]->stream);
    cudaStreamWaitEvent(stream, ev[m], 0);
  }
  if ((rc = cuda_check(cudaMemcpyAsync(jd, jh, sizeof(HeviJob) * need, cudaMemcpyHostToDevice, stream),
                       "copy ensemble jobs")))
    return rc;
  if (eager) cudaEventRecord(staged, stream);
  for (int st = 0; st < nsstp; ++st) {
    if ((rc = batch(jd + (size_t)st * n, nblocks, nk_max)))
      return set_error(rc, "ensemble small-step launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    ++launches;
  }
  cudaEventRecord(done, stream);
  for (int m = 0; m < n; ++m) {
    Ctx* c = members[m];
    cudaStreamWaitEvent(c->stream, done, 0);
    if ((rc = c->large_step(filter, dtb, nsstp, dts, 2))) return rc;
  }
  for (int m = 0; m < n; ++m) {   // join: the ensemble's stream follows every member
    cudaEventRecord(ev[m], members[m]->stream);
    cudaStreamWaitEvent(stream, ev[m], 0);
  }
  return CRESS_OK;
}

// The acoustic jobs of one large step: nsstp x members HeviJobs in jh
// (substep-major, members in block order), the blocks of one launch and
// the deepest member.
int Ensemble::jobs_for(int nsstp, float dts, HeviJob* jh, int* nblocks, int* nk_max) {
  const int n = (int)members.size();
  int rc;
  *nblocks = 0;
  *nk_max = 0;
  for (int m = 0; m < n; ++m) {
    std::vector<HeviJob> per;
    if ((rc = members[m]->small_steps(nsstp, dts, &per))) return rc;
    *nk_max = std::max(*nk_max, members[m]->g.nk);
    int tx, ty;
    hevi_job_tiles(members[m]->g, &tx, &ty);
    for (int st = 0; st < nsstp; ++st) {
      HeviJob& j = jh[(size_t)st * n + m];
      j = per[st];
      j.first_block = *nblocks;
      j.tiles_x = tx;
    }
    *nblocks += tx * ty;
  }
  return CRESS_OK;
}

// Tile 13 holds each column's eliminated right-hand sides on chip, so every
// member needs nk <= kHevi3MaxNk.
int Ensemble::set_tile(int t) {
  if (t != 0 && t != 13) return set_error(CRESS_E_ARG, "ensemble tile %d (0 or 13)", t);
  if (t == 13)
    for (Ctx* c : members)
      if (c->g.nk > kHevi3MaxNk || c->g.nk < 8)
        return set_error(CRESS_E_UNSUPPORTED, "ensemble tile 13 needs 8 <= nk <= %d", kHevi3MaxNk);
  cudaStreamSynchronize(stream);
  free_graphs();
  for (Ctx* c : members) {
    cudaStreamSynchronize(c->stream);
    c->free_graphs();
    c->cfg.tile = t;
  }
  tile = t;
  return CRESS_OK;
}

// Time the batched substep with each tile on the members' present forcing
// (the future levels are overwritten, the present and past are not) and
// keep the faster.  ms[0], ms[1]: tile 0, tile 13 (-1: not usable).
int Ensemble::autotune(int nsstp, float dts, int reps, int* best, float* ms) {
  if (nsstp < 1 || reps < 1) return set_error(CRESS_E_ARG, "cress_ensemble_autotune: nsstp=%d reps=%d", nsstp, reps);
  const int n = (int)members.size(), keep = tile;
  const size_t need = (size_t)nsstp * n;
  HeviJob* jd = nullptr;
  HeviJob* jh = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = CRESS_OK, best_t = -1;
  float best_ms = 0.f;
  if (cudaMalloc(&jd, sizeof(HeviJob) * need) != cudaSuccess ||
      cudaMallocHost(&jh, sizeof(HeviJob) * need) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess)
    rc = set_error(CRESS_E_CUDA, "cress_ensemble_autotune: allocation failed");
  const int cand[2] = {0, 13};
  for (int q = 0; q < 2 && !rc; ++q) {
    if (ms) ms[q] = -1.f;
    if (set_tile(cand[q]) != CRESS_OK) continue;   // tile 13 needs nk <= kHevi3MaxNk
    int nblocks = 0, nk_max = 0;
    if ((rc = jobs_for(nsstp, dts, jh, &nblocks, &nk_max))) break;
    if ((rc = cuda_check(cudaMemcpyAsync(jd, jh, sizeof(HeviJob) * need, cudaMemcpyHostToDevice, stream),
                         "copy ensemble jobs")))
      break;
    for (int st = 0; st < nsstp && !rc; ++st) rc = batch(jd + (size_t)st * n, nblocks, nk_max);   // warm-up
    cudaEventRecord(e0, stream);
    for (int r = 0; r < reps && !rc; ++r)
      for (int st = 0; st < nsstp && !rc; ++st) rc = batch(jd + (size_t)st * n, nblocks, nk_max);
    cudaEventRecord(e1, stream);
    if (rc == CRESS_E_UNSUPPORTED) { rc = CRESS_OK; continue; }
    if (rc || (rc = cuda_check(cudaEventSynchronize(e1), "ensemble autotune sync"))) break;
    for (Ctx* c : members)
      if ((rc = c->check_device_error())) break;
    if (rc) break;
    float t_ms = 0.f;
    cudaEventElapsedTime(&t_ms, e0, e1);
    t_ms /= (float)(reps * nsstp);
    if (ms) ms[q] = t_ms;
    if (best_t < 0 || t_ms < best_ms) { best_ms = t_ms; best_t = cand[q]; }
  }
  cudaStreamSynchronize(stream);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (jd) cudaFree(jd);
  if (jh) cudaFreeHost(jh);
  if (rc || best_t < 0) {
    set_tile(keep);
    return rc ? rc : set_error(CRESS_E_UNSUPPORTED, "cress_ensemble_autotune: no batched tile fits");
  }
  if (best) *best = best_t;
  return set_tile(best_t);
}

int Ensemble::step(long long ctime, float dtb, int nsstp, float dts) {
  const int n = (int)members.size();
  const size_t need = (size_t)nsstp * n;
  auto eager = [&]() -> int {
    if (need > cap) {
      cudaEventSynchronize(staged);
      if (jobs_d) cudaFree(jobs_d);
      if (jobs_h) cudaFreeHost(jobs_h);
      jobs_d = nullptr;
      jobs_h = nullptr;
      cap = 0;
      int rc;
      if ((rc = cuda_check(cudaMalloc(&jobs_d, sizeof(HeviJob) * need), "cudaMalloc ensemble jobs")) ||
          (rc = cuda_check(cudaMallocHost(&jobs_h, sizeof(HeviJob) * need), "cudaMallocHost ensemble jobs")))
        return rc;
      cap = need;
    }
    return large_step(ctime, dtb, nsstp, dts, jobs_d, jobs_h, true);
  };
  bool sampling = false;
  for (Ctx* c : members) sampling |= c->sampler != nullptr;
  if (!graphs || sampling) return eager();
  std::string key;
  for (Ctx* c : members) {
    const std::vector<float*> ps = c->pointer_state();
    key.append(reinterpret_cast<const char*>(ps.data()), ps.size() * sizeof(float*));
    const struct { float resid; const void* mlp; int chunk; } q{c->resid_tol, c->mlp, c->lb.chunk};
    key.append(reinterpret_cast<const char*>(&q), sizeof q);
  }
  const struct { long long filter; int nsstp; float dtb, dts; } p{ctime != 0 ? 1 : 0, nsstp, dtb, dts};
  key.append(reinterpret_cast<const char*>(&p), sizeof p);
  auto it = grec.find(key);
  if (it == grec.end()) {
    if (gseen[key]++ == 0) return eager();
    std::vector<std::vector<float*>> pre;
    std::vector<long long> l0;
    for (Ctx* c : members) { pre.push_back(c->pointer_state()); l0.push_back(c->launches); }
    const long long e0 = launches;
    Rec r;
    if (cudaMalloc(&r.jobs_d, sizeof(HeviJob) * need) != cudaSuccess ||
        cudaMallocHost(&r.jobs_h, sizeof(HeviJob) * need) != cudaSuccess) {
      cudaGetLastError();
      if (r.jobs_d) cudaFree(r.jobs_d);
      graphs = false;
      return eager();
    }
    cudaGraph_t graph = nullptr;
    int rc = CRESS_E_CUDA;
    if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      rc = large_step(ctime, dtb, nsstp, dts, r.jobs_d, r.jobs_h, false);
      const cudaError_t e = cudaStreamEndCapture(stream, &graph);
      if (!rc && (e != cudaSuccess || cudaGraphInstantiate(&r.exec, graph, 0) != cudaSuccess)) rc = CRESS_E_CUDA;
    }
    if (graph) cudaGraphDestroy(graph);
    for (int m = 0; m < n; ++m) {
      r.member_launches.push_back(members[m]->launches - l0[m]);
      members[m]->launches = l0[m];
      r.post.push_back(members[m]->pointer_state());
      members[m]->set_pointer_state(pre[m]);
    }
    r.nlaunch = launches - e0;
    launches = e0;
    if (rc) {   // nothing ran: run eagerly from the same state
      cudaGetLastError();
      if (r.exec) cudaGraphExecDestroy(r.exec);
      cudaFree(r.jobs_d);
      cudaFreeHost(r.jobs_h);
      graphs = false;
      return eager();
    }
    it = grec.emplace(key, std::move(r)).first;
  }
  // the graph starts after each member's queued work and its end orders
  // each member's later work
  for (int m = 0; m < n; ++m) {
    cudaEventRecord(ev[m], members[m]->stream);
    cudaStreamWaitEvent(stream, ev[m], 0);
  }
  if (cudaGraphLaunch(it->second.exec, stream) != cudaSuccess)
    return set_error(CRESS_E_CUDA, "cudaGraphLaunch: %s", cudaGetErrorString(cudaGetLastError()));
  cudaEventRecord(done, stream);
  launches += it->second.nlaunch;
  for (int m = 0; m < n; ++m) {
    Ctx* c = members[m];
    cudaStreamWaitEvent(c->stream, done, 0);
    c->launches += it->second.member_launches[m];
    c->set_pointer_state(it->second.post[m]);
  }
  return CRESS_OK;
}

}  // namespace cress

using namespace cress;

extern "C" {

const char* cress_last_error(void) { return g_last_error.c_str(); }
int cress_abi_version(void) { return 5; }

int cress_create(const cress_cfg* cfg, int device, cress_ctx** out) {
  if (!cfg || !out) return set_error(CRESS_E_ARG, "cress_create: null argument");
  *out = nullptr;
  if (cfg->ni < 8 || cfg->nj < 8 || cfg->nk < 8)
    return set_error(CRESS_E_ARG, "cress_create: dims too small (%d,%d,%d)", cfg->ni, cfg->nj, cfg->nk);
  if ((cfg->impopt != 0 && cfg->impopt != 1) || cfg->gwmopt != 0)
    return set_error(CRESS_E_UNSUPPORTED, "only impopt=0 (HE-VE) or 1 (HE-VI), gwmopt=0 run on the GPU");
  const bool periodic = cfg->wbc == -1 && cfg->ebc == -1 && cfg->sbc == -1 && cfg->nbc == -1;
  const bool openx = cfg->wbc == cfg->ebc && (cfg->wbc == 4 || cfg->wbc == 5 || cfg->wbc == 7) &&
                     cfg->sbc == -1 && cfg->nbc == -1;
  if (!periodic && !openx)
    return set_error(CRESS_E_UNSUPPORTED,
                     "lateral boundaries: periodic (-1) on all sides, or open x (wbc = ebc = 4, 5 or 7) with periodic y");
  if (openx && (cfg->impopt != 1 || cfg->tubopt != 0 || cfg->advopt != 2))
    return set_error(CRESS_E_UNSUPPORTED, "open x boundaries run with impopt=1, tubopt=0, advopt=2");
  if (cfg->bbc != 2 || cfg->tbc != 2)
    return set_error(CRESS_E_UNSUPPORTED, "only rigid bottom/top (bbc=tbc=2) run on the GPU");
  if (cfg->dx <= 0.f || cfg->dy <= 0.f || cfg->dz <= 0.f)
    return set_error(CRESS_E_ARG, "cress_create: non-positive grid spacing");
  int rc = cuda_check(cudaSetDevice(device), "cudaSetDevice");
  if (rc) return rc;
  Ctx* c = new Ctx();
  c->device = device;
  c->cfg = *cfg;
  c->g = make_grid(cfg->ni, cfg->nj, cfg->nk);
  c->g.openx = openx ? 1 : 0;
  if ((rc = cuda_check(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate"))) {
    delete c;
    return rc;
  }
  c->own_stream = c->stream;
  for (int f = 0; f < CRESS_NFIELD; ++f) {
    for (int l = 0; l < 4; ++l) c->lev[f][l] = nullptr;
    c->spare[f] = nullptr;
  }
  const int dyn[4] = {CRESS_U, CRESS_V, CRESS_W, CRESS_PP};
  for (int f : dyn) {
    for (int l = 0; l < 4; ++l) c->lev[f][l] = c->alloc_field();
    c->spare[f] = c->alloc_field();
    for (int l = 0; l < 4; ++l)
      if (!c->lev[f][l]) { delete c; return set_error(CRESS_E_CUDA, "cudaMalloc of the state failed"); }
    if (!c->spare[f]) { delete c; return set_error(CRESS_E_CUDA, "cudaMalloc of the state failed"); }
  }
  // theta' has three time levels (its forcing goes straight into s_steps)
  for (int l = 0; l < 3; ++l) {
    c->lev[CRESS_PTP][l] = c->alloc_field();
    if (!c->lev[CRESS_PTP][l]) { delete c; return set_error(CRESS_E_CUDA, "cudaMalloc of the state failed"); }
  }
  if (cfg->cphopt == 3) {
    // moist species: three time levels each (their forcings go straight
    // into s_steps), plus the surface precipitation planes and the
    // sedimentation minimum word
    for (int f = CRESS_QV; f <= CRESS_NG; ++f)
      for (int l = 0; l < 3; ++l) {
        c->lev[f][l] = c->alloc_field();
        if (!c->lev[f][l]) { delete c; return set_error(CRESS_E_CUDA, "cudaMalloc of the moist state failed"); }
      }
    const size_t pb = sizeof(float) * 10 * (size_t)c->g.px * c->g.py;
    if ((rc = cuda_check(cudaMalloc(&c->prec_d, pb), "cudaMalloc precip")) ||
        (rc = cuda_check(cudaMalloc(&c->dtp_d, sizeof(int)), "cudaMalloc dtp"))) {
      delete c;
      return rc;
    }
    c->owned.push_back(c->prec_d);
    c->owned.push_back(c->dtp_d);
    cudaMemsetAsync(c->prec_d, 0, pb, c->stream);
    // fall speeds of the 8 sedimenting quantities (written by the process
    // rates, read by the column sedimentation)
    const size_t ub = sizeof(float) * 8 * (size_t)c->g.plane * c->g.nk;
    if ((rc = cuda_check(cudaMalloc(&c->uspd_d, ub), "cudaMalloc fall speeds"))) {
      delete c;
      return rc;
    }
    c->owned.push_back(c->uspd_d);
    cudaMemsetAsync(c->uspd_d, 0, ub, c->stream);
    if ((rc = micro_init_tables())) { delete c; return set_error(rc, "Koenig table upload failed"); }
  } else if (cfg->cphopt != 0) {
    delete c;
    return set_error(CRESS_E_UNSUPPORTED, "cphopt=%d: only 0 (dry) and 3 (cold rain) run on the GPU", cfg->cphopt);
  }
  if (cfg->tubopt == 1 || cfg->tubopt == 2) {
    c->rkv_d = c->alloc_field();   // eddy viscosity
    if (!c->rkv_d) { delete c; return set_error(CRESS_E_CUDA, "cudaMalloc of the eddy viscosity failed"); }
  } else if (cfg->tubopt != 0) {
    delete c;
    return set_error(CRESS_E_UNSUPPORTED, "tubopt=%d: 0, 1 (Smagorinsky) and 2 (TKE) run on the GPU", cfg->tubopt);
  }
  if (cfg->tubopt == 2) {
    // the TKE (three time levels, its forcing goes straight into s_steps)
    // and the per-point fields of the closure
    for (int l = 0; l < 3; ++l) c->lev[CRESS_TKE][l] = c->alloc_field();
    c->rks_d = c->alloc_field();
    c->nsq_d = c->alloc_field();
    c->shr_d = c->alloc_field();
    c->dsp_d = c->alloc_field();
    bool ok = c->rks_d && c->nsq_d && c->shr_d && c->dsp_d;
    for (int l = 0; l < 3; ++l) ok = ok && c->lev[CRESS_TKE][l];
    if (!ok) { delete c; return set_error(CRESS_E_CUDA, "cudaMalloc of the TKE fields failed"); }
  }
  c->col_h.assign((size_t)C_NFIELDS_ALL * (cfg->nk + 1), 0.f);
  if ((rc = cuda_check(cudaMalloc(&c->col_d, sizeof(float) * c->col_h.size()), "cudaMalloc cols"))) {
    delete c;
    return rc;
  }
  c->owned.push_back(c->col_d);
  if ((rc = cuda_check(cudaMalloc(&c->err_d, sizeof(int)), "cudaMalloc error word"))) {
    delete c;
    return rc;
  }
  c->owned.push_back(c->err_d);
  cudaMemsetAsync(c->err_d, 0, sizeof(int), c->stream);
  if (openx) {   // phase speeds, zero until the first large step ends (a fresh start)
    const size_t rb = sizeof(float) * rad_floats(c->g);
    if ((rc = cuda_check(cudaMalloc(&c->rad_d, rb), "cudaMalloc phase speeds"))) {
      delete c;
      return rc;
    }
    c->owned.push_back(c->rad_d);
    cudaMemsetAsync(c->rad_d, 0, rb, c->stream);
  }
  if (cfg->impopt == 0) {   // HE-VE side buffers (two planes each)
    for (int b = 0; b < 2; ++b) {
      if ((rc = cuda_check(cudaMalloc(&c->wcside[b], sizeof(float) * 2 * c->g.plane), "cudaMalloc wc planes"))) {
        delete c;
        return rc;
      }
      c->owned.push_back(c->wcside[b]);
      cudaMemsetAsync(c->wcside[b], 0, sizeof(float) * 2 * c->g.plane, c->stream);
    }
  }
  *out = reinterpret_cast<cress_ctx*>(c);
  return CRESS_OK;
}

void cress_destroy(cress_ctx* ctx) { delete reinterpret_cast<Ctx*>(ctx); }

int cress_set_stream(cress_ctx* ctx, void* stream) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "null context");
  cudaSetDevice(c->device);
  c->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : c->own_stream;
  return CRESS_OK;
}

int cress_set_spin_limit(cress_ctx* ctx, int probes) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "null context");
  c->spin_limit = probes < 0 ? kSpinLimit : (uint32_t)probes;
  c->free_graphs();   // captured steps carry the old limit
  return CRESS_OK;
}

int cress_sync(cress_ctx* ctx) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "null context");
  cudaSetDevice(c->device);
  int rc = cuda_check(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  return rc ? rc : c->check_device_error();
}

int cress_set_base3d(cress_ctx* ctx, const float* const* b3) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !b3) return set_error(CRESS_E_ARG, "cress_set_base3d: null argument");
  for (int n = 0; n < CRESS_B_N; ++n)
    if (!b3[n]) return set_error(CRESS_E_ARG, "cress_set_base3d: array %d is null", n);
  cudaSetDevice(c->device);
  const int ni = c->cfg.ni, nj = c->cfg.nj, nk = c->cfg.nk;
  // The columns are taken at the domain centre; every point the small step
  // reads (i in 1..ni, j in 1..nj) must carry the same value.
  const NonUniform bad = base_columns(b3, ni, nj, nk, c->col_h.data());
  if (bad.n >= 0)
    return set_error(CRESS_E_NONUNIFORM, "base array %d varies horizontally at (%d,%d,%d): %g vs %g", bad.n,
                     bad.i, bad.j, bad.k, (double)bad.x, (double)bad.v);
  int rc = cuda_check(cudaMemcpyAsync(c->col_d, c->col_h.data(), sizeof(float) * c->col_h.size(),
                                      cudaMemcpyHostToDevice, c->stream),
                      "copy base columns");
  if (rc) return rc;
  rc = cuda_check(cudaStreamSynchronize(c->stream), "sync base columns");
  if (rc) return rc;
  c->thomas.clear();
  c->base_set = true;
  return CRESS_OK;
}

int cress_put_field(cress_ctx* ctx, int field, int level, const float* host) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !host) return set_error(CRESS_E_ARG, "cress_put_field: null argument");
  if (field < 0 || field >= CRESS_NFIELD || level < 0 || level > 3 || !c->lev[field][level])
    return set_error(CRESS_E_ARG, "cress_put_field: field %d level %d not held", field, level);
  cudaSetDevice(c->device);
  return c->put_host(c->lev[field][level], host);
}

int cress_get_field(cress_ctx* ctx, int field, int level, float* host) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !host) return set_error(CRESS_E_ARG, "cress_get_field: null argument");
  if (field < 0 || field >= CRESS_NFIELD || level < 0 || level > 3 || !c->lev[field][level])
    return set_error(CRESS_E_ARG, "cress_get_field: field %d level %d not held", field, level);
  cudaSetDevice(c->device);
  int rc = c->get_host(host, c->lev[field][level]);
  if (rc) return rc;
  rc = cuda_check(cudaStreamSynchronize(c->stream), "sync after device->host copy");
  return rc ? rc : c->check_device_error();
}

int cress_get_fields_async(cress_ctx* ctx, int level, int nfield, const int* fields, float* const* host) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !fields || !host || nfield < 1 || nfield > CRESS_NFIELD)
    return set_error(CRESS_E_ARG, "cress_get_fields_async: bad argument");
  if (level < 0 || level > 3) return set_error(CRESS_E_ARG, "cress_get_fields_async: level %d", level);
  for (int q = 0; q < nfield; ++q)
    if (fields[q] < 0 || fields[q] >= CRESS_NFIELD || !c->lev[fields[q]][level] || !host[q])
      return set_error(CRESS_E_ARG, "cress_get_fields_async: field %d not held or null buffer", fields[q]);
  cudaSetDevice(c->device);
  return c->get_async(level, nfield, fields, host);
}

int cress_put_fields_async(cress_ctx* ctx, int level, int nfield, const int* fields, const float* const* host) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !fields || !host || nfield < 1 || nfield > CRESS_NFIELD)
    return set_error(CRESS_E_ARG, "cress_put_fields_async: bad argument");
  if (level < 0 || level > 3) return set_error(CRESS_E_ARG, "cress_put_fields_async: level %d", level);
  for (int q = 0; q < nfield; ++q) {
    if (fields[q] < 0 || fields[q] >= CRESS_NFIELD || !c->lev[fields[q]][level] || !host[q])
      return set_error(CRESS_E_ARG, "cress_put_fields_async: field %d not held or null buffer", fields[q]);
    for (int r = 0; r < q; ++r)
      if (fields[r] == fields[q]) return set_error(CRESS_E_ARG, "cress_put_fields_async: field %d twice", fields[q]);
  }
  cudaSetDevice(c->device);
  return c->put_async(level, nfield, fields, host);
}

int cress_wait_fields(cress_ctx* ctx) {
  return cress_wait_fields_to(ctx, 0);
}

int cress_wait_fields_to(cress_ctx* ctx, int in_flight) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "null context");
  if (in_flight < 0 || in_flight > 1) return set_error(CRESS_E_ARG, "cress_wait_fields_to: in_flight %d (0 or 1)", in_flight);
  cudaSetDevice(c->device);
  return c->wait_async(in_flight);
}

int cress_small_steps(cress_ctx* ctx, int nsstp, float dts) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "null context");
  cudaSetDevice(c->device);
  return c->small_steps(nsstp, dts);
}

int cress_smalldrv(cress_ctx* ctx, int nsstp, float dts, const float* up, const float* vp,
                   const float* wp, const float* ppp, const float* ufrc, const float* vfrc,
                   const float* wfrc, const float* pfrc, float* uf, float* vf, float* wf,
                   float* ppf) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "null context");
  const float* in[8] = {up, vp, wp, ppp, ufrc, vfrc, wfrc, pfrc};
  float* out[4] = {uf, vf, wf, ppf};
  for (auto p : in) if (!p) return set_error(CRESS_E_ARG, "cress_smalldrv: null input");
  for (auto p : out) if (!p) return set_error(CRESS_E_ARG, "cress_smalldrv: null output");
  cudaSetDevice(c->device);
  const int F[4] = {CRESS_U, CRESS_V, CRESS_W, CRESS_PP};
  int rc;
  for (int n = 0; n < 4; ++n) {
    if ((rc = c->put_host(c->lev[F[n]][CRESS_PAST], in[n]))) return rc;
    if ((rc = c->put_host(c->lev[F[n]][CRESS_FORCING], in[4 + n]))) return rc;
  }
  if ((rc = c->small_steps(nsstp, dts))) return rc;
  for (int n = 0; n < 4; ++n)
    if ((rc = c->get_host(out[n], c->lev[F[n]][CRESS_FUTURE]))) return rc;
  rc = cuda_check(cudaStreamSynchronize(c->stream), "cress_smalldrv sync");
  return rc ? rc : c->check_device_error();
}

int cress_set_base_large(cress_ctx* ctx, const float* ubr, const float* vbr, const float* rbct,
                         int ksp0) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !ubr || !vbr || !rbct) return set_error(CRESS_E_ARG, "cress_set_base_large: null argument");
  cudaSetDevice(c->device);
  const int ni = c->cfg.ni, nj = c->cfg.nj, nk = c->cfg.nk;
  if (ksp0 < 2 || ksp0 > nk) return set_error(CRESS_E_ARG, "cress_set_base_large: ksp0=%d", ksp0);
  auto at = [&](const float* a, int i, int j, int k) {
    return a[(size_t)i + (size_t)(ni + 2) * ((size_t)j + (size_t)(nj + 2) * (size_t)(k - 1))];
  };
  const float* src[3] = {ubr, vbr, rbct};
  const int dst[3] = {C_UBR, C_VBR, C_RBCT};
  const int ic = ni / 2, jc = nj / 2;
  for (int n = 0; n < 3; ++n)
    for (int k = 1; k <= nk; ++k) {
      const float v = at(src[n], ic, jc, k);
      c->col_h[(size_t)dst[n] * (nk + 1) + k] = v;
      for (int j = 1; j <= nj - 1; ++j)
        for (int i = 1; i <= ni - 1; ++i)
          if (at(src[n], i, j, k) != v)
            return set_error(CRESS_E_NONUNIFORM, "large-step base array %d varies horizontally at (%d,%d,%d)",
                             n, i, j, k);
    }
  c->ksp0 = ksp0;
  int rc = cuda_check(cudaMemcpyAsync(c->col_d, c->col_h.data(), sizeof(float) * c->col_h.size(),
                                      cudaMemcpyHostToDevice, c->stream),
                      "copy large-step columns");
  if (rc) return rc;
  rc = cuda_check(cudaStreamSynchronize(c->stream), "sync large-step columns");
  if (rc) return rc;
  c->large_set = true;
  return CRESS_OK;
}

int cress_set_base_moist(cress_ctx* ctx, const float* pbr, const float* qvbr) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !pbr || !qvbr) return set_error(CRESS_E_ARG, "cress_set_base_moist: null argument");
  cudaSetDevice(c->device);
  const int ni = c->cfg.ni, nj = c->cfg.nj, nk = c->cfg.nk;
  auto at = [&](const float* a, int i, int j, int k) {
    return a[(size_t)i + (size_t)(ni + 2) * ((size_t)j + (size_t)(nj + 2) * (size_t)(k - 1))];
  };
  const float* src[2] = {pbr, qvbr};
  const int dst[2] = {C_PBR, C_QVBR};
  for (int n = 0; n < 2; ++n)
    for (int k = 1; k <= nk; ++k) {
      const float v = at(src[n], ni / 2, nj / 2, k);
      c->col_h[(size_t)dst[n] * (nk + 1) + k] = v;
      for (int j = 1; j <= nj - 1; ++j)
        for (int i = 1; i <= ni - 1; ++i)
          if (at(src[n], i, j, k) != v)
            return set_error(CRESS_E_NONUNIFORM, "moist base array %d varies horizontally at (%d,%d,%d)", n, i, j, k);
    }
  int rc = cuda_check(cudaMemcpyAsync(c->col_d, c->col_h.data(), sizeof(float) * c->col_h.size(),
                                      cudaMemcpyHostToDevice, c->stream), "copy moist columns");
  if (rc) return rc;
  if ((rc = cuda_check(cudaStreamSynchronize(c->stream), "sync moist columns"))) return rc;
  c->moist_set = true;
  return CRESS_OK;
}

int cress_cloudphy(cress_ctx* ctx, float dtb, float thresq) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "null context");
  cudaSetDevice(c->device);
  return c->cloudphy(dtb, thresq);
}

int cress_satadjst(cress_ctx* ctx, int level, float thresq) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "null context");
  if (level != CRESS_NOW && level != CRESS_FUTURE) return set_error(CRESS_E_ARG, "cress_satadjst: level %d", level);
  cudaSetDevice(c->device);
  return c->satadjst(level, thresq);
}

int cress_get_precip(cress_ctx* ctx, float* host) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !host) return set_error(CRESS_E_ARG, "cress_get_precip: null argument");
  if (!c->prec_d) return set_error(CRESS_E_STATE, "cress_get_precip: context has no microphysics");
  cudaSetDevice(c->device);
  const size_t wb = sizeof(float) * (c->g.ni + 2);
  int rc = cuda_check(cudaMemcpy2DAsync(host, wb, c->prec_d, sizeof(float) * c->g.px, wb,
                                        (size_t)10 * c->g.py, cudaMemcpyDeviceToHost, c->stream), "precip copy");
  if (rc) return rc;
  return cuda_check(cudaStreamSynchronize(c->stream), "precip sync");
}

int cress_put_precip(cress_ctx* ctx, const float* host) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !host) return set_error(CRESS_E_ARG, "cress_put_precip: null argument");
  if (!c->prec_d) return set_error(CRESS_E_STATE, "cress_put_precip: context has no microphysics");
  cudaSetDevice(c->device);
  const size_t wb = sizeof(float) * (c->g.ni + 2);
  int rc = cuda_check(cudaMemcpy2DAsync(c->prec_d, sizeof(float) * c->g.px, host, wb, wb,
                                        (size_t)10 * c->g.py, cudaMemcpyHostToDevice, c->stream), "precip copy");
  if (rc) return rc;
  return cuda_check(cudaStreamSynchronize(c->stream), "precip sync");
}

// The phase speeds of one variable: device rows (nj+2 floats, j = 0..nj+1)
// of levels k = 0..nk per side, host ucpx(1:nj,1:nk,1:2).
static int phase_copy(Ctx* c, int field, float* host, const float* src_host, bool get) {
  if (!c->rad_d) return set_error(CRESS_E_STATE, "phase speeds: the context has periodic x boundaries");
  if (field < 0 || field >= RAD_N) return set_error(CRESS_E_ARG, "phase speeds: field %d", field);
  const Grid& g = c->g;
  const size_t hw = sizeof(float) * (size_t)g.nj, dp = sizeof(float) * (size_t)(g.nj + 2);
  int rc = CRESS_OK;
  for (int side = 0; side < 2 && !rc; ++side) {
    float* dev = c->rad_d + rad_at(g, field, side, 1, 1);
    const size_t hoff = (size_t)side * g.nj * g.nk;
    rc = get ? cuda_check(cudaMemcpy2DAsync(host + hoff, hw, dev, dp, hw, (size_t)g.nk, cudaMemcpyDeviceToHost,
                                            c->stream), "phase copy")
             : cuda_check(cudaMemcpy2DAsync(dev, dp, src_host + hoff, hw, hw, (size_t)g.nk, cudaMemcpyHostToDevice,
                                            c->stream), "phase copy");
  }
  if (rc) return rc;
  return cuda_check(cudaStreamSynchronize(c->stream), "phase sync");
}

int cress_get_phase(cress_ctx* ctx, int field, float* host) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !host) return set_error(CRESS_E_ARG, "cress_get_phase: null argument");
  cudaSetDevice(c->device);
  return phase_copy(c, field, host, nullptr, true);
}

int cress_put_phase(cress_ctx* ctx, int field, const float* host) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !host) return set_error(CRESS_E_ARG, "cress_put_phase: null argument");
  cudaSetDevice(c->device);
  return phase_copy(c, field, nullptr, host, false);
}

int cress_large_step(cress_ctx* ctx, long long ctime, float dtb, int nsstp, float dts) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "null context");
  cudaSetDevice(c->device);
  return c->step(ctime != 0, dtb, nsstp, dts);
}

long long cress_launch_count(const cress_ctx* ctx) {
  const Ctx* c = reinterpret_cast<const Ctx*>(ctx);
  return c ? c->launches : -1;
}

// Learned microphysics: MLP in place of the process rates of s_coldblk.
int cress_set_learned_micro(cress_ctx* ctx, cress_mlp* mh, int chunk, float resid_tol) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "null context");
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  c->free_graphs();   // captured steps refer to the old buffers
  c->free_learned();
  if (!mh) return CRESS_OK;
  Mlp* m = reinterpret_cast<Mlp*>(mh);
  if (c->cfg.cphopt != 3) return set_error(CRESS_E_STATE, "cress_set_learned_micro: context is not cphopt=3");
  if (c->g.openx)   // the learned kernels cover the interior columns only
    return set_error(CRESS_E_UNSUPPORTED, "cress_set_learned_micro: open x boundaries run the plain scheme");
  if (m->device != c->device) return set_error(CRESS_E_ARG, "MLP and context live on different devices");
  if (!(resid_tol > 0.f)) return set_error(CRESS_E_ARG, "resid_tol must be positive");
  // chunk 0: the fused kernel over all cells (the fallback list can hold
  // every cell); chunk > 0: chunks of that many cells through the GEMMs
  const bool fused = chunk <= 0;
  const long long ncell = (long long)(c->g.ni - 3) * (c->g.nj - 3) * (c->g.nk - 1);
  if (fused) {
    if (ncell > 0x7FFFFFFFLL) return set_error(CRESS_E_ARG, "domain too large for the fused learned form");
    chunk = (int)ncell;
  } else {
    chunk = (chunk + 127) / 128 * 128;
  }
  auto al = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    c->lb_owned.push_back(p);
    return p;
  };
  LearnedBuffers& L = c->lb;
  L.fused = fused;
  L.chunk = chunk;
  if (!fused) {
    L.xb = static_cast<__nv_bfloat16*>(al(sizeof(__nv_bfloat16) * (size_t)chunk * kMlpK1));
    L.h0 = static_cast<__nv_bfloat16*>(al(sizeof(__nv_bfloat16) * (size_t)chunk * kMlpH));
    L.h1 = static_cast<__nv_bfloat16*>(al(sizeof(__nv_bfloat16) * (size_t)chunk * kMlpH));
    L.y = static_cast<float*>(al(sizeof(float) * (size_t)chunk * kMlpN4));
    L.env = static_cast<unsigned char*>(al((size_t)chunk));
  }
  L.fb_list = static_cast<int*>(al(sizeof(int) * (size_t)chunk));
  L.fb_count = static_cast<int*>(al(sizeof(int)));
  L.stats = static_cast<unsigned long long*>(al(2 * sizeof(unsigned long long)));
  L.err = static_cast<int*>(al(sizeof(int)));
  if ((!fused && (!L.xb || !L.h0 || !L.h1 || !L.y || !L.env)) || !L.fb_list || !L.fb_count || !L.stats || !L.err) {
    c->free_learned();
    return set_error(CRESS_E_CUDA, "cudaMalloc of the learned-microphysics buffers failed");
  }
  cudaMemsetAsync(L.stats, 0, 2 * sizeof(unsigned long long), c->stream);
  cudaMemsetAsync(L.err, 0, sizeof(int), c->stream);
  c->mlp = m;
  c->resid_tol = resid_tol;
  return cuda_check(cudaStreamSynchronize(c->stream), "learned setup");
}

// Cells the MLP handled and cells sent to the plain scheme since the
// learned form was enabled; a bounded-wait failure inside the GEMMs is
// reported here as CRESS_E_TIMEOUT.
int cress_learned_stats(cress_ctx* ctx, long long* mlp_cells, long long* fallback_cells) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !mlp_cells || !fallback_cells) return set_error(CRESS_E_ARG, "null argument");
  if (!c->mlp) return set_error(CRESS_E_STATE, "learned microphysics is not enabled");
  cudaSetDevice(c->device);
  unsigned long long s[2] = {0, 0};
  int e = 0;
  cudaMemcpyAsync(s, c->lb.stats, sizeof(s), cudaMemcpyDeviceToHost, c->stream);
  cudaMemcpyAsync(&e, c->lb.err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  int rc = cuda_check(cudaStreamSynchronize(c->stream), "stats");
  if (rc) return rc;
  *mlp_cells = (long long)s[0];
  *fallback_cells = (long long)s[1];
  return e ? set_error(e, "a tensor-core GEMM of the learned form gave up waiting") : CRESS_OK;
}

// Sample (features, plain tendencies) tuples into the MLP's store on every
// following s_cloudphy, 1 cell in `stride` (cells without any tendency 1 in
// stride/keep_zero); NULL stops sampling.
int cress_set_tuple_sampling(cress_ctx* ctx, cress_mlp* mh, int stride, float keep_zero, unsigned long long seed) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "null context");
  c->sampler = nullptr;
  if (!mh) return CRESS_OK;
  Mlp* m = reinterpret_cast<Mlp*>(mh);
  if (c->cfg.cphopt != 3) return set_error(CRESS_E_STATE, "cress_set_tuple_sampling: context is not cphopt=3");
  if (m->device != c->device) return set_error(CRESS_E_ARG, "MLP and context live on different devices");
  if (stride < 1 || keep_zero < 0.f || keep_zero > 1.f) return set_error(CRESS_E_ARG, "bad stride / keep_zero");
  cudaSetDevice(c->device);
  if (!c->count_d) {
    if (cudaMalloc(&c->count_d, sizeof(unsigned long long)) != cudaSuccess)
      return set_error(CRESS_E_CUDA, "cudaMalloc failed");
    c->owned.push_back(c->count_d);
  }
  c->sampler = m;
  c->sample_stride = stride;
  c->sample_keep_zero = keep_zero;
  c->sample_seed = seed;
  return CRESS_OK;
}

// Replay whole large steps from CUDA graphs (on) or launch every kernel
// from the host (off, the default).
int cress_set_graphs(cress_ctx* ctx, int on) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "null context");
  if (on && c->slab) return set_error(CRESS_E_UNSUPPORTED, "cress_set_graphs: not for a y-slab rank");
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  c->free_graphs();
  c->graphs = on != 0;
  return CRESS_OK;
}

int cress_diagnostics(cress_ctx* ctx, int level, double* out) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !out) return set_error(CRESS_E_ARG, "cress_diagnostics: null argument");
  cudaSetDevice(c->device);
  return c->diagnostics(level, out);
}

int cress_autotune(cress_ctx* ctx, int nsstp, float dts, int reps, int* best_tile, float* ms_per_substep) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "cress_autotune: null context");
  if (!c->base_set) return set_error(CRESS_E_STATE, "cress_autotune: base state not set");
  cudaSetDevice(c->device);
  return c->autotune(nsstp, dts, reps, best_tile, ms_per_substep);
}

int cress_ensemble_create(cress_ctx* const* members, int n, cress_ensemble** out) {
  if (!members || n < 1 || !out) return set_error(CRESS_E_ARG, "cress_ensemble_create: bad arguments");
  *out = nullptr;
  Ctx* c0 = reinterpret_cast<Ctx*>(members[0]);
  for (int m = 0; m < n; ++m) {
    Ctx* c = reinterpret_cast<Ctx*>(members[m]);
    if (!c) return set_error(CRESS_E_ARG, "cress_ensemble_create: null member %d", m);
    if (c->device != c0->device) return set_error(CRESS_E_ARG, "ensemble members live on different devices");
    if (!c->base_set || !c->large_set) return set_error(CRESS_E_STATE, "member %d: base state not set", m);
    if (c->cfg.impopt != 1 || c->cfg.divopt != c0->cfg.divopt || (c->cfg.sthopt != 0) != (c0->cfg.sthopt != 0) ||
        c->cfg.buyopt != c0->cfg.buyopt || c->g.openx || c->slab)
      return set_error(CRESS_E_UNSUPPORTED,
                       "ensemble members need impopt=1, periodic x and y and the same divopt, sthopt, buyopt");
  }
  cudaSetDevice(c0->device);
  Ensemble* e = new Ensemble;
  e->device = c0->device;
  bool ok = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&e->staged, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming) == cudaSuccess;
  for (int m = 0; ok && m < n; ++m) {
    cudaEvent_t x = nullptr;
    ok = cudaEventCreateWithFlags(&x, cudaEventDisableTiming) == cudaSuccess;
    if (ok) e->ev.push_back(x);
  }
  if (!ok) {
    delete e;
    return set_error(CRESS_E_CUDA, "cress_ensemble_create: stream or event creation failed");
  }
  for (int m = 0; m < n; ++m) {
    Ctx* c = reinterpret_cast<Ctx*>(members[m]);
    cudaStreamSynchronize(c->stream);
    c->free_graphs();
    e->members.push_back(c);
  }
  // the batched acoustic kernel: tile 13 when every member asks for it,
  // else tile 0 (the members follow the ensemble's choice)
  bool all13 = true;
  for (Ctx* c : e->members) all13 = all13 && c->cfg.tile == 13;
  if (!(all13 && e->set_tile(13) == CRESS_OK)) e->set_tile(0);
  *out = reinterpret_cast<cress_ensemble*>(e);
  return CRESS_OK;
}

void cress_ensemble_destroy(cress_ensemble* e) { delete reinterpret_cast<Ensemble*>(e); }

int cress_ensemble_large_step(cress_ensemble* eh, long long ctime, float dtb, int nsstp, float dts) {
  Ensemble* e = reinterpret_cast<Ensemble*>(eh);
  if (!e) return set_error(CRESS_E_ARG, "null ensemble");
  if (nsstp < 1) return set_error(CRESS_E_ARG, "cress_ensemble_large_step: nsstp=%d", nsstp);
  cudaSetDevice(e->device);
  return e->step(ctime, dtb, nsstp, dts);
}

int cress_ensemble_set_tile(cress_ensemble* eh, int tile) {
  Ensemble* e = reinterpret_cast<Ensemble*>(eh);
  if (!e) return set_error(CRESS_E_ARG, "null ensemble");
  cudaSetDevice(e->device);
  return e->set_tile(tile);
}

int cress_ensemble_autotune(cress_ensemble* eh, int nsstp, float dts, int reps, int* best, float* ms) {
  Ensemble* e = reinterpret_cast<Ensemble*>(eh);
  if (!e) return set_error(CRESS_E_ARG, "null ensemble");
  cudaSetDevice(e->device);
  return e->autotune(nsstp, dts, reps, best, ms);
}

int cress_ensemble_set_graphs(cress_ensemble* eh, int on) {
  Ensemble* e = reinterpret_cast<Ensemble*>(eh);
  if (!e) return set_error(CRESS_E_ARG, "null ensemble");
  cudaSetDevice(e->device);
  cudaStreamSynchronize(e->stream);
  e->free_graphs();
  e->graphs = on != 0;
  return CRESS_OK;
}

}  // extern "C"


// The two transports of the y-slab decomposition (slab.h).
//
// LocalLink: the ranks are contexts of this process (on one device or
// several with peer access), each stepped by its own host thread.  An
// exchange is a host barrier between the ranks' threads plus CUDA events:
// every rank records "written" on its stream, waits on its neighbours'
// events, copies the neighbours' rows into its ghost rows (device-to-device
// copies on its own stream), records "read", and before going on waits
// until its neighbours have read its rows.  No kernel waits on another
// rank's kernel; the ordering is the streams'.  The barrier gives up after
// a bounded time and a rank that fails breaks it for the others, so a
// failing rank cannot leave the rest waiting.
//
// NcclLink: one rank per process and GPU.  The rows travel with
// ncclSend/ncclRecv (packed by 2-D copies into contiguous buffers), the
// sub-step word with ncclAllReduce(min), all on the context's stream.
// NCCL is loaded at run time (dlopen of libnccl.so.2), so the library has
// no link-time dependency on it.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <vector>
#include "../../include/cress_b200.h"
#include "common.cuh"
#include "ctx.h"
#include "slab.h"

namespace cress {
namespace {

// first destination / source rows (two rows each) of the exchange
struct RowPlan {
  int lo_dst, lo_src, hi_dst, hi_src;
};
RowPlan rows_for(int stag, int nj_self, int nj_south) {
  RowPlan p;
  p.lo_dst = 0;
  p.lo_src = nj_south - 3;   // rows 0, 1 <- south's nj-3, nj-2
  if (stag == STAG_V) {
    p.hi_dst = nj_self;      // rows nj, nj+1 <- north's 3, 4
    p.hi_src = 3;
  } else {
    p.hi_dst = nj_self - 1;  // rows nj-1, nj <- north's 2, 3
    p.hi_src = 2;
  }
  return p;
}

// two rows (2 px floats) of every level, between fields of grids g (dst)
// and gs (src)
int copy_rows(cudaStream_t st, const Grid& g, float* dst, int dst_row, const Grid& gs, const float* src,
              int src_row) {
  return cuda_check(cudaMemcpy2DAsync(dst + (long long)dst_row * g.px, (size_t)g.plane * 4,
                                      src + (long long)src_row * gs.px, (size_t)gs.plane * 4, 2 * (size_t)g.px * 4,
                                      (size_t)g.nk, cudaMemcpyDeviceToDevice, st),
                    "slab row copy");
}

__global__ void k_min_words(int* const* words, int n, int* out) {
  int m = *out;
  for (int q = 0; q < n; ++q) m = min(m, *(volatile int*)words[q]);
  *out = m;
}

}  // namespace

// The ranks of one process (cress_slab_group).
struct SlabGroup {
  int n = 0;
  std::mutex m;
  std::condition_variable cv;
  int arrived = 0;
  long long gen = 0;
  bool broken = false;
  std::vector<Ctx*> ctx;
  std::vector<float* const*> fields;
  std::vector<int*> words;
  std::vector<cudaEvent_t> ready, done;
  int** words_d = nullptr;   // device copy of `words`
  int timeout_ms = 60000;

  // Host barrier of the n ranks, bounded (timeout_ms), or at once when a rank broke it.
  int barrier() {
    std::unique_lock<std::mutex> lk(m);
    if (broken) return set_error(CRESS_E_STATE, "slab exchange: another rank failed");
    const long long my = gen;
    if (++arrived == n) {
      arrived = 0;
      ++gen;
      cv.notify_all();
      return CRESS_OK;
    }
    const bool ok = cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return gen != my || broken; });
    if (broken) return set_error(CRESS_E_STATE, "slab exchange: another rank failed");
    if (!ok) {
      broken = true;
      cv.notify_all();
      return set_error(CRESS_E_TIMEOUT, "slab exchange: the other ranks did not arrive within %d ms", timeout_ms);
    }
    return CRESS_OK;
  }
  void fail() {
    std::lock_guard<std::mutex> lk(m);
    broken = true;
    cv.notify_all();
  }
};

namespace {

struct LocalLink : SlabLink {
  SlabGroup* G;
  int south() const { return (rank - 1 + nranks) % nranks; }
  int north() const { return (rank + 1) % nranks; }
  int guard(int rc) {
    if (rc) G->fail();
    return rc;
  }
  int exchange(Ctx* c, int nf, float* const* f, const int* stag) override {
    int rc;
    G->fields[rank] = f;
    if ((rc = cuda_check(cudaEventRecord(G->ready[rank], c->stream), "slab event"))) return guard(rc);
    if ((rc = G->barrier())) return rc;
    const int s = south(), nn = north();
    Ctx* cs = G->ctx[s];
    Ctx* cn = G->ctx[nn];
    if ((rc = cuda_check(cudaStreamWaitEvent(c->stream, G->ready[s], 0), "slab wait")) ||
        (rc = cuda_check(cudaStreamWaitEvent(c->stream, G->ready[nn], 0), "slab wait")))
      return guard(rc);
    for (int q = 0; q < nf && !rc; ++q) {
      const RowPlan p = rows_for(stag[q], c->g.nj, cs->g.nj);
      rc = copy_rows(c->stream, c->g, f[q], p.lo_dst, cs->g, G->fields[s][q], p.lo_src);
      if (!rc) rc = copy_rows(c->stream, c->g, f[q], p.hi_dst, cn->g, G->fields[nn][q], p.hi_src);
    }
    if (rc) return guard(rc);
    if ((rc = cuda_check(cudaEventRecord(G->done[rank], c->stream), "slab event"))) return guard(rc);
    if ((rc = G->barrier())) return rc;
    if ((rc = cuda_check(cudaStreamWaitEvent(c->stream, G->done[s], 0), "slab wait")) ||
        (rc = cuda_check(cudaStreamWaitEvent(c->stream, G->done[nn], 0), "slab wait")))
      return guard(rc);
    return CRESS_OK;
  }
  int min_word(Ctx* c, int* word) override {
    int rc;
    G->words[rank] = word;
    if ((rc = cuda_check(cudaEventRecord(G->ready[rank], c->stream), "slab event"))) return guard(rc);
    if ((rc = G->barrier())) return rc;
    if (rank == 0 &&
        (rc = cuda_check(cudaMemcpyAsync(G->words_d, G->words.data(), sizeof(int*) * G->n, cudaMemcpyHostToDevice,
                                         c->stream), "slab words")))
      return guard(rc);
    for (int q = 0; q < nranks && !rc; ++q)
      if (q != rank) rc = cuda_check(cudaStreamWaitEvent(c->stream, G->ready[q], 0), "slab wait");
    if (rc) return guard(rc);
    // rank 0 uploads the word table; the others take it once rank 0 has
    if ((rc = cuda_check(cudaEventRecord(G->done[rank], c->stream), "slab event"))) return guard(rc);
    if ((rc = G->barrier())) return rc;
    if (rank != 0 && (rc = cuda_check(cudaStreamWaitEvent(c->stream, G->done[0], 0), "slab wait")))
      return guard(rc);
    k_min_words<<<1, 1, 0, c->stream>>>(G->words_d, nranks, word);
    ++c->launches;
    if ((rc = cuda_check(cudaGetLastError(), "slab minimum"))) return guard(rc);
    if ((rc = cuda_check(cudaEventRecord(G->done[rank], c->stream), "slab event"))) return guard(rc);
    if ((rc = G->barrier())) return rc;
    for (int q = 0; q < nranks && !rc; ++q)
      if (q != rank) rc = cuda_check(cudaStreamWaitEvent(c->stream, G->done[q], 0), "slab wait");
    return guard(rc);
  }
};

// NCCL entry points, resolved at run time.
struct Nccl {
  bool ok = false;
  decltype(&ncclGetUniqueId) getUniqueId = nullptr;
  decltype(&ncclCommInitRank) commInitRank = nullptr;
  decltype(&ncclCommDestroy) commDestroy = nullptr;
  decltype(&ncclGroupStart) groupStart = nullptr;
  decltype(&ncclGroupEnd) groupEnd = nullptr;
  decltype(&ncclSend) send = nullptr;
  decltype(&ncclRecv) recv = nullptr;
  decltype(&ncclAllReduce) allReduce = nullptr;
  decltype(&ncclGetErrorString) errorString = nullptr;
};
Nccl& nccl() {
  static Nccl N;
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) return;
    N.getUniqueId = (decltype(N.getUniqueId))dlsym(h, "ncclGetUniqueId");
    N.commInitRank = (decltype(N.commInitRank))dlsym(h, "ncclCommInitRank");
    N.commDestroy = (decltype(N.commDestroy))dlsym(h, "ncclCommDestroy");
    N.groupStart = (decltype(N.groupStart))dlsym(h, "ncclGroupStart");
    N.groupEnd = (decltype(N.groupEnd))dlsym(h, "ncclGroupEnd");
    N.send = (decltype(N.send))dlsym(h, "ncclSend");
    N.recv = (decltype(N.recv))dlsym(h, "ncclRecv");
    N.allReduce = (decltype(N.allReduce))dlsym(h, "ncclAllReduce");
    N.errorString = (decltype(N.errorString))dlsym(h, "ncclGetErrorString");
    N.ok = N.getUniqueId && N.commInitRank && N.commDestroy && N.groupStart && N.groupEnd && N.send && N.recv &&
           N.allReduce && N.errorString;
  });
  return N;
}
int nccl_check(ncclResult_t r, const char* what) {
  if (r == ncclSuccess) return CRESS_OK;
  return set_error(CRESS_E_CUDA, "%s: %s", what, nccl().errorString(r));
}

struct NcclLink : SlabLink {
  ncclComm_t comm = nullptr;
  float* buf = nullptr;   // send south | send north | recv south | recv north
  size_t cap = 0;         // floats per quarter
  ~NcclLink() override {
    if (comm) nccl().commDestroy(comm);
    if (buf) cudaFree(buf);
  }
  int exchange(Ctx* c, int nf, float* const* f, const int* stag) override {
    const Grid& g = c->g;
    const size_t slab = 2 * (size_t)g.px * g.nk;   // two rows of every level
    const size_t need = slab * nf;
    int rc = CRESS_OK;
    if (need > cap) {
      if (buf) cudaFree(buf);
      buf = nullptr;
      cap = 0;
      if ((rc = cuda_check(cudaMalloc(&buf, 4 * need * sizeof(float)), "slab buffers"))) return rc;
      cap = need;
    }
    float *sS = buf, *sN = buf + cap, *rS = buf + 2 * cap, *rN = buf + 3 * cap;
    const Grid packed{g.ni, 2, g.nk, g.px, 2, 2LL * g.px, 0};   // two rows per level, contiguous
    for (int q = 0; q < nf && !rc; ++q) {
      const RowPlan p = rows_for(stag[q], g.nj, g.nj);
      // to the south: the rows its high ghosts take; to the north: rows nj-3, nj-2
      rc = copy_rows(c->stream, packed, sS + q * slab, 0, g, f[q], p.hi_src);
      if (!rc) rc = copy_rows(c->stream, packed, sN + q * slab, 0, g, f[q], g.nj - 3);
    }
    if (rc) return rc;
    const int s = (rank - 1 + nranks) % nranks, nn = (rank + 1) % nranks;
    Nccl& N = nccl();
    if ((rc = nccl_check(N.groupStart(), "ncclGroupStart"))) return rc;
    // per peer, sends and receives pair up in order: the northward message
    // first, then the southward one (ranks 2 apart from both sides agree)
    N.send(sN, need, ncclFloat32, nn, comm, c->stream);
    N.recv(rS, need, ncclFloat32, s, comm, c->stream);
    N.send(sS, need, ncclFloat32, s, comm, c->stream);
    N.recv(rN, need, ncclFloat32, nn, comm, c->stream);
    if ((rc = nccl_check(N.groupEnd(), "ncclGroupEnd"))) return rc;
    for (int q = 0; q < nf && !rc; ++q) {
      const RowPlan p = rows_for(stag[q], g.nj, g.nj);
      rc = copy_rows(c->stream, g, f[q], p.lo_dst, packed, rS + q * slab, 0);
      if (!rc) rc = copy_rows(c->stream, g, f[q], p.hi_dst, packed, rN + q * slab, 0);
    }
    return rc;
  }
  int min_word(Ctx* c, int* word) override {
    return nccl_check(nccl().allReduce(word, word, 1, ncclInt32, ncclMin, comm, c->stream), "ncclAllReduce");
  }
};

int slab_attach_checks(Ctx* c) {
  if (c->g.openx) return set_error(CRESS_E_UNSUPPORTED, "slab decomposition: periodic x only");
  // the HE-VE step keeps the contravariant w of two levels in side buffers
  // whose y ghosts it wraps itself
  if (c->cfg.impopt != 1) return set_error(CRESS_E_UNSUPPORTED, "slab decomposition: HE-VI (impopt=1) only");
  if (c->mlp || c->sampler)
    return set_error(CRESS_E_UNSUPPORTED, "slab decomposition: plain microphysics only (no learned form or sampling)");
  if (c->slab) return set_error(CRESS_E_STATE, "slab decomposition: context already attached");
  return CRESS_OK;
}

void slab_attach(Ctx* c, SlabLink* link) {
  c->free_graphs();
  c->graphs = false;   // the exchanges order ranks through host barriers
  c->slab = link;
  c->g.slaby = 1;
}

}  // namespace
}  // namespace cress

using namespace cress;

extern "C" int cress_slab_group_create(int n, cress_slab_group** out) {
  if (n < 1 || !out) return set_error(CRESS_E_ARG, "cress_slab_group_create: n=%d", n);
  SlabGroup* G = new SlabGroup();
  G->n = n;
  G->ctx.assign(n, nullptr);
  G->fields.assign(n, nullptr);
  G->words.assign(n, nullptr);
  G->ready.assign(n, nullptr);
  G->done.assign(n, nullptr);
  bool ok = cudaMalloc(&G->words_d, sizeof(int*) * n) == cudaSuccess;
  for (int r = 0; r < n && ok; ++r)
    ok = cudaEventCreateWithFlags(&G->ready[r], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&G->done[r], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    cress_slab_group_destroy(reinterpret_cast<cress_slab_group*>(G));
    return set_error(CRESS_E_CUDA, "cress_slab_group_create: CUDA allocation failed");
  }
  *out = reinterpret_cast<cress_slab_group*>(G);
  return CRESS_OK;
}

extern "C" int cress_slab_group_set_timeout(cress_slab_group* grp, int ms) {
  SlabGroup* G = reinterpret_cast<SlabGroup*>(grp);
  if (!G || ms < 1) return set_error(CRESS_E_ARG, "cress_slab_group_set_timeout: bad arguments");
  G->timeout_ms = ms;
  return CRESS_OK;
}

extern "C" void cress_slab_group_destroy(cress_slab_group* grp) {
  SlabGroup* G = reinterpret_cast<SlabGroup*>(grp);
  if (!G) return;
  for (cudaEvent_t e : G->ready)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : G->done)
    if (e) cudaEventDestroy(e);
  if (G->words_d) cudaFree(G->words_d);
  delete G;
}

extern "C" int cress_slab_attach_local(cress_ctx* ctx, cress_slab_group* grp, int rank) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  SlabGroup* G = reinterpret_cast<SlabGroup*>(grp);
  if (!c || !G || rank < 0 || rank >= G->n) return set_error(CRESS_E_ARG, "cress_slab_attach_local: bad arguments");
  int rc = slab_attach_checks(c);
  if (rc) return rc;
  if (G->ctx[rank]) return set_error(CRESS_E_STATE, "cress_slab_attach_local: rank %d taken", rank);
  for (Ctx* o : G->ctx)
    if (o && (o->g.ni != c->g.ni || o->g.nk != c->g.nk))
      return set_error(CRESS_E_ARG, "cress_slab_attach_local: ranks must share ni and nk (y slabs)");
  if (c->g.nj < 8) return set_error(CRESS_E_ARG, "cress_slab_attach_local: a slab needs nj >= 8");
  LocalLink* L = new LocalLink();
  L->G = G;
  L->rank = rank;
  L->nranks = G->n;
  G->ctx[rank] = c;
  slab_attach(c, L);
  return CRESS_OK;
}

extern "C" int cress_slab_nccl_id(void* out) {
  if (!out) return set_error(CRESS_E_ARG, "cress_slab_nccl_id: null argument");
  Nccl& N = nccl();
  if (!N.ok) return set_error(CRESS_E_UNSUPPORTED, "cress_slab_nccl_id: libnccl.so.2 could not be loaded");
  ncclUniqueId id;
  int rc = nccl_check(N.getUniqueId(&id), "ncclGetUniqueId");
  if (!rc) std::memcpy(out, &id, sizeof id);
  return rc;
}

extern "C" int cress_slab_attach_nccl(cress_ctx* ctx, int rank, int nranks, const void* id) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !id || nranks < 1 || rank < 0 || rank >= nranks)
    return set_error(CRESS_E_ARG, "cress_slab_attach_nccl: bad arguments");
  int rc = slab_attach_checks(c);
  if (rc) return rc;
  Nccl& N = nccl();
  if (!N.ok) return set_error(CRESS_E_UNSUPPORTED, "cress_slab_attach_nccl: libnccl.so.2 could not be loaded");
  cudaSetDevice(c->device);
  ncclUniqueId uid;
  std::memcpy(&uid, id, sizeof uid);
  NcclLink* L = new NcclLink();
  L->rank = rank;
  L->nranks = nranks;
  if ((rc = nccl_check(N.commInitRank(&L->comm, nranks, uid, rank), "ncclCommInitRank"))) {
    delete L;
    return rc;
  }
  slab_attach(c, L);
  return CRESS_OK;
}

extern "C" int cress_slab_detach(cress_ctx* ctx) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "cress_slab_detach: null context");
  if (!c->slab) return CRESS_OK;
  cudaStreamSynchronize(c->stream);
  LocalLink* L = dynamic_cast<LocalLink*>(c->slab);
  if (L && L->G->ctx[L->rank] == c) L->G->ctx[L->rank] = nullptr;
  delete c->slab;
  c->slab = nullptr;
  c->g.slaby = 0;
  return CRESS_OK;
}

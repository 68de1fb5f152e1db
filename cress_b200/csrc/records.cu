// Dump and restart records in the reference's file layouts, formed on the
// device so that a host that writes CReSS's files copies one finished byte
// stream per file instead of every array.
//
// Dump (SrcOrig/outdmp.f90:380-870 with SrcOrig/outdmp3d.f90:159-238,
// dmplev = 1, dmpfmt = 2): for every variable dmpvar selects, in the order
// s_outdmp calls s_outdmp3d, the nz records k = 2..nk-2 of nx*ny floats
// (i = 2..ni-2 fastest, j = 2..nj-2), staggered variables averaged to the
// scalar points (u: .5(u(i)+u(i+1)), v: .5(v(j)+v(j+1)), w:
// .5(w(k)+w(k+1))), "bar" variables from the base state, totals
// (dmpvar '-': p = pbr + pp, pt = ptbr + ptp, s_totals).  Direct access
// records carry no framing, so the byte stream is the .bin file.
//
// Restart (SrcOrig/outres.f90:903-1289 after the base-state records): the
// device-held records, each a Fortran sequential unformatted record (a
// 4-byte length before and after the payload, the framing gfortran and
// ifort write for records below 2 GiB): u, v, w, pp, ptp; up .. ptpp; with
// open x the phase speeds ucpx, ucpy, ... ptcpy; with cold rain qv, qvp,
// (qvcpx, qvcpy), qwtr (qc, qr), qwtrp, (qwcpx, qwcpy), qice (qi, qs, qg),
// nice (ni, ns, ng), qicep, nicep, (qicpx, qicpy, nicpx, nicpy), the rate
// and accumulation planes of prwtr and price; with the TKE closure tke,
// tkep.  Arrays keep their full shape (0:ni+1, 0:nj+1, 1:nk).  The y phase
// speeds (ucpy, ...) exist in the file but the periodic y of this library
// never forms them: they are written as zeros, as the reference holds
// them, and skipped on reading.
//
// One device staging buffer per context holds the stream; the fields
// cross into or out of it with the repitch kernel, the dump values with
// k_dump_pack, and the host sees one contiguous copy.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/cress_b200.h"
#include "common.cuh"
#include "ctx.h"
#include "forcing.cuh"
#include "hevi.cuh"
#include "openbc.cuh"

namespace cress {
namespace {

constexpr int kDumpMax = 24;
enum DumpKind { DK_XXX = 0, DK_OXX, DK_XOX, DK_XXO };

struct DumpItem {
  const float* f;   // field, or null: the base column alone ("bar")
  int kind;         // DumpKind
  int col;          // base column added (s_totals), or -1; the column itself when f is null
  long long out;    // first float of the item's records
};
struct DumpArgs {
  Grid g;
  const float* col;   // base columns, col[f*(nk+1) + k]
  int n;
  DumpItem it[kDumpMax];
  float* out;
};

// One thread per record value: x along i, blockIdx.y = j, blockIdx.z =
// item * nz + (k-2).
__global__ void __launch_bounds__(128) k_dump_pack(const __grid_constant__ DumpArgs a) {
  const Grid g = a.g;
  const int nx = g.ni - 3, ny = g.nj - 3, nz = g.nk - 3;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= nx) return;
  const int y = blockIdx.y, t = blockIdx.z / nz, kz = blockIdx.z % nz;
  const int i = x + 2, j = y + 2, k = kz + 2;
  const DumpItem& it = a.it[t];
  const int nc = g.nk + 1;
  float v;
  if (!it.f) {
    v = __ldg(a.col + it.col * nc + k);
  } else {
    const long long id = g.at(i, j, k);
    const float* f = it.f;
    switch (it.kind) {
      case DK_OXX: v = .5f * (__ldg(f + id) + __ldg(f + id + 1)); break;
      case DK_XOX: v = .5f * (__ldg(f + id) + __ldg(f + id + g.px)); break;
      case DK_XXO: v = .5f * (__ldg(f + id) + __ldg(f + id + g.plane)); break;
      default: v = __ldg(f + id);
    }
    if (it.col >= 0) v = __ldg(a.col + it.col * nc + k) + v;   // s_totals: sbr + sp
  }
  a.out[it.out + ((long long)kz * ny + y) * nx + x] = v;
}

// The 4-byte record lengths of a restart stream, before and after each
// payload.
constexpr int kMarkMax = 128;
struct MarkArgs {
  uint32_t* base;
  int n;
  long long at[kMarkMax];   // uint32 index of the marker
  uint32_t val[kMarkMax];
};
__global__ void k_marks(const __grid_constant__ MarkArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < a.n) a.base[a.at[t]] = a.val[t];
}

// A restart record: payload parts in file order.
enum PartKind { PK_FIELD = 0, PK_PLANE, PK_RAD, PK_ZERO };
struct Part {
  int kind;
  float* dev;        // device source / destination (first element)
  int pitch, width;  // floats
  long long rows;
  long long floats() const { return (long long)width * rows; }
};
struct Rec {
  std::vector<Part> parts;
  long long floats() const {
    long long n = 0;
    for (const Part& p : parts) n += p.floats();
    return n;
  }
};

Part field_part(const Ctx* c, float* f) {
  const Grid& g = c->g;
  return Part{PK_FIELD, f, g.px, g.ni + 2, (long long)(g.nj + 2) * g.nk};
}
// precipitation plane p (2*species + 0 rate / 1 accumulation), (0:ni+1, 0:nj+1)
Part plane_part(const Ctx* c, int p) {
  const Grid& g = c->g;
  return Part{PK_PLANE, c->prec_d + (long long)p * g.plane, g.px, g.ni + 2, (long long)g.nj + 2};
}
// x phase speeds of one variable and side, (1:nj, 1:nk)
Part rad_part(const Ctx* c, int var, int side) {
  const Grid& g = c->g;
  return Part{PK_RAD, c->rad_d + rad_at(g, var, side, 1, 1), g.nj + 2, g.nj, (long long)g.nk};
}
// y phase speeds of one variable, both sides (1:ni, 1:nk, 1:2): zero with periodic y
Part zero_part(const Ctx* c) {
  const Grid& g = c->g;
  return Part{PK_ZERO, nullptr, 0, g.ni, 2LL * g.nk};
}

// The device-held records of s_outres in file order (outres.f90:903-1289
// for advopt <= 3, cphopt 0 or 3 with haiopt = 0, sfcopt = aslopt = trkopt
// = 0, no maximum-wind dump).
std::vector<Rec> restart_records(Ctx* c) {
  std::vector<Rec> r;
  const int N = CRESS_NOW, P = CRESS_PAST;
  auto one = [&](Part p) { r.push_back(Rec{{p}}); };
  auto fld = [&](int f, int lvl) { return field_part(c, c->lev[f][lvl]); };
  const bool open = c->g.openx != 0, moist = c->cfg.cphopt == 3, tke = c->cfg.tubopt == 2;
  for (int f = CRESS_U; f <= CRESS_PTP; ++f) one(fld(f, N));   // :905-918
  for (int f = CRESS_U; f <= CRESS_PTP; ++f) one(fld(f, P));   // :922-935
  auto cp = [&](int var) {                                       // xcpx then xcpy
    r.push_back(Rec{{rad_part(c, var, 0), rad_part(c, var, 1)}});
    r.push_back(Rec{{zero_part(c)}});
  };
  if (open)
    for (int v = RAD_U; v <= RAD_PT; ++v) cp(v);                 // :939-967
  if (moist) {
    one(fld(CRESS_QV, N));                                       // :973-974
    one(fld(CRESS_QV, P));                                       // :980-981
    if (open) cp(RAD_QV);                                        // :988-992
    r.push_back(Rec{{fld(CRESS_QC, N), fld(CRESS_QR, N)}});      // qwtr  :999-1000
    r.push_back(Rec{{fld(CRESS_QC, P), fld(CRESS_QR, P)}});      // qwtrp :1014-1015
    if (open) {                                                   // qwcpx, qwcpy :1031-1035
      r.push_back(Rec{{rad_part(c, RAD_QV + 1, 0), rad_part(c, RAD_QV + 1, 1), rad_part(c, RAD_QV + 2, 0),
                       rad_part(c, RAD_QV + 2, 1)}});
      r.push_back(Rec{{zero_part(c), zero_part(c)}});
    }
    r.push_back(Rec{{fld(CRESS_QI, N), fld(CRESS_QS, N), fld(CRESS_QG, N)}});   // qice  :1054-1055
    r.push_back(Rec{{fld(CRESS_NI, N), fld(CRESS_NS, N), fld(CRESS_NG, N)}});   // nice  :1070-1071
    r.push_back(Rec{{fld(CRESS_QI, P), fld(CRESS_QS, P), fld(CRESS_QG, P)}});   // qicep :1080-1081
    r.push_back(Rec{{fld(CRESS_NI, P), fld(CRESS_NS, P), fld(CRESS_NG, P)}});   // nicep :1095-1096
    if (open) {                                                   // qicpx .. nicpy :1106-1126
      for (int base : {RAD_QV + 3, RAD_QV + 6}) {
        Rec x, y;
        for (int n = 0; n < 3; ++n) {
          x.parts.push_back(rad_part(c, base + n, 0));
          x.parts.push_back(rad_part(c, base + n, 1));
          y.parts.push_back(zero_part(c));
        }
        r.push_back(x);
        r.push_back(y);
      }
    }
    // prwtr(:,:,1,n), prwtr(:,:,2,n) for prc, prr; price for pri, prs, prg (:1136-1163)
    r.push_back(Rec{{plane_part(c, 0), plane_part(c, 2)}});
    r.push_back(Rec{{plane_part(c, 1), plane_part(c, 3)}});
    r.push_back(Rec{{plane_part(c, 4), plane_part(c, 6), plane_part(c, 8)}});
    r.push_back(Rec{{plane_part(c, 5), plane_part(c, 7), plane_part(c, 9)}});
  }
  if (tke) {
    one(fld(CRESS_TKE, N));   // :1280-1281
    one(fld(CRESS_TKE, P));   // :1287-1288
  }
  return r;
}

long long stream_bytes(const std::vector<Rec>& recs) {
  long long n = 0;
  for (const Rec& r : recs) n += 8 + 4 * r.floats();
  return n;
}

int ensure_records_buffer(Ctx* c, long long bytes) {
  if (c->rec_bytes >= bytes) return CRESS_OK;
  if (c->rec_d) cudaFree(c->rec_d);
  c->rec_d = nullptr;
  c->rec_bytes = 0;
  int rc = cuda_check(cudaMalloc(&c->rec_d, (size_t)bytes), "cudaMalloc record buffer");
  if (!rc) c->rec_bytes = bytes;
  return rc;
}

// The variables s_outdmp dumps for dmpvar (dmplev = 1), in its order.
struct DumpVar {
  const char* name;
  int field;   // CRESS_* field, or -1 (base column alone)
  int kind;
  int col;     // base column (bar, or added for totals), or -1
};
int dump_vars(const Ctx* c, const char* dmpvar, std::vector<DumpVar>& out) {
  char v[16];
  std::memset(v, 'x', sizeof v);
  for (int q = 0; q < 16 && dmpvar[q]; ++q) v[q] = dmpvar[q];
  const bool moist = c->cfg.cphopt == 3;
  // as in s_outdmp, a switch dumps only for the characters it tests ('o',
  // and '-' for u, v, p, pt, qv); any other character leaves it out
  auto sel = [&](int q, const char* ok) { return std::strchr(ok, v[q]) != nullptr; };
  if (c->cfg.tubopt >= 2 && sel(11, "+-"))
    return set_error(CRESS_E_UNSUPPORTED, "cress_dump_3d: the maximum wind (dmpvar(12:12) '+' or '-') is not kept");
  const bool have_p = c->moist_set;   // pbr comes with the moist base state
  if (sel(3, "o-") && !have_p)
    return set_error(CRESS_E_STATE, "cress_dump_3d: pbar/p need the base pressure (cress_set_base_moist)");
  out.clear();
  // outdmp.f90:394-419 (u, v), 509-513 (w), 520-534 (p), 541-555 (pt)
  if (v[0] == 'o') out.push_back({"ubar", -1, DK_OXX, C_UBR});
  if (sel(0, "o-")) out.push_back({"u", CRESS_U, DK_OXX, -1});
  if (v[1] == 'o') out.push_back({"vbar", -1, DK_XOX, C_VBR});
  if (sel(1, "o-")) out.push_back({"v", CRESS_V, DK_XOX, -1});
  if (v[2] == 'o') out.push_back({"w", CRESS_W, DK_XXO, -1});
  if (v[3] == 'o') { out.push_back({"pbar", -1, DK_XXX, C_PBR}); out.push_back({"pp", CRESS_PP, DK_XXX, -1}); }
  if (v[3] == '-') out.push_back({"p", CRESS_PP, DK_XXX, C_PBR});
  if (v[4] == 'o') { out.push_back({"ptbar", -1, DK_XXX, C_PTBR}); out.push_back({"ptp", CRESS_PTP, DK_XXX, -1}); }
  if (v[4] == '-') out.push_back({"pt", CRESS_PTP, DK_XXX, C_PTBR});
  if (moist) {   // outdmp.f90:564-575 (qv), 590-635 (cphopt = 3, haiopt = 0)
    if (v[5] == 'o') out.push_back({"qvbar", -1, DK_XXX, C_QVBR});
    if (sel(5, "o-")) out.push_back({"qv", CRESS_QV, DK_XXX, -1});
    if (v[6] == 'o')
      for (int f : {CRESS_QC, CRESS_QR, CRESS_QI, CRESS_QS, CRESS_QG})
        out.push_back({f == CRESS_QC ? "qc" : f == CRESS_QR ? "qr" : f == CRESS_QI ? "qi" : f == CRESS_QS ? "qs" : "qg",
                       f, DK_XXX, -1});
    if (v[7] == 'o')
      for (int f : {CRESS_NI, CRESS_NS, CRESS_NG})
        out.push_back({f == CRESS_NI ? "nci" : f == CRESS_NS ? "ncs" : "ncg", f, DK_XXX, -1});
  }
  if (c->cfg.tubopt >= 2 && v[11] == 'o') out.push_back({"tke", CRESS_TKE, DK_XXX, -1});   // :858-862
  return CRESS_OK;
}

}  // namespace
}  // namespace cress

using namespace cress;

extern "C" int cress_dump_3d(cress_ctx* ctx, int level, const char* dmpvar, void* host, long long cap_bytes,
                             long long* nbytes, char* names, int names_cap) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !dmpvar) return set_error(CRESS_E_ARG, "cress_dump_3d: null argument");
  if (level < CRESS_PAST || level > CRESS_FUTURE) return set_error(CRESS_E_ARG, "cress_dump_3d: level %d", level);
  if (!c->base_set || !c->large_set) return set_error(CRESS_E_STATE, "cress_dump_3d: base state not set");
  std::vector<DumpVar> vars;
  int rc = dump_vars(c, dmpvar, vars);
  if (rc) return rc;
  if ((int)vars.size() > kDumpMax) return set_error(CRESS_E_UNSUPPORTED, "cress_dump_3d: too many variables");
  const Grid& g = c->g;
  const long long rec = (long long)(g.ni - 3) * (g.nj - 3), per_var = rec * (g.nk - 3);
  const long long bytes = 4 * per_var * (long long)vars.size();
  if (nbytes) *nbytes = bytes;
  if (names && names_cap > 0) {
    std::string s;
    for (const DumpVar& d : vars) s += (s.empty() ? "" : ",") + std::string(d.name);
    if ((int)s.size() + 1 > names_cap) return set_error(CRESS_E_ARG, "cress_dump_3d: names buffer too small");
    std::memcpy(names, s.c_str(), s.size() + 1);
  }
  if (!host || vars.empty()) return CRESS_OK;
  if (cap_bytes < bytes) return set_error(CRESS_E_ARG, "cress_dump_3d: %lld bytes needed", bytes);
  for (const DumpVar& d : vars)
    if (d.field >= 0 && !c->lev[d.field][level]) return set_error(CRESS_E_STATE, "cress_dump_3d: %s not held", d.name);
  cudaSetDevice(c->device);
  if ((rc = ensure_records_buffer(c, bytes))) return rc;
  DumpArgs a{};
  a.g = g;
  a.col = c->col_d;
  a.n = (int)vars.size();
  a.out = reinterpret_cast<float*>(c->rec_d);
  for (int t = 0; t < a.n; ++t)
    a.it[t] = DumpItem{vars[t].field >= 0 ? c->lev[vars[t].field][level] : nullptr, vars[t].kind, vars[t].col,
                       per_var * t};
  dim3 grid((g.ni - 3 + 127) / 128, g.nj - 3, (unsigned)(a.n * (g.nk - 3)));
  k_dump_pack<<<grid, 128, 0, c->stream>>>(a);
  ++c->launches;
  if ((rc = cuda_check(cudaGetLastError(), "dump pack launch")) ||
      (rc = cuda_check(cudaMemcpyAsync(host, c->rec_d, (size_t)bytes, cudaMemcpyDeviceToHost, c->stream),
                       "dump copy")))
    return rc;
  return cuda_check(cudaStreamSynchronize(c->stream), "dump sync");
}

extern "C" int cress_restart_write(cress_ctx* ctx, void* host, long long cap_bytes, long long* nbytes) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c) return set_error(CRESS_E_ARG, "cress_restart_write: null context");
  const std::vector<Rec> recs = restart_records(c);
  const long long bytes = stream_bytes(recs);
  if (nbytes) *nbytes = bytes;
  if (!host) return CRESS_OK;
  if (cap_bytes < bytes) return set_error(CRESS_E_ARG, "cress_restart_write: %lld bytes needed", bytes);
  if ((int)recs.size() * 2 > kMarkMax) return set_error(CRESS_E_UNSUPPORTED, "cress_restart_write: too many records");
  for (const Rec& r : recs)
    if (4 * r.floats() > 0x7fffffffLL)
      return set_error(CRESS_E_UNSUPPORTED, "cress_restart_write: a record of %lld bytes needs 2 GiB subrecords",
                       4 * r.floats());
  cudaSetDevice(c->device);
  int rc;
  if ((rc = ensure_records_buffer(c, bytes))) return rc;
  MarkArgs m{};
  m.base = reinterpret_cast<uint32_t*>(c->rec_d);
  long long off = 0;   // in floats
  for (const Rec& r : recs) {
    const uint32_t len = (uint32_t)(4 * r.floats());
    m.at[m.n] = off; m.val[m.n++] = len;
    ++off;
    for (const Part& p : r.parts) {
      float* dst = reinterpret_cast<float*>(c->rec_d) + off;
      if (p.kind == PK_ZERO) {
        rc = cuda_check(cudaMemsetAsync(dst, 0, 4 * (size_t)p.floats(), c->stream), "zero record part");
      } else {
        rc = launch_repitch(p.dev, p.pitch, dst, p.width, p.width, p.rows, c->stream);
        ++c->launches;
      }
      if (rc) return rc;
      off += p.floats();
    }
    m.at[m.n] = off; m.val[m.n++] = len;
    ++off;
  }
  k_marks<<<1, kMarkMax, 0, c->stream>>>(m);
  ++c->launches;
  if ((rc = cuda_check(cudaGetLastError(), "record marker launch")) ||
      (rc = cuda_check(cudaMemcpyAsync(host, c->rec_d, (size_t)bytes, cudaMemcpyDeviceToHost, c->stream),
                       "restart copy")))
    return rc;
  return cuda_check(cudaStreamSynchronize(c->stream), "restart sync");
}

extern "C" int cress_restart_read(cress_ctx* ctx, const void* host, long long nbytes) {
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  if (!c || !host) return set_error(CRESS_E_ARG, "cress_restart_read: null argument");
  const std::vector<Rec> recs = restart_records(c);
  const long long bytes = stream_bytes(recs);
  if (nbytes != bytes)
    return set_error(CRESS_E_ARG, "cress_restart_read: %lld bytes given, this configuration's records take %lld",
                     nbytes, bytes);
  // the framing must be the one this configuration writes
  const unsigned char* h = static_cast<const unsigned char*>(host);
  long long off = 0;
  for (size_t q = 0; q < recs.size(); ++q) {
    const uint32_t len = (uint32_t)(4 * recs[q].floats());
    uint32_t a, b;
    std::memcpy(&a, h + off, 4);
    std::memcpy(&b, h + off + 4 + len, 4);
    if (a != len || b != len)
      return set_error(CRESS_E_ARG, "cress_restart_read: record %d framed %u/%u, expected %u", (int)q + 1, a, b, len);
    off += 8 + len;
  }
  cudaSetDevice(c->device);
  int rc;
  if ((rc = ensure_records_buffer(c, bytes)) ||
      (rc = cuda_check(cudaMemcpyAsync(c->rec_d, host, (size_t)bytes, cudaMemcpyHostToDevice, c->stream),
                       "restart copy")))
    return rc;
  long long at = 0;   // in floats
  for (const Rec& r : recs) {
    ++at;
    for (const Part& p : r.parts) {
      if (p.kind != PK_ZERO) {
        const float* src = reinterpret_cast<const float*>(c->rec_d) + at;
        if ((rc = launch_repitch(src, p.width, p.dev, p.pitch, p.width, p.rows, c->stream))) return rc;
        ++c->launches;
      }
      at += p.floats();
    }
    ++at;
  }
  return cuda_check(cudaStreamSynchronize(c->stream), "restart sync");
}

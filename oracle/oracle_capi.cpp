// Oracle C entry points (ctypes-callable).
//
// TEST INFRASTRUCTURE ONLY.  The parity tests, __graft_entry__.smoke() and
// bench.py's cpu_baseline / --impl reference legs load this library as the
// CPU checker; the product library never links it.
//
// Array arguments are float32 buffers in the reference's layout
// a(0:ni+1, 0:nj+1, 1:nk), x fastest.  prec = 32 runs the restatement in
// float (like the reference's default `real`), prec = 64 in double.
#include <cstdint>
#include <cstring>
#include <vector>
#include "small.h"
#include "base.h"

using namespace oracle;

namespace {

// Order of the base-state array list passed by callers.
enum BaseIdx { B_JCB, B_JCB8U, B_JCB8V, B_JCB8W, B_RBR, B_PTBR, B_RST, B_RST8U, B_RST8V, B_RST8W,
               B_RCSQ, B_N };

Opts make_opts(const int* io, const double* ro) {
  Opts o;
  o.ni = io[0]; o.nj = io[1]; o.nk = io[2];
  o.divopt = io[3]; o.buyopt = io[4]; o.gwmopt = io[5];
  o.periodic = io[6]; o.bbc = io[7]; o.tbc = io[8]; o.fp64_solve = io[9]; o.impopt = io[10];
  o.dx = ro[0]; o.dy = ro[1]; o.dz = ro[2];
  o.weicoe = ro[3];
  return o;
}

template <class R>
void load_base(Base<R>& b, const Opts& o, const float* const* base) {
  b.resize(o.ni, o.nj, o.nk);
  b.jcb.load(base[B_JCB]); b.jcb8u.load(base[B_JCB8U]); b.jcb8v.load(base[B_JCB8V]);
  b.jcb8w.load(base[B_JCB8W]); b.rbr.load(base[B_RBR]); b.ptbr.load(base[B_PTBR]);
  b.rst.load(base[B_RST]); b.rst8u.load(base[B_RST8U]); b.rst8v.load(base[B_RST8V]);
  b.rst8w.load(base[B_RST8W]); b.rcsq.load(base[B_RCSQ]);
}

// s_smalldrv, SrcOrig/smalldrv.f90:343-398, HE-VI branch: the caller has
// already copied t-dt into the future arrays (smalldrv.f90:343-346), the
// contravariant w is rebuilt (smalldrv.f90:358), then nsstp substeps.
template <class R>
int run_small(const Opts& o, int sthopt, double dts, int nsstp, const float* const* base,
              const float* const* frc, float* const* st) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  Base<R> b;
  load_base(b, o, base);
  F3<R> ufrc(ni, nj, nk), vfrc(ni, nj, nk), wfrc(ni, nj, nk), pfrc(ni, nj, nk);
  ufrc.load(frc[0]); vfrc.load(frc[1]); wfrc.load(frc[2]); pfrc.load(frc[3]);
  F3<R> uf(ni, nj, nk), vf(ni, nj, nk), wf(ni, nj, nk), ppf(ni, nj, nk), wc(ni, nj, nk), ptpf(ni, nj, nk);
  uf.load(st[0]); vf.load(st[1]); wf.load(st[2]); ppf.load(st[3]);
  SmallScratch<R> s;
  s.resize(ni, nj, nk);
  phy2cnt(o, sthopt, b, wf, wc);
  for (int n = 0; n < nsstp; ++n)
    small_substep<R>(o, sthopt, (R)dts, b, ufrc, vfrc, wfrc, pfrc, ptpf, uf, vf, wf, wc, ppf, s);
  uf.store(st[0]); vf.store(st[1]); wf.store(st[2]); ppf.store(st[3]);
  return 0;
}

}  // namespace

extern "C" {

// io: ni,nj,nk,divopt,buyopt,gwmopt,periodic,bbc,tbc,fp64_solve,impopt
// ro: dx,dy,dz,weicoe
// base: B_N arrays (see BaseIdx); frc: ufrc,vfrc,wfrc,pfrc; st (in/out): uf,vf,wf,ppf
int oracle_small_steps(int prec, int sthopt, const int* io, const double* ro, double dts,
                       int nsstp, const float* const* base, const float* const* frc,
                       float* const* st) {
  Opts o = make_opts(io, ro);
  if (o.ni < 5 || o.nj < 5 || o.nk < 6) return 1;
  if (prec == 64) return run_small<double>(o, sthopt, dts, nsstp, base, frc, st);
  return run_small<float>(o, sthopt, dts, nsstp, base, frc, st);
}

// The base state from a height-level sounding (set1d, vextlow, intrpsnd,
// setbase/bcbase, baserho, sndwave; base.h) on one column.  snd: nlev
// levels each of z, u, v, pt (theta, or T when tvar == 't'), qv (RH in
// percent when hvar == 'r'); zph, jcb: nk+1 entries (index k).  out: 11
// columns of nk+1 entries (ubr, vbr, pbr, ptbr, qvbr, rbr, ptvbr, pibr,
// rst, rst8w, rcsq).  Returns 0, or 1 when the integration fails.
int oracle_base_state(int prec, int nk, const double* zph, const double* jcb, int nlev, const double* snd,
                      int tvar, int hvar, double psnd0, double thresq, double* out) {
  auto run = [&](auto one) -> int {
    using R = decltype(one);
    Sounding<R> s;
    s.nlev = nlev;
    for (auto* v : {&s.z, &s.u, &s.v, &s.p, &s.pt, &s.qv, &s.t}) v->assign(nlev + 1, R(0));
    for (int kl = 1; kl <= nlev; ++kl) {
      s.z[kl] = (R)snd[kl - 1];
      s.u[kl] = (R)snd[nlev + kl - 1];
      s.v[kl] = (R)snd[2 * nlev + kl - 1];
      s.pt[kl] = (R)snd[3 * nlev + kl - 1];
      s.qv[kl] = (R)snd[4 * nlev + kl - 1];
    }
    if (set1d_z<R>((char)tvar, (char)hvar, (R)psnd0, (R)thresq, s)) return 1;
    vextlow(s);
    std::vector<R> z(nk + 1), j(nk + 1);
    for (int k = 0; k <= nk; ++k) { z[k] = (R)zph[k]; j[k] = (R)jcb[k]; }
    BaseColumn<R> c;
    base_column(nk, z.data(), j.data(), s, c);
    const std::vector<R>* cols[11] = {&c.ubr, &c.vbr, &c.pbr, &c.ptbr, &c.qvbr, &c.rbr, &c.ptvbr, &c.pibr,
                                      &c.rst, &c.rst8w, &c.rcsq};
    for (int f = 0; f < 11; ++f)
      for (int k = 0; k <= nk; ++k) out[(size_t)f * (nk + 1) + k] = (double)(*cols[f])[k];
    return 0;
  };
  if (nlev < 3 || nk < 6) return 2;
  return prec == 64 ? run(0.0) : run(0.0f);
}

int oracle_abi_version(void) { return 1; }

}  // extern "C"

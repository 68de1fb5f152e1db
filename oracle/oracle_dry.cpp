// Oracle C entry point for whole dry large steps (ctypes-callable).
//
// TEST INFRASTRUCTURE ONLY: parity checker and CPU baseline; the product
// library never links it.
#include <cstring>
#include <vector>
#include "step.h"

using namespace oracle;

namespace {

template <class R>
int run_dry(const int* io, const double* ro, const double* zph, const float* const* base,
            float* const* st, int nsteps, double dtbig, double dtsml, int start) {
  DryRun<R> r;
  Opts& o = r.o;
  o.ni = io[0]; o.nj = io[1]; o.nk = io[2];
  o.divopt = io[3]; o.buyopt = io[4]; o.gwmopt = 0; o.periodic = 1; o.bbc = 2; o.tbc = 2;
  o.fp64_solve = io[5];
  r.sthopt = io[6];
  r.lo.smtopt = io[7];
  r.lo.vspopt = io[8];
  r.lo.coropt = io[9];
  r.lo.tubopt = io[10];
  o.impopt = io[11];
  o.obc = io[12];          // 0 periodic x, 4/5/7 open radiation x (wbc = ebc)
  o.advopt = io[13];       // 2 or 3 (4th-order vertical advection)
  o.gwave = ro[10];
  o.dx = ro[0]; o.dy = ro[1]; o.dz = ro[2]; o.weicoe = ro[3];
  r.lo.smhcoe = ro[4]; r.lo.smvcoe = ro[5]; r.lo.filcoe = ro[6];
  const double vspbar = ro[7], botbar = ro[8];
  r.fc = R(ro[9]);
  if (o.ni < 8 || o.nj < 8 || o.nk < 8) return 1;
  r.alloc();
  Base<R>& b = r.b;
  b.resize(o.ni, o.nj, o.nk);
  F3<R>* bl[] = {&b.jcb, &b.jcb8u, &b.jcb8v, &b.jcb8w, &b.rbr, &b.ptbr, &b.rst, &b.rst8u, &b.rst8v,
                 &b.rst8w, &b.rcsq, &b.ubr, &b.vbr};
  for (int n = 0; n < 13; ++n) bl[n]->load(base[n]);
  std::vector<double> z(zph, zph + o.nk + 1);
  r.lo.ksp0 = vspdmp<R>(o, z, vspbar, botbar, r.rbct);
  // st: past u, v, w, pp, ptp (+ tke with tubopt=2), then the present level
  auto slots = [&]() {
    std::vector<F3<R>*> v;
    for (Level<R>* L : {&r.p, &r.c}) {
      for (F3<R>* a : {&L->u, &L->v, &L->w, &L->pp, &L->ptp}) v.push_back(a);
      if (r.lo.tubopt == 2) v.push_back(&L->tke);
    }
    return v;
  };
  {
    const std::vector<F3<R>*> sl = slots();
    for (size_t n = 0; n < sl.size(); ++n) sl[n]->load(st[n]);
  }
  // slvstep.f90:176 nsstp; timeint.f90:160-190 half steps at the start
  const int nsstp = 20 * (int)(1.e2f * ((float)dtbig + .001f)) / (int)(1.e3f * ((float)dtsml + .0001f));
  for (int s = 0; s < nsteps; ++s) {
    const bool first = start && s == 0;
    const R dtb = first ? R(.5) * R(dtbig) : R(dtbig);
    const R dts = first ? R(.5) * R(dtsml) : R(dtsml);
    intgdrv_dry<R>(r, dtb, nsstp, dts, !first);   // no s_timeflt at ctime=0
  }
  const std::vector<F3<R>*> so = slots();
  for (size_t n = 0; n < so.size(); ++n) so[n]->store(st[n]);
  return 0;
}

}  // namespace

extern "C" {

// io: ni,nj,nk,divopt,buyopt,fp64_solve,sthopt,smtopt,vspopt,coropt,tubopt,impopt,obc,advopt
// ro: dx,dy,dz,weicoe,smhcoe,smvcoe,filcoe,vspbar,botbar,fc,gwave
// zph: w-level heights, index k = 1..nk (entry 0 unused)
// base: jcb,jcb8u,jcb8v,jcb8w,rbr,ptbr,rst,rst8u,rst8v,rst8w,rcsq,ubr,vbr
// st (in/out): past u,v,w,pp,ptp then present u,v,w,pp,ptp; with tubopt=2
//   each level's list ends with tke (12 arrays)
int oracle_dry_steps(int prec, const int* io, const double* ro, const double* zph,
                     const float* const* base, float* const* st, int nsteps, double dtbig,
                     double dtsml, int start) {
  if (prec == 64) return run_dry<double>(io, ro, zph, base, st, nsteps, dtbig, dtsml, start);
  return run_dry<float>(io, ro, zph, base, st, nsteps, dtbig, dtsml, start);
}

// s_vspdmp for vspopt=2 (vspdmp.f90:222-292) in float: rbct(k), k=1..nk
// into rbct[k]; returns ksp0(2).
int oracle_vspdmp(int nk, const double* zph, double vspbar, double botbar, float* rbct) {
  Opts o;
  o.nk = nk;
  std::vector<double> z(zph, zph + nk + 1);
  std::vector<float> r;
  const int ksp0 = vspdmp<float>(o, z, vspbar, botbar, r);
  for (int k = 0; k <= nk; ++k) rbct[k] = r[k];
  return ksp0;
}

}  // extern "C"

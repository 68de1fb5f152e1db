// Oracle C entry points for the cold-rain microphysics and whole moist
// large steps (ctypes-callable).
//
// TEST INFRASTRUCTURE ONLY: parity checker and CPU baseline; the product
// library never links it.
#include <algorithm>
#include <cmath>
#include <vector>
#include "moist_step.h"

using namespace oracle;

namespace {

// Field order of the state arrays passed in/out by oracle_cloudphy.
enum { P_PTP, P_QV, P_QC, P_QR, P_QI, P_QS, P_QG, P_NI, P_NS, P_NG, P_PP, NPAST };
enum { F_PTP, F_QV, F_QC, F_QR, F_QI, F_QS, F_QG, F_NI, F_NS, F_NG, NFUT };
enum { B_PTBR, B_RBR, B_PBR, B_JCB, B_RST, NBASE };

template <class R>
int run_cloudphy(int ni, int nj, int nk, double dtb_leap, double dz, double thresq,
                 const float* const* base, const float* const* past, float* const* fut, float* prec) {
  F3<R> b[NBASE], ptpp(ni, nj, nk), ppp(ni, nj, nk), ptpf(ni, nj, nk);
  for (int n = 0; n < NBASE; ++n) { b[n].resize(ni, nj, nk); b[n].load(base[n]); }
  MoistLevel<R> mp, mf;
  mp.resize(ni, nj, nk);
  mf.resize(ni, nj, nk);
  ptpp.load(past[P_PTP]);
  ppp.load(past[P_PP]);
  ptpf.load(fut[F_PTP]);
  for (int n = 0; n < M_N; ++n) {
    mp.q[n].load(past[P_QV + n]);
    mf.q[n].load(fut[F_QV + n]);
  }
  const size_t np = (size_t)10 * (ni + 2) * (nj + 2);
  std::vector<R> pr(prec, prec + np);
  const int npstp = cloudphy_fields<R>(ni, nj, nk, dz, R(thresq), R(dtb_leap), b[B_PTBR], b[B_RBR], b[B_PBR],
                                       b[B_JCB], b[B_RST], ptpp, ppp, mp, ptpf, mf, pr);
  ptpf.store(fut[F_PTP]);
  for (int n = 0; n < M_N; ++n) mf.q[n].store(fut[F_QV + n]);
  for (size_t n = 0; n < np; ++n) prec[n] = (float)pr[n];
  return npstp;
}

template <class R>
int run_moist(const int* io, const double* ro, const double* zph, const float* const* base,
              float* const* st, float* prec, int nsteps, double dtbig, double dtsml, int start) {
  MoistRun<R> m;
  DryRun<R>& r = m.r;
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
  o.gwave = ro[11];
  o.dx = ro[0]; o.dy = ro[1]; o.dz = ro[2]; o.weicoe = ro[3];
  r.lo.smhcoe = ro[4]; r.lo.smvcoe = ro[5]; r.lo.filcoe = ro[6];
  const double vspbar = ro[7], botbar = ro[8];
  r.fc = R(ro[9]);
  m.thresq = R(ro[10]);
  if (o.ni < 8 || o.nj < 8 || o.nk < 8) return -1;
  m.alloc();
  Base<R>& b = r.b;
  b.resize(o.ni, o.nj, o.nk);
  F3<R>* bl[] = {&b.jcb, &b.jcb8u, &b.jcb8v, &b.jcb8w, &b.rbr, &b.ptbr, &b.rst, &b.rst8u, &b.rst8v,
                 &b.rst8w, &b.rcsq, &b.ubr, &b.vbr, &b.pbr, &b.qvbr};
  for (int n = 0; n < 15; ++n) bl[n]->load(base[n]);
  std::vector<double> z(zph, zph + o.nk + 1);
  r.lo.ksp0 = vspdmp<R>(o, z, vspbar, botbar, r.rbct);
  // st: past u,v,w,pp,ptp,qv..ng (14), then present (14)
  auto slots = [&](Level<R>& L, MoistLevel<R>& M, std::vector<F3<R>*>& v) {
    for (F3<R>* a : {&L.u, &L.v, &L.w, &L.pp, &L.ptp}) v.push_back(a);
    for (auto& a : M.q) v.push_back(&a);
    if (r.lo.tubopt == 2) v.push_back(&L.tke);
  };
  std::vector<F3<R>*> sl;
  slots(r.p, m.mp, sl);
  slots(r.c, m.mc, sl);
  for (size_t n = 0; n < sl.size(); ++n) sl[n]->load(st[n]);
  const size_t np = (size_t)10 * (o.ni + 2) * (o.nj + 2);
  for (size_t n = 0; n < np; ++n) m.prec[n] = R(prec[n]);
  // slvstep.f90:176 nsstp; timeint.f90:160-190 half steps at ctime=0
  const int nsstp = 20 * (int)(1.e2f * ((float)dtbig + .001f)) / (int)(1.e3f * ((float)dtsml + .0001f));
  for (int s = 0; s < nsteps; ++s) {
    const bool first = start && s == 0;
    const R dtb = first ? R(.5) * R(dtbig) : R(dtbig);
    const R dts = first ? R(.5) * R(dtsml) : R(dtsml);
    intgdrv_moist<R>(m, dtb, nsstp, dts, !first);
  }
  std::vector<F3<R>*> so;
  slots(r.p, m.mp, so);
  slots(r.c, m.mc, so);
  for (size_t n = 0; n < so.size(); ++n) so[n]->store(st[n]);
  for (size_t n = 0; n < np; ++n) prec[n] = (float)m.prec[n];
  return m.npstp;
}

}  // namespace

extern "C" {

// One s_cloudphy call for cphopt=3 (cloudphy.f90:277-466).  dtb is the
// leapfrog step (the microphysics runs over 2*dtb).  base: ptbr, rbr, pbr,
// jcb, rst; past: ptp, qv, qc, qr, qi, qs, qg, ni, ns, ng, pp; fut (in/out):
// ptp, qv, qc, qr, qi, qs, qg, ni, ns, ng; prec (in/out): for prc, prr,
// pri, prs, prg the 2-D rate and accumulation planes, (ni+2)*(nj+2) each.
// Returns npstp (>0) or a negative error.
int oracle_cloudphy(int prec_bits, int ni, int nj, int nk, double dtb, double dz, double thresq,
                    const float* const* base, const float* const* past, float* const* fut,
                    float* prec) {
  if (ni < 5 || nj < 5 || nk < 6) return -1;
  if (prec_bits == 64) return run_cloudphy<double>(ni, nj, nk, dtb, dz, thresq, base, past, fut, prec);
  return run_cloudphy<float>(ni, nj, nk, dtb, dz, thresq, base, past, fut, prec);
}

// s_satadjst for cphopt=3 on whole arrays (siadjst + swadjst), range
// i=1..ni-1, j=1..nj-1, k=1..nk-1.  st (in/out): ptp, qv, qc, qi, ni; pp
// is the level's pressure perturbation (satadjst.f90:158).
void oracle_satadjst(int ni, int nj, int nk, double thresq, const float* ptbr, const float* pbr,
                     const float* pp, float* const* st) {
  F3<float> b(ni, nj, nk), p(ni, nj, nk), q(ni, nj, nk), a[5];
  b.load(ptbr);
  p.load(pbr);
  q.load(pp);
  for (int n = 0; n < 5; ++n) { a[n].resize(ni, nj, nk); a[n].load(st[n]); }
  satadjst_fields<float>(ni, nj, nk, (float)thresq, b, p, q, a[0], a[1], a[2], a[3], a[4]);
  for (int n = 0; n < 5; ++n) a[n].store(st[n]);
}

// Whole moist large steps (cphopt=3).
// io: ni,nj,nk,divopt,buyopt,fp64_solve,sthopt,smtopt,vspopt,coropt,tubopt,impopt,obc,advopt
// ro: dx,dy,dz,weicoe,smhcoe,smvcoe,filcoe,vspbar,botbar,fc,thresq,gwave
// base: jcb,jcb8u,jcb8v,jcb8w,rbr,ptbr,rst,rst8u,rst8v,rst8w,rcsq,ubr,vbr,pbr,qvbr
// st (in/out): past u,v,w,pp,ptp,qv,qc,qr,qi,qs,qg,ni,ns,ng then present (28);
//   with tubopt=2 each level's list ends with tke (30 arrays)
// prec (in/out): 10 precipitation planes.  Returns the last npstp.
int oracle_moist_steps(int prec_bits, const int* io, const double* ro, const double* zph,
                       const float* const* base, float* const* st, float* prec, int nsteps, double dtbig,
                       double dtsml, int start) {
  if (prec_bits == 64) return run_moist<double>(io, ro, zph, base, st, prec, nsteps, dtbig, dtsml, start);
  return run_moist<float>(io, ro, zph, base, st, prec, nsteps, dtbig, dtsml, start);
}

}  // extern "C"

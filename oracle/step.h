// Oracle: one leapfrog large step of the dry solver (s_intgdrv with
// s_fdmdrv, SrcOrig/intgdrv.f90:866-1119, SrcOrig/fdmdrv.f90:661-704).
//
// TEST INFRASTRUCTURE ONLY (see arr.h).
#pragma once
#include <vector>
#include "large.h"
#include "turb.h"

namespace oracle {

// Prognostic state of one time level (tke only with tubopt=2).
template <class R>
struct Level {
  F3<R> u, v, w, pp, ptp, tke;
  void resize(int ni, int nj, int nk, bool with_tke) {
    u.resize(ni, nj, nk); v.resize(ni, nj, nk); w.resize(ni, nj, nk);
    pp.resize(ni, nj, nk); ptp.resize(ni, nj, nk);
    if (with_tke) tke.resize(ni, nj, nk);
  }
};

template <class R>
struct DryRun {
  Opts o;
  LargeOpts lo;
  int sthopt = 0;
  Base<R> b;
  std::vector<R> rbct;   // vspdmp coefficient rbct(k,2)
  R fc = R(0);           // 0.5*omega*sin(lat)
  Level<R> p, c, f;      // t-dt, t, t+dt
  // moist buoyancy inputs at t (buoywb.f90:202-299); null for a dry run
  const F3<R>* bqv = nullptr;
  const F3<R>* bqall = nullptr;
  // Smagorinsky turbulence (tubopt=1): moist inputs at t-dt (bruntv.f90),
  // null for a dry run; the step's dtb (eddyvis.f90: ckmax = 0.125/dtb)
  const F3<R>* tqv = nullptr;
  const F3<R>* tqall = nullptr;
  R thresq = R(1.e-12);
  R dtb_cur = R(0);
  TurbWork<R> tw;
  Radiation<R> rad;      // phase speeds of the open x boundaries (o.obc != 0)
  // scratch
  F3<R> ufrc, vfrc, wfrc, pfrc, ptfrc, tkefrc, wc, rxu, rxv, rxw, t1, t2, t3, t4, t5, jxu, jxv, jxw;
  SmallScratch<R> ss;
  void alloc() {
    const int ni = o.ni, nj = o.nj, nk = o.nk;
    const bool tke = lo.tubopt == 2;
    p.resize(ni, nj, nk, tke); c.resize(ni, nj, nk, tke); f.resize(ni, nj, nk, tke);
    for (F3<R>* a : {&ufrc, &vfrc, &wfrc, &pfrc, &ptfrc, &wc, &rxu, &rxv, &rxw, &t1, &t2, &t3, &t4,
                     &t5, &jxu, &jxv, &jxw})
      a->resize(ni, nj, nk);
    if (tke) tkefrc.resize(ni, nj, nk);
    ss.resize(ni, nj, nk);
    if (lo.tubopt >= 1) tw.resize(ni, nj, nk);
    rad.resize(nj, nk);   // zero until the first s_phasev (a fresh start)
    o.rad = &rad;
  }
};

// s_forceuvw (forceuvw.f90:423-626) for tubopt=0, advopt=2: zero forcing,
// phy2cnt, smoo4uvw on the past level, vspuvw, coriuv, buoywb, rstuvwc,
// advuvw on the present level.
template <class R>
void forceuvw(DryRun<R>& r) {
  const Opts& o = r.o;
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  r.ufrc.fill(R(0)); r.vfrc.fill(R(0)); r.wfrc.fill(R(0));
  if (r.lo.tubopt >= 1) {                                               // forceuvw.f90:423-431, turbdrv.f90:245-287
    bruntv(o, r.tqv != nullptr, r.thresq, r.b, r.p.pp, r.p.ptp, r.tqv, r.tqall, r.tw);
    defomten(o, r.b, r.p.u, r.p.v, r.p.w, r.tw);
    if (r.lo.tubopt == 1)
      eddyvis(o, r.dtb_cur, r.b, r.tw);
    else
      eddyvis_tke(o, r.dtb_cur, r.b, r.p.tke, r.tw);
    strsten(o, r.tw);
    turbuvw(o, r.b, r.tw, r.ufrc, r.vfrc, r.wfrc);
  }
  phy2cnt(o, r.sthopt, r.b, r.c.w, r.wc);                               // forceuvw.f90:446
  if (r.lo.smtopt % 10 == 2 || r.lo.smtopt % 10 == 3) {                 // forceuvw.f90:469
    // smoo4uvw.f90:220-233: a = rst8u*(up-ubr)/jcb8u over k=1..nk-1, j=0..nj, i=0..ni+1
    for (int k = 1; k <= nk - 1; ++k)
      for (int j = 0; j <= nj; ++j)
        for (int i = 0; i <= ni + 1; ++i)
          r.t4(i, j, k) = r.b.rst8u(i, j, k) * (r.p.u(i, j, k) - r.b.ubr(i, j, k)) / r.b.jcb8u(i, j, k);
    smooth4(o, r.lo.smtopt, r.lo.smhcoe, r.lo.smvcoe, r.t4, 2, ni - 1, 2, nj - 2, 2, nk - 2, false,
            r.ufrc, r.t1, r.t2, r.t3);
    for (int k = 1; k <= nk - 1; ++k)                                   // smoo4uvw.f90:338-351
      for (int j = 0; j <= nj + 1; ++j)
        for (int i = 0; i <= ni; ++i)
          r.t4(i, j, k) = r.b.rst8v(i, j, k) * (r.p.v(i, j, k) - r.b.vbr(i, j, k)) / r.b.jcb8v(i, j, k);
    smooth4(o, r.lo.smtopt, r.lo.smhcoe, r.lo.smvcoe, r.t4, 2, ni - 2, 2, nj - 1, 2, nk - 2, false,
            r.vfrc, r.t1, r.t2, r.t3);
    for (int k = 1; k <= nk; ++k)                                       // smoo4uvw.f90:456-469
      for (int j = 0; j <= nj; ++j)
        for (int i = 0; i <= ni; ++i)
          r.t4(i, j, k) = r.b.rst8w(i, j, k) * r.p.w(i, j, k) / r.b.jcb8w(i, j, k);
    smooth4(o, r.lo.smtopt, r.lo.smhcoe, r.lo.smvcoe, r.t4, 2, ni - 2, 2, nj - 2, 2, nk - 1, true,
            r.wfrc, r.t1, r.t2, r.t3);
  }
  if (r.lo.vspopt >= 1)                                                 // forceuvw.f90:519
    vspuvw(o, r.lo, r.b, r.rbct, r.p.u, r.p.v, r.p.w, r.ufrc, r.vfrc, r.wfrc, r.t5);
  if (r.lo.coropt == 1) coriuv(o, r.fc, r.b, r.c.u, r.c.v, r.ufrc, r.vfrc, r.t1);   // :544
  buoywb(o, r.bqv != nullptr, r.b, r.c.ptp, r.bqv, r.bqall, r.wfrc, r.t1);   // forceuvw.f90:596
  rstuvwc(o, r.b, r.c.u, r.c.v, r.wc, r.rxu, r.rxv, r.rxw);             // :614
  advuvw(o, r.rxu, r.rxv, r.rxw, r.c.u, r.c.v, r.c.w, r.ufrc, r.vfrc, r.wfrc, r.t1, r.t2, r.t3, r.t4);  // :626
}

// s_forcep (forcep.f90:254-311): advp (J-weighted fluxes, advp.f90:249-291),
// smoo4p on the past level, vspp when vspvar(4:4)='o'.
template <class R>
void forcep(DryRun<R>& r) {
  const Opts& o = r.o;
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  for (int k = 1; k <= nk - 1; ++k) {                                   // advp.f90:255-277
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni; ++i) r.jxu(i, j, k) = r.b.jcb8u(i, j, k) * r.c.u(i, j, k);
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni - 1; ++i) r.jxv(i, j, k) = r.b.jcb8v(i, j, k) * r.c.v(i, j, k);
  }
  for (int k = 1; k <= nk; ++k)                                         // advp.f90:279-291
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) r.jxw(i, j, k) = r.b.jcb8w(i, j, k) * r.wc(i, j, k);
  advs(o, r.jxu, r.jxv, r.jxw, r.c.pp, r.pfrc, r.t1, r.t2, r.t3);
  if (r.lo.smtopt % 10 == 2 || r.lo.smtopt % 10 == 3)
    smooth4(o, r.lo.smtopt, r.lo.smhcoe, r.lo.smvcoe, r.p.pp, 2, ni - 2, 2, nj - 2, 2, nk - 2, false,
            r.pfrc, r.t1, r.t2, r.t3);
  if (r.lo.vspopt >= 1 && r.lo.vspvar[3] == 'o') vsp_scalar(o, r.lo.ksp0, r.rbct, r.b.jcb, r.p.pp, r.pfrc);
}

// s_forcept (forcept.f90:344-446), tubopt=0: advs, smoo4s on rbr*ptpp,
// vsps (rst-weighted), advbspt.
template <class R>
void forcept(DryRun<R>& r) {
  const Opts& o = r.o;
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  advs(o, r.rxu, r.rxv, r.rxw, r.c.ptp, r.ptfrc, r.t1, r.t2, r.t3);
  if (r.lo.smtopt % 10 == 2 || r.lo.smtopt % 10 == 3) {
    for (int k = 1; k <= nk - 1; ++k)                                   // smoo4s.f90:184-197
      for (int j = 0; j <= nj; ++j)
        for (int i = 0; i <= ni; ++i) r.t4(i, j, k) = r.b.rbr(i, j, k) * r.p.ptp(i, j, k);
    smooth4(o, r.lo.smtopt, r.lo.smhcoe, r.lo.smvcoe, r.t4, 2, ni - 2, 2, nj - 2, 2, nk - 2, false,
            r.ptfrc, r.t1, r.t2, r.t3);
  }
  if (r.lo.tubopt >= 1) {                                               // forcept.f90:313-320, 383-393
    F3<R>& pt = r.tw.ptv;   // free after bruntv: the full potential temperature at t-dt
    for (int k = 1; k <= nk - 1; ++k)
      for (int j = 1; j <= nj - 1; ++j)
        for (int i = 1; i <= ni - 1; ++i) pt(i, j, k) = r.b.ptbr(i, j, k) + r.p.ptp(i, j, k);
    turbs(o, r.b, pt, r.tw, r.ptfrc);
  }
  if (r.lo.vspopt >= 1 && r.lo.vspvar[4] == 'o') vsp_scalar(o, r.lo.ksp0, r.rbct, r.b.rst, r.p.ptp, r.ptfrc);
  advbspt(o, r.b, r.c.w, r.ptfrc, r.t1);
}

// s_vbcs, SrcOrig/vbcs.f90:116-132: zero-gradient scalar below the ground
// and above the lid.
template <class R>
void vbcs(const Opts& o, F3<R>& sf) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  for (int j = 1; j <= nj - 1; ++j)
    for (int i = 1; i <= ni - 1; ++i) sf(i, j, 1) = sf(i, j, 2);
  for (int j = 1; j <= nj - 1; ++j)
    for (int i = 1; i <= ni - 1; ++i) sf(i, j, nk - 1) = sf(i, j, nk - 2);
}

// s_forcetke (SrcOrig/forcetke.f90:269-354, smtopt 0/2/3, no lateral
// sponge): advs of the present TKE, shear production, 4th-order smoothing
// of rbr*tkep, dissipation, eddyvisj + tkeflx + turbtke, vsps0 when
// vspvar(10:10)='o', eddydif (the scalar diffusivities every later s_turbs
// uses) and the buoyancy production.
template <class R>
void forcetke(DryRun<R>& r) {
  const Opts& o = r.o;
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  advs(o, r.rxu, r.rxv, r.rxw, r.c.tke, r.tkefrc, r.t1, r.t2, r.t3);
  sheartke(o, r.b, r.tw, r.tkefrc);
  if (r.lo.smtopt % 10 == 2 || r.lo.smtopt % 10 == 3) {
    for (int k = 1; k <= nk - 1; ++k)                                   // smoo4s.f90:184-197
      for (int j = 0; j <= nj; ++j)
        for (int i = 0; i <= ni; ++i) r.t4(i, j, k) = r.b.rbr(i, j, k) * r.p.tke(i, j, k);
    smooth4(o, r.lo.smtopt, r.lo.smhcoe, r.lo.smvcoe, r.t4, 2, ni - 2, 2, nj - 2, 2, nk - 2, false,
            r.tkefrc, r.t1, r.t2, r.t3);
  }
  disptke(o, r.b, r.tw, r.p.tke, r.tkefrc);
  eddyvisj(o, r.b, r.tw);
  turbtke(o, r.b, r.p.tke, r.tw, r.tkefrc);
  if (r.lo.vspopt >= 1 && r.lo.vspvar[9] == 'o')                       // vsps0.f90:114-124
    for (int k = r.lo.ksp0 - 1; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 2; ++i)
          r.tkefrc(i, j, k) =
              r.tkefrc(i, j, k) - R(.5) * (r.rbct[k] + r.rbct[k + 1]) * r.b.rst(i, j, k) * r.p.tke(i, j, k);
  eddydif_tke(o, r.b, r.tw);
  buoytke(o, r.b, r.tw, r.tkefrc);
}

// Phases of one large step (s_intgdrv, intgdrv.f90:866-1119), split so
// the moist step can interleave its own parts.
template <class R>
void phase_forcing(DryRun<R>& r) {   // s_forcedrv (forcedrv.f90:548-608)
  forceuvw(r);
  if (r.lo.tubopt == 1) eddydif(r.o, r.b, r.tw);   // forcedrv.f90:565-570
  if (r.lo.tubopt == 2) forcetke(r);               // forcedrv.f90:576-592
  forcep(r);
  forcept(r);
}

template <class R>
void phase_small(DryRun<R>& r, int nsstp, R dts) {   // s_smalldrv (smalldrv.f90:343-398)
  r.f.u = r.p.u; r.f.v = r.p.v; r.f.w = r.p.w; r.f.pp = r.p.pp;
  phy2cnt(r.o, r.sthopt, r.b, r.f.w, r.wc);
  for (int n = 0; n < nsstp; ++n)
    small_substep<R>(r.o, r.sthopt, dts, r.b, r.ufrc, r.vfrc, r.wfrc, r.pfrc, r.f.ptp, r.f.u, r.f.v, r.f.w, r.wc,
            r.f.pp, r.ss);
}

// s_steps for one scalar (steps.f90:506-590): f = p + frc*2dtb/rst, clipped
// at zero for mixing ratios, the radiation boundaries of an open x domain
// (steps.f90:1024-1260; var, kind as in rbc_leapfrog, now = the present
// level), then bcycle (3979) and vbcs (4362).
template <class R>
void step_scalar(const DryRun<R>& r, R dtb, const F3<R>& sp, const F3<R>& frc, F3<R>& sf, bool clip,
                 int var = -1, int kind = 0, const F3<R>* now = nullptr) {
  const Opts& o = r.o;
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dtb2 = R(2) * dtb;
  for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) {
        const R dtdrst = dtb2 / r.b.rst(i, j, k);
        const R v = sp(i, j, k) + frc(i, j, k) * dtdrst;
        sf(i, j, k) = clip ? std::max(R(0), v) : v;
      }
  if (var >= 0 && now) rbc_leapfrog(o, r.b, var, kind, *now, sp, sf);
  bcycle(o, 2, 1, ni - 2, ni - 1, 2, 1, nj - 2, nj - 1, nk, sf);
  vbcs(o, sf);
}

template <class R>
void timeflt_field(const Opts& o, R filcoe, int ihi, int jhi, int khi, F3<R>& c, const F3<R>& f, const F3<R>& p) {
  const R m1fc2 = R(1) - R(2) * filcoe;
  for (int k = 1; k <= khi; ++k)
    for (int j = 1; j <= jhi; ++j)
      for (int i = 1; i <= ihi; ++i) c(i, j, k) = m1fc2 * c(i, j, k) + filcoe * (f(i, j, k) + p(i, j, k));
}

template <class R>
void phase_timeflt(DryRun<R>& r) {   // s_timeflt (timeflt.f90:335-404)
  const Opts& o = r.o;
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R fc = R(r.lo.filcoe);
  timeflt_field(o, fc, ni, nj - 1, nk - 1, r.c.u, r.f.u, r.p.u);
  timeflt_field(o, fc, ni - 1, nj, nk - 1, r.c.v, r.f.v, r.p.v);
  timeflt_field(o, fc, ni - 1, nj - 1, nk, r.c.w, r.f.w, r.p.w);
  timeflt_field(o, fc, ni - 1, nj - 1, nk - 1, r.c.pp, r.f.pp, r.p.pp);
  timeflt_field(o, fc, ni - 1, nj - 1, nk - 1, r.c.ptp, r.f.ptp, r.p.ptp);
  if (r.lo.tubopt == 2) {   // timeflt.f90:866-884: twice the coefficient for the TKE
    const R fc2 = R(2) * fc, m1fc4 = R(1) - R(4) * fc;
    for (int k = 1; k <= nk - 1; ++k)
      for (int j = 1; j <= nj - 1; ++j)
        for (int i = 1; i <= ni - 1; ++i)
          r.c.tke(i, j, k) = m1fc4 * r.c.tke(i, j, k) + fc2 * (r.f.tke(i, j, k) + r.p.tke(i, j, k));
  }
}

template <class R>
void phase_halo(DryRun<R>& r) {   // shift2nd on t and t+dt (intgdrv.f90:1005,1013)
  for (Level<R>* L : {&r.c, &r.f}) {
    halo_both(r.o, 'u', L->u); halo_both(r.o, 'v', L->v); halo_both(r.o, 's', L->w);
    halo_both(r.o, 's', L->pp); halo_both(r.o, 's', L->ptp);
    if (r.lo.tubopt == 2) halo_both(r.o, 's', L->tke);
  }
}

// s_phasev (intgdrv.f90:1023-1056) for u, v, w, p' ('sml': scaled to the
// small step) and theta' ('big', gwmopt=0), from the filtered present,
// the past and the future level (phasev.f90:464-500).
template <class R>
void phasev_dry(DryRun<R>& r, R dtb, R dts) {
  const Opts& o = r.o;
  if (!o.obc) return;
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  phase_var(o, RV_U, true, ni - 1, nj - 1, nk - 2, dtb, dts, r.c.u, r.p.u, r.f.u, r.rad);
  phase_var(o, RV_V, true, ni - 2, nj, nk - 2, dtb, dts, r.c.v, r.p.v, r.f.v, r.rad);
  phase_var(o, RV_W, true, ni - 2, nj - 1, nk - 1, dtb, dts, r.c.w, r.p.w, r.f.w, r.rad);
  phase_var(o, RV_P, true, ni - 2, nj - 1, nk - 2, dtb, dts, r.c.pp, r.p.pp, r.f.pp, r.rad);
  phase_var(o, RV_PT, false, ni - 2, nj - 1, nk - 2, dtb, dts, r.c.ptp, r.p.ptp, r.f.ptp, r.rad);
}

// One dry large step (leapfrog from t-dt to t+dt with dtb, nsstp
// substeps of dts): forcing, small steps, s_steps for theta', s_timeflt
// (skipped on the first step, ctime=0: intgdrv.f90:968), shift2nd planes
// and the swp2nxt rotation.
template <class R>
void intgdrv_dry(DryRun<R>& r, R dtb, int nsstp, R dts, bool filter) {
  r.dtb_cur = dtb;
  phase_forcing(r);
  phase_small(r, nsstp, dts);
  step_scalar(r, dtb, r.p.ptp, r.ptfrc, r.f.ptp, false, RV_PT, 0, &r.c.ptp);
  if (r.lo.tubopt == 2) step_scalar(r, dtb, r.p.tke, r.tkefrc, r.f.tke, true);   // steps.f90:999-1014
  if (filter) phase_timeflt(r);
  phase_halo(r);
  phasev_dry(r, dtb, dts);
  std::swap(r.p, r.c);   // swp2nxt: past <- t, t <- t+dt
  std::swap(r.c, r.f);
}

}  // namespace oracle

// Oracle: the cold-rain (cphopt=3, haiopt=0) parts of a large step and the
// moist leapfrog step driver (s_intgdrv for fmois='moist').
//
// TEST INFRASTRUCTURE ONLY (see arr.h).
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>
#include "micro.h"
#include "step.h"

namespace oracle {

// Moist species in the order the C-ABI and the tests use.
enum MoistIdx { M_QV = 0, M_QC, M_QR, M_QI, M_QS, M_QG, M_NI, M_NS, M_NG, M_N };

template <class R>
struct MoistLevel {
  F3<R> q[M_N];
  void resize(int ni, int nj, int nk) {
    for (auto& a : q) a.resize(ni, nj, nk);
  }
};

// s_upwqp (SrcOrig/upwqp.f90:149-225, advopt<=3) / s_upwnp (upwnp.f90:
// 132-176) on one column with flux rbr*u*q; precip (rate, accumulated)
// when given.
template <class R>
void upw_column(int nk, R dziv, R dtp, const R* rbr, const R* rst, const R* u, R* q, R* flx, R* precip) {
  const R dzvdt = dziv * dtp;
  for (int k = 1; k <= nk - 1; ++k) flx[k] = rbr[k] * u[k] * q[k];
  for (int k = 1; k <= nk - 2; ++k) q[k] = std::max(q[k] + (flx[k + 1] - flx[k]) / rst[k] * dzvdt, R(0));
  q[nk - 1] = q[nk - 2];
  if (precip) {
    const R rwiv05 = R(.5) / R(MP::rhow);
    const R dtp05 = R(.5) * dtp;
    precip[0] = (flx[1] + flx[2]) * rwiv05;
    precip[1] = precip[1] + precip[0] * dtp05;
  }
}

// s_cloudphy for cphopt=3 (SrcOrig/cloudphy.f90:277-466 -> s_coldblk,
// coldblk.f90:321-481) on whole arrays over i=1..ni-1, j=1..nj-1,
// k=1..nk-1.  Process rates come from the past level (ptpp, ppp, mp),
// applied to the future level (ptpf, mf).  prec holds, for prc, prr, pri,
// prs, prg, the (rate, accumulation) planes of (ni+2)*(nj+2).  dtb_leap is
// the leapfrog step; the scheme integrates over 2*dtb_leap.  Returns npstp.
template <class R>
int cloudphy_fields(int ni, int nj, int nk, double dz, R thresq, R dtb_leap, const F3<R>& ptbr,
                    const F3<R>& rbr, const F3<R>& pbr, const F3<R>& jcb, const F3<R>& rst,
                    const F3<R>& ptpp, const F3<R>& ppp, const MoistLevel<R>& mp, F3<R>& ptpf,
                    MoistLevel<R>& mf, std::vector<R>& prec) {
  const R dtb = R(2) * dtb_leap;   // cloudphy.f90:282 dtb_sub
  const R dziv = R(1) / R(dz);
  const Koenig<R> kt;
  const size_t plane = (size_t)(ni + 2) * (nj + 2);
  std::vector<Cell<R>> cells(plane * nk);
  const R rddvcp = R(Phys::rd) / R(Phys::cp), p0iv = R(1) / R(Phys::p0);
  auto idx = [&](int i, int j, int k) {
    return (size_t)i + (size_t)(ni + 2) * ((size_t)j + (size_t)(nj + 2) * (size_t)(k - 1));
  };
  auto each = [&](auto fn) {
    OMP_FOR for (int k = 1; k <= nk - 1; ++k)
      for (int j = 1; j <= nj - 1; ++j)
        for (int i = 1; i <= ni - 1; ++i) fn(i, j, k, cells[idx(i, j, k)]);
  };
  each([&](int i, int j, int k, Cell<R>& c) {
    c.ptbr = ptbr(i, j, k); c.rbr = rbr(i, j, k);
    c.rbv = R(1) / c.rbr;                                                     // getvdens.f90:106
    c.p = pbr(i, j, k) + ppp(i, j, k);                                        // getexner.f90:129
    c.pi = std::exp(rddvcp * std::log(p0iv * c.p));                           // getexner.f90:131
    c.ptpp = ptpp(i, j, k);
    c.qvp = mp.q[M_QV](i, j, k); c.qcp = mp.q[M_QC](i, j, k); c.qrp = mp.q[M_QR](i, j, k);
    c.qip = mp.q[M_QI](i, j, k); c.qsp = mp.q[M_QS](i, j, k); c.qgp = mp.q[M_QG](i, j, k);
    c.ncip = mp.q[M_NI](i, j, k); c.ncsp = mp.q[M_NS](i, j, k); c.ncgp = mp.q[M_NG](i, j, k);
    diagnw_cell(c.rbr, c.qrp, c.nccp, c.ncrp);                                // cloudphy.f90:366
    c.ptpf = ptpf(i, j, k);
    c.qvf = mf.q[M_QV](i, j, k); c.qcf = mf.q[M_QC](i, j, k); c.qrf = mf.q[M_QR](i, j, k);
    c.qif = mf.q[M_QI](i, j, k); c.qsf = mf.q[M_QS](i, j, k); c.qgf = mf.q[M_QG](i, j, k);
    c.ncif = mf.q[M_NI](i, j, k); c.ncsf = mf.q[M_NS](i, j, k); c.ncgf = mf.q[M_NG](i, j, k);
  });
  auto adj = [&](int, int, int, Cell<R>& c) {
    adjstni_cell(c.rbr, c.rbv, c.qif, c.qsf, c.qgf, c.ncif, c.ncsf, c.ncgf);
  };
  each(adj);                                                                   // coldblk.f90:327
  each([&](int, int, int, Cell<R>& c) { termblk_cell(thresq, c); });          // coldblk.f90:344
  each([&](int, int, int, Cell<R>& c) { srcblk_cell(dtb, thresq, kt, c); });  // coldblk.f90:356
  each(adj);                                                                   // coldblk.f90:425
  // s_fallblk (fallblk.f90:298-449): the sub-step is the domain minimum
  // of dz*jcb/(terminal speed) over all species (chkfall), per level first.
  const R eps = R(MP::eps);
  std::vector<R> kmin((size_t)(nk + 1) * 5, dtb);
  OMP_FOR for (int k = 1; k <= nk - 1; ++k) {
    R* m = &kmin[(size_t)k * 5];
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) {
        const Cell<R>& c = cells[idx(i, j, k)];
        const R dzjcb = R(dz) * jcb(i, j, k);
        m[0] = std::min(dzjcb / (c.ucq + eps), m[0]);
        m[1] = std::min(dzjcb / (c.urq + eps), m[1]);
        m[2] = std::min(dzjcb / (c.uiq + eps), m[2]);
        m[3] = std::min(dzjcb / (c.usq + eps), m[3]);
        m[4] = std::min(dzjcb / (c.ugq + eps), m[4]);
      }
  }
  R dtpc = dtb, dtpr = dtb, dtpi = dtb, dtps = dtb, dtpg = dtb;
  for (int k = 1; k <= nk - 1; ++k) {
    const R* m = &kmin[(size_t)k * 5];
    dtpc = std::min(m[0], dtpc); dtpr = std::min(m[1], dtpr); dtpi = std::min(m[2], dtpi);
    dtps = std::min(m[3], dtps); dtpg = std::min(m[4], dtpg);
  }
  R dtp = std::min(std::min(std::min(dtpc, dtpr), std::min(dtpi, dtps)), dtpg);
  int npstp;
  if (dtp < dtb) {
    npstp = (int)((dtb + R(.001)) / dtp) + 1;
    dtp = dtb / R(npstp);
  } else {
    npstp = 1;
    dtp = dtb;
  }
  OMP_FOR for (int j = 1; j <= nj - 1; ++j) {
    std::vector<R> rb(nk + 1), rs(nk + 1), u(nk + 1), q(nk + 1), flx(nk + 1);
    for (int i = 1; i <= ni - 1; ++i) {
      for (int k = 1; k <= nk - 1; ++k) { rb[k] = rbr(i, j, k); rs[k] = rst(i, j, k); }
      auto col = [&](R Cell<R>::*uf, R Cell<R>::*qf, int pslot) {
        for (int k = 1; k <= nk - 1; ++k) { u[k] = cells[idx(i, j, k)].*uf; q[k] = cells[idx(i, j, k)].*qf; }
        R pr[2] = {R(0), R(0)};
        const size_t p0 = (size_t)(2 * std::max(pslot, 0)) * plane + idx(i, j, 1), p1 = p0 + plane;
        if (pslot >= 0) { pr[0] = prec[p0]; pr[1] = prec[p1]; }
        for (int s = 0; s < npstp; ++s)
          upw_column(nk, dziv, dtp, rb.data(), rs.data(), u.data(), q.data(), flx.data(),
                     pslot >= 0 ? pr : nullptr);
        for (int k = 1; k <= nk - 1; ++k) cells[idx(i, j, k)].*qf = q[k];
        if (pslot >= 0) { prec[p0] = pr[0]; prec[p1] = pr[1]; }
      };
      // fallblk.f90:455-487 (cloud water, cloud ice, ice number) then
      // 489-524 (rain, snow, graupel, snow and graupel numbers).  Each
      // species' sub-steps touch only that species, so running them field
      // by field equals the reference's sub-step-major order.
      col(&Cell<R>::ucq, &Cell<R>::qcf, 0);
      col(&Cell<R>::uiq, &Cell<R>::qif, 2);
      col(&Cell<R>::uin, &Cell<R>::ncif, -1);
      col(&Cell<R>::urq, &Cell<R>::qrf, 1);
      col(&Cell<R>::usq, &Cell<R>::qsf, 3);
      col(&Cell<R>::ugq, &Cell<R>::qgf, 4);
      col(&Cell<R>::usn, &Cell<R>::ncsf, -1);
      col(&Cell<R>::ugn, &Cell<R>::ncgf, -1);
    }
  }
  each(adj);                                                                   // coldblk.f90:469
  each([&](int i, int j, int k, Cell<R>& c) {
    ptpf(i, j, k) = c.ptpf;
    mf.q[M_QV](i, j, k) = c.qvf; mf.q[M_QC](i, j, k) = c.qcf; mf.q[M_QR](i, j, k) = c.qrf;
    mf.q[M_QI](i, j, k) = c.qif; mf.q[M_QS](i, j, k) = c.qsf; mf.q[M_QG](i, j, k) = c.qgf;
    mf.q[M_NI](i, j, k) = c.ncif; mf.q[M_NS](i, j, k) = c.ncsf; mf.q[M_NG](i, j, k) = c.ncgf;
  });
  return npstp;
}

// s_satadjst for cphopt=3 (SrcOrig/satadjst.f90:154-189: s_siadjst then
// s_swadjst) over i=1..ni-1, j=1..nj-1, k=1..nk-1 of one time level, with
// that level's p' (satadjst.f90:158 getexner).
template <class R>
void satadjst_fields(int ni, int nj, int nk, R thresq, const F3<R>& ptbr, const F3<R>& pbr, const F3<R>& pp,
                     F3<R>& ptp, F3<R>& qv, F3<R>& qc, F3<R>& qi, F3<R>& nci) {
  const R rddvcp = R(Phys::rd) / R(Phys::cp), p0iv = R(1) / R(Phys::p0);
  OMP_FOR for (int k = 1; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) {
        const R p = pbr(i, j, k) + pp(i, j, k);
        const R pi = std::exp(rddvcp * std::log(p0iv * p));
        satadjst_cell<R>(thresq, ptbr(i, j, k), pi, p, ptp(i, j, k), qv(i, j, k), qc(i, j, k), qi(i, j, k),
                         nci(i, j, k));
      }
}

template <class R>
struct MoistRun {
  DryRun<R> r;
  MoistLevel<R> mp, mc, mf;
  F3<R> qall, qallp, qfrc;
  std::vector<R> prec;   // 5 species x (rate, accumulation) planes
  R thresq = R(1.e-12);
  int npstp = 0;         // sedimentation sub-steps of the last step
  void alloc() {
    const int ni = r.o.ni, nj = r.o.nj, nk = r.o.nk;
    r.alloc();
    mp.resize(ni, nj, nk); mc.resize(ni, nj, nk); mf.resize(ni, nj, nk);
    qall.resize(ni, nj, nk); qallp.resize(ni, nj, nk); qfrc.resize(ni, nj, nk);
    prec.assign((size_t)10 * (ni + 2) * (nj + 2), R(0));
  }
};

// Forcing and s_steps of one moist scalar (s_forceqv, SrcOrig/forceqv.f90:
// 290-374, for qv; s_forceq, forceq.f90:384-1941, for the species): advs
// on the present level, 4th-order smoothing of rbr*(qvp-qvbr) or rbr*sp on
// the past level (smoo4qv / smoo4s), Rayleigh damping of (qvp-qvbr) or sp
// (vspqv.f90:181-198, vsps.f90:181-198, vsps0.f90:114-124), then the
// leapfrog step, clipped at zero for the mixing ratios only
// (steps.f90:590-764).
template <class R>
void moist_scalar(MoistRun<R>& m, int n, R dtb) {
  DryRun<R>& r = m.r;
  const Opts& o = r.o;
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const F3<R>& sc = m.mc.q[n];
  const F3<R>& sp = m.mp.q[n];
  const bool isqv = n == M_QV;
  advs(o, r.rxu, r.rxv, r.rxw, sc, m.qfrc, r.t1, r.t2, r.t3);
  if (r.lo.smtopt % 10 == 2 || r.lo.smtopt % 10 == 3) {
    OMP_FOR for (int k = 1; k <= nk - 1; ++k)
      for (int j = 0; j <= nj; ++j)
        for (int i = 0; i <= ni; ++i)
          r.t4(i, j, k) = isqv ? r.b.rbr(i, j, k) * (sp(i, j, k) - r.b.qvbr(i, j, k)) : r.b.rbr(i, j, k) * sp(i, j, k);
    smooth4(o, r.lo.smtopt, r.lo.smhcoe, r.lo.smvcoe, r.t4, 2, ni - 2, 2, nj - 2, 2, nk - 2, false, m.qfrc,
            r.t1, r.t2, r.t3);
  }
  if (r.lo.tubopt >= 1) turbs(o, r.b, sp, r.tw, m.qfrc);   // forceqv.f90:331-345, forceq.f90:438-452
  const char sw = isqv ? r.lo.vspvar[5] : r.lo.vspvar[6];
  if (r.lo.vspopt >= 1 && sw == 'o') {
    OMP_FOR for (int k = r.lo.ksp0 - 1; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 2; ++i) {
          const R d = isqv ? sp(i, j, k) - r.b.qvbr(i, j, k) : sp(i, j, k);
          m.qfrc(i, j, k) = m.qfrc(i, j, k) - R(.5) * (r.rbct[k] + r.rbct[k + 1]) * r.b.rst(i, j, k) * d;
        }
  }
  step_scalar(r, dtb, sp, m.qfrc, m.mf.q[n], n < M_NI, RV_QV + n, n == M_QV ? 1 : n < M_NI ? 2 : 3, &sc);
}

// One moist large step (s_intgdrv, SrcOrig/intgdrv.f90:832-1119 with
// fmois='moist', advopt=2, cphopt=3): totalqwi at t (832-846), forcing with
// moist buoyancy (s_forcedrv -> buoywb with qv, qall at t), small steps,
// s_steps for theta', qv and the nine species, s_cloudphy (940-953),
// s_timeflt unless it is the first step (968-983), s_satadjst on t and
// t+dt (985-998), shift2nd planes (1003-1020) and swp2nxt.
template <class R>
void intgdrv_moist(MoistRun<R>& m, R dtb, int nsstp, R dts, bool filter) {
  DryRun<R>& r = m.r;
  const Opts& o = r.o;
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  for (size_t n = 0; n < m.qall.size(); ++n)   // totalqwi.f90:163-164
    m.qall.d[n] = m.mc.q[M_QC].d[n] + m.mc.q[M_QR].d[n] + m.mc.q[M_QI].d[n] + m.mc.q[M_QS].d[n] +
                  m.mc.q[M_QG].d[n];
  r.bqv = &m.mc.q[M_QV];
  r.bqall = &m.qall;
  for (size_t n = 0; n < m.qallp.size(); ++n)   // totalqwi at t-dt (intgdrv.f90:841)
    m.qallp.d[n] = m.mp.q[M_QC].d[n] + m.mp.q[M_QR].d[n] + m.mp.q[M_QI].d[n] + m.mp.q[M_QS].d[n] +
                   m.mp.q[M_QG].d[n];
  r.tqv = &m.mp.q[M_QV];
  r.tqall = &m.qallp;
  r.thresq = m.thresq;
  r.dtb_cur = dtb;
  phase_forcing(r);
  phase_small(r, nsstp, dts);
  step_scalar(r, dtb, r.p.ptp, r.ptfrc, r.f.ptp, false, RV_PT, 0, &r.c.ptp);
  if (r.lo.tubopt == 2) step_scalar(r, dtb, r.p.tke, r.tkefrc, r.f.tke, true);   // steps.f90:999-1014
  for (int n = 0; n < M_N; ++n) moist_scalar(m, n, dtb);
  m.npstp = cloudphy_fields(ni, nj, nk, o.dz, m.thresq, dtb, r.b.ptbr, r.b.rbr, r.b.pbr, r.b.jcb, r.b.rst,
                            r.p.ptp, r.p.pp, m.mp, r.f.ptp, m.mf, m.prec);
  if (filter) {
    phase_timeflt(r);
    for (int n = 0; n < M_N; ++n)   // timeflt.f90:405-520
      timeflt_field(o, R(r.lo.filcoe), ni - 1, nj - 1, nk - 1, m.mc.q[n], m.mf.q[n], m.mp.q[n]);
  }
  for (int lvl = 0; lvl < 2; ++lvl) {
    Level<R>& L = lvl == 0 ? r.c : r.f;
    MoistLevel<R>& M = lvl == 0 ? m.mc : m.mf;
    satadjst_fields(ni, nj, nk, m.thresq, r.b.ptbr, r.b.pbr, L.pp, L.ptp, M.q[M_QV], M.q[M_QC], M.q[M_QI],
                    M.q[M_NI]);
  }
  phase_halo(r);
  for (MoistLevel<R>* M : {&m.mc, &m.mf})
    for (auto& a : M->q) halo_both(o, 's', a);
  if (o.obc) {   // phasev.f90:506-800 ('big' for qv and the species)
    phasev_dry(r, dtb, dts);
    for (int n = 0; n < M_N; ++n)
      phase_var(o, RV_QV + n, false, ni - 2, nj - 1, nk - 2, dtb, dts, m.mc.q[n], m.mp.q[n], m.mf.q[n], r.rad);
  }
  std::swap(r.p, r.c);
  std::swap(r.c, r.f);
  std::swap(m.mp, m.mc);
  std::swap(m.mc, m.mf);
  r.bqv = nullptr;
  r.bqall = nullptr;
  r.tqv = nullptr;
  r.tqall = nullptr;
}

}  // namespace oracle

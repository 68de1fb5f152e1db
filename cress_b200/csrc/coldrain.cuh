// Per-cell cold-rain bulk microphysics (cphopt=3, haiopt=0) for the
// device: s_diagnw, s_adjstni, s_termblk, s_srcblk (s_setblk and the
// process routines through s_more0q and s_newblk) and s_satadjst
// (s_siadjst + s_swadjst), with the temparam.f90 switches of the default
// build (SrcDevelop/0rig/UserModAdd/temparam.f90: evapor_opt=1,
// nuc2nd_opt=1, flqcqi_opt=1).  Every function names the reference lines
// it follows; arithmetic is float with the CUDA math library.
#pragma once
#include <cuda_runtime.h>

namespace cress {

typedef float R;
constexpr float kGrav = 9.8f, kCpAir = 1004.f;   // SrcOrig/comphy.f90:49,61

// Koenig coefficients of ice depositional growth (SrcOrig/setref.f90:
// 473-601), ckoe pre-multiplied by exp(3*pkoe*ln10) as setref does; set by
// the host (micro.cu, micro_init_tables) before the first launch.  This
// header is included by micro.cu only.
__constant__ float kKoeC[41];
__constant__ float kKoeP[41];

struct MP {  // SrcOrig/comphy.f90:49-459, SrcOrig/commath.f90:42-192
  static constexpr double cc = 3.141592, oned3 = 1.0 / 3.0, oned6 = 1.0 / 6.0, oned9 = 1.0 / 9.0;
  static constexpr double sevnd3 = 7.0 / 3.0, ln10 = 2.30259;
  static constexpr double gf4 = 6.0, gf7 = 720.0, gfbus = 1.77245, hfbus = 1610.0, eps = 1.e-20;
  static constexpr double gf1bur = .931384, gf1bus = .886227, gf1bug = .898642;
  static constexpr double gf3bur = 4.69417, gf3bus = 3.32335, gf3bug = 3.89076;
  static constexpr double gf4bur = 17.8379, gf4bus = 11.6314, gf4bug = 14.1624;
  static constexpr double gf5bur = 1.82736, gf5bus = 1.60836, gf5bug = 1.70506;
  static constexpr double cw = 4.218e3, ci = 2.106e3, rv = 461.0, epsva = .622, epsav = 1.6077;
  static constexpr double es0 = 610.78, r0 = 1.225, t0 = 273.16, tlow = 233.16, t0cel = 0.0;
  static constexpr double t20 = 293.16, t23 = 296.16, p20 = 101325.0, lmb20 = 6.6e-8;
  static constexpr double diasl = 6.e-7, boltz = 1.38066e-23, sc = .6, lv0 = 2.50078e6;
  static constexpr double lf0 = 3.34e5, kp0 = 10.79, kpa = 2.4e-1, nu0 = 1.328e-5, dv0 = 2.23e-5;
  static constexpr double xl = .25, nclcst = 1.e8, nr0 = 8.e6, ns0 = 1.8e6, ng0 = 1.1e6;
  static constexpr double aur = 842.0, aui = 770.0, aus = 27.0, aug = 132.0;
  static constexpr double bur = .8, bus = .5, bug = .64;
  static constexpr double gur = .5, gus = .5, gug = .5;
  static constexpr double rhow = 1.e3, rhoi = 2.e2, rhos = 1.e2, rhog = 4.e2;
  static constexpr double ers = 1.0, erg = 1.0, eir = 1.0, eis = .1, eig = .1, esr = 1.0, esg = .001;
  static constexpr double ecc = .55, eii = .1, ess = .1;
  static constexpr double mr0 = 2.7e-10, mi0 = 1.e-12, ms0 = 1.76e-10, mg0 = 7.e-10;
  static constexpr double mrmax = 2.68e-4, mimax = 1.4e-10, msmax = 6.e-4, mgmax = 8.e-3;
  static constexpr double diaqcm = 2.e-5;
  // temparam.f90 (SrcDevelop/0rig/UserModAdd)
  static constexpr double ucqcst = .1, ucncst = .1, uiqcst = .0001, uincst = .0001;
};

// Per-cell state seen by the cold-rain routines.
struct MCell {
  // base state and thermodynamics (getvdens/getexner, cloudphy.f90:291-297)
  R ptbr, rbr, rbv, pi, p;
  // past level (t-dt): the process rates are formed from these
  R ptpp, qvp, qcp, qrp, qip, qsp, qgp, nccp, ncrp, ncip, ncsp, ncgp;
  // future level (t+dt), updated
  R ptpf, qvf, qcf, qrf, qif, qsf, qgf, ncif, ncsf, ncgf;
  // fall speeds of the past level (termblk)
  R ucq, urq, uiq, usq, ugq, ucn, urn, uin, usn, ugn;
};

// sqrt(sqrt(x)); for x = +-0 it returns x, which is what the two square
// roots give there, without taking the square root's special-operand path
// (clear-air cells have zero hydrometeors, so most calls see a zero).
__device__ __forceinline__ R root4(R x) { return x == R(0) ? x : sqrtf(sqrtf(x)); }

// s_diagnw, SrcOrig/diagnw.f90:120-160: diagnosed cloud and rain numbers.
__device__ inline void diagnw_cell(R rbr, R qr, R& ncc, R& ncr) {
  const R mrmiv2 = R(1.e-2) / R(MP::mrmax), mr0iv2 = R(1.e2) / R(MP::mr0);
  const R cdiaqr = R(MP::nr0) * R(MP::nr0) * R(MP::nr0) / (R(MP::cc) * R(MP::rhow));
  const R rbv = R(1) / rbr;
  ncc = R(MP::nclcst) * rbv;
  ncr = root4(cdiaqr * rbr * qr) * rbv;
  ncr = fminf(fmaxf(ncr, mrmiv2 * qr), mr0iv2 * qr);
}

// s_adjstni haiopt=0, SrcOrig/adjstni.f90:166-220.
__device__ inline void adjstni_cell(R rbr, R rbv, R qi, R qs, R qg, R& nci, R& ncs, R& ncg) {
  const R mimiv5 = R(.5) / R(MP::mimax), mi0iv2 = R(1.e2) / R(MP::mi0);
  const R msmiv2 = R(1.e-2) / R(MP::msmax), ms0iv2 = R(1.e2) / R(MP::ms0);
  const R mgmiv2 = R(1.e-2) / R(MP::mgmax), mg0iv2 = R(1.e2) / R(MP::mg0);
  const R cdiaqs = R(MP::ns0) * R(MP::ns0) * R(MP::ns0) / (R(MP::cc) * R(MP::rhos));
  const R cdiaqg = R(MP::ng0) * R(MP::ng0) * R(MP::ng0) / (R(MP::cc) * R(MP::rhog));
  nci = fminf(fmaxf(nci, mimiv5 * qi), mi0iv2 * qi);
  R ndia = root4(cdiaqs * rbr * qs) * rbv;
  ncs = fmaxf(fmaxf(ncs, msmiv2 * qs), R(5.62341e-3) * ndia);
  ncs = fminf(fminf(ncs, ms0iv2 * qs), R(1.77838e2) * ndia);
  ndia = root4(cdiaqg * rbr * qg) * rbv;
  ncg = fmaxf(fmaxf(ncg, mgmiv2 * qg), R(5.62341e-3) * ndia);
  ncg = fminf(fminf(ncg, mg0iv2 * qg), R(1.77838e2) * ndia);
}

// s_termblk cphopt=3, haiopt=0, flqcqi_opt=1, SrcOrig/termblk.f90:267-500.
__device__ inline void termblk_cell(R thresq, MCell& c) {
  const R oned3 = R(MP::oned3), oned6 = R(MP::oned6);
  const R bur3 = oned3 * R(MP::bur), bus3 = oned3 * R(MP::bus), bug3 = oned3 * R(MP::bug);
  const R curq = oned6 * R(MP::aur) * R(MP::gf4bur), cusq = oned6 * R(MP::aus) * R(MP::gf4bus);
  const R cugq = oned6 * R(MP::aug) * R(MP::gf4bug);
  const R curn = R(6) * R(MP::gf1bur) / R(MP::gf4bur), cusn = R(6) * R(MP::gf1bus) / R(MP::gf4bus);
  const R cugn = R(6) * R(MP::gf1bug) / R(MP::gf4bug);
  const R cdiaqr = R(1) / (R(MP::cc) * R(MP::rhow)), cdiaqs = R(1) / (R(MP::cc) * R(MP::rhos));
  const R cdiaqg = R(1) / (R(MP::cc) * R(MP::rhog));
  if (c.qcp > thresq) { c.ucq = R(MP::ucqcst); c.ucn = R(MP::ucncst); } else { c.ucq = R(0); c.ucn = R(0); }
  if (c.qip > thresq) { c.uiq = R(MP::uiqcst); c.uin = R(MP::uincst); } else { c.uiq = R(0); c.uin = R(0); }
  const R lnr0r = logf(R(MP::r0) * c.rbv);
  if (c.qrp > thresq) {
    c.urq = curq * expf(R(MP::gur) * lnr0r) * expf(bur3 * logf(cdiaqr * c.qrp / c.ncrp));
    c.urn = curn * c.urq;
  } else { c.urq = R(0); c.urn = R(0); }
  if (c.qsp > thresq) {
    c.usq = cusq * expf(R(MP::gus) * lnr0r) * expf(bus3 * logf(cdiaqs * c.qsp / c.ncsp));
    c.usn = cusn * c.usq;
  } else { c.usq = R(0); c.usn = R(0); }
  if (c.qgp > thresq) {
    c.ugq = cugq * expf(R(MP::gug) * lnr0r) * expf(bug3 * logf(cdiaqg * c.qgp / c.ncgp));
    c.ugn = cugn * c.ugq;
  } else { c.ugq = R(0); c.ugn = R(0); }
}

// s_srcblk cphopt=3, haiopt=0 (SrcOrig/srcblk.f90:488-630) on one cell:
// setblk, the process routines, more0q and newblk in the reference order.
// dtb is the microphysics step passed to coldblk (2*dtb of the leapfrog).
__device__ inline void srcblk_cell(R dtb, R thresq, MCell& c) {
    const R oned3 = R(MP::oned3), cc = R(MP::cc), t0 = R(MP::t0), tlow = R(MP::tlow);
  const R qv = c.qvp, qc = c.qcp, qr = c.qrp, qi = c.qip, qs = c.qsp, qg = c.qgp;
  const R ncc = c.nccp, ncr = c.ncrp, nci = c.ncip, ncs = c.ncsp, ncg = c.ncgp;
  const R rbr = c.rbr, rbv = c.rbv, p = c.p;

  // ---- s_setblk (setblk.f90:269-294, 789-930)
  const R cwmci = R(MP::cw) - R(MP::ci);
  const R epses0 = R(MP::epsva) * R(MP::es0);
  const R t23iv = R(1) / R(MP::t23);
  R cdv = R(1) / t0;
  const R cnu = expf(R(.57013) * logf(R(MP::nu0))) * cdv;
  cdv = expf(R(.55249) * logf(R(MP::dv0))) * cdv;
  const R pdiaqr = R(.5) * (R(5) + R(MP::bur)) - R(1);
  const R pdiaqs = R(.5) * (R(5) + R(MP::bus)) - R(1);
  const R pdiaqg = R(.5) * (R(5) + R(MP::bug)) - R(1);
  const R ccrw6 = R(6) / (cc * R(MP::rhow)), ccri6 = R(6) / (cc * R(MP::rhoi));
  const R cdiaqr = R(1) / (cc * R(MP::rhow)), cdiaqs = R(1) / (cc * R(MP::rhos));
  const R cdiaqg = R(1) / (cc * R(MP::rhog));
  const R cvntr = R(.31) * sqrtf(R(MP::aur)) * expf(oned3 * logf(R(MP::sc))) * R(MP::gf5bur);
  const R cvnts = R(.31) * sqrtf(R(MP::aus)) * expf(oned3 * logf(R(MP::sc))) * R(MP::gf5bus);
  const R cvntg = R(.31) * sqrtf(R(MP::aug)) * expf(oned3 * logf(R(MP::sc))) * R(MP::gf5bug);
  const R t = (c.ptbr + c.ptpp) * c.pi;
  const R tcel = t - t0;
  const R esi = R(MP::es0) * expf(R(21.875) * tcel / (t - R(7.66)));
  const R qvsi = R(MP::epsva) * esi / (p - esi);
  // Clear air: no hydrometeor above thresq at t-dt and no ice nucleation
  // from vapour (s_nuc1stv's condition below does not hold).  Every process
  // rate that follows is then exactly zero (each is guarded by one of those
  // conditions), and s_newblk reduces to subtracting or adding zero sinks
  // and its clipping at zero; with no negative future mixing ratio for its
  // sink cascade to act on, that is all that happens to the cell.
  if (!(qc > thresq) && !(qr > thresq) && !(qi > thresq) && !(qs > thresq) && !(qg > thresq) &&
      !(qv > thresq && qv > qvsi && t > tlow && t < t0) && c.qrf >= R(0) && c.qcf >= R(0) && c.qif >= R(0)) {
    c.ptpf = c.ptpf + R(0);
    c.qrf = c.qrf - R(0);
    c.qcf = c.qcf - R(0);
    c.qif = c.qif - R(0);
    c.qvf = fmaxf(c.qvf - R(0), R(0));
    c.qsf = fmaxf(c.qsf - R(0), R(0));
    c.qgf = fmaxf(c.qgf + R(0), R(0));
    c.ncif = c.ncif + R(0);
    c.ncsf = c.ncsf + R(0);
    c.ncgf = c.ncgf + R(0);
    return;
  }
  const R esw = R(MP::es0) * expf(R(17.269) * tcel / (t - R(35.86)));
  const R qvsst0 = qv - epses0 / (p - R(MP::es0));
  const R qvsw = R(MP::epsva) * esw / (p - esw);
  const R lv = R(MP::lv0) * expf((R(.167) + R(3.67e-4) * t) * logf(t0 / t));
  const R lf = R(MP::lf0) + cwmci * tcel;
  const R ls = lv + lf;
  const R p20dvp = R(MP::p20) / p;
  const R nu = p20dvp * expf(R(1.754) * logf(cnu * t));
  const R kp = (R(MP::kp0) / (R(120) + t)) * expf(R(1.5) * logf(t23iv * t));
  const R mu = rbr * nu;
  const R dv = p20dvp * expf(R(1.81) * logf(cdv * t));
  const R cvnt = sqrtf(sqrtf(R(MP::r0) * rbv) / nu);
  R diaqc, diaqr, vntr, mi, diaqi, diaqs, vnts, diaqg, vntg;
  if (qc > thresq) diaqc = expf(oned3 * logf(ccrw6 * qc / ncc)); else diaqc = R(0);
  if (qr > thresq) {
    diaqr = expf(oned3 * logf(cdiaqr * qr / ncr));
    vntr = rbr * ncr * (R(.78) * diaqr + cvnt * cvntr * expf(pdiaqr * logf(diaqr)));
  } else { diaqr = R(0); vntr = R(0); }
  if (qi > thresq) { mi = qi / nci; diaqi = expf(oned3 * logf(ccri6 * mi)); } else { mi = R(0); diaqi = R(0); }
  if (qs > thresq) {
    diaqs = expf(oned3 * logf(cdiaqs * qs / ncs));
    vnts = rbr * ncs * (R(.78) * diaqs + cvnt * cvnts * expf(pdiaqs * logf(diaqs)));
  } else { diaqs = R(0); vnts = R(0); }
  if (qg > thresq) {
    diaqg = expf(oned3 * logf(cdiaqg * qg / ncg));
    vntg = rbr * ncg * (R(.78) * diaqg + cvnt * cvntg * expf(pdiaqg * logf(diaqg)));
  } else { diaqg = R(0); vntg = R(0); }

  // ---- s_nuc1stv (nuc1stv.f90:179-216)
  R nuvi;
  if (qv > thresq) {
    if (qv > qvsi && t > tlow && t < t0) {
      const R qvssi = qv - qvsi;
      const R a = R(15.25) * qv / qvsi - R(10.08);
      if (a < R(40)) nuvi = fmaxf(R(0), fminf(R(MP::mi0) * expf(a) * rbv - qi, qvssi));
      else nuvi = qvssi;
    } else nuvi = R(0);
  } else nuvi = R(0);

  // ---- s_nuc1stc (nuc1stc.f90:172-401)
  R nuci;
  {
    const R rwdt2 = (R(100) / R(MP::rhow)) * dtb;
    const R cc45 = R(4.e5) * cc;
    const R cknd = R(2) * R(MP::lmb20) * R(MP::p20) / (R(MP::t20) * R(MP::diasl));
    const R cdar = R(MP::boltz) / (R(3) * cc * R(MP::diasl));
    const R kpa = R(MP::kpa), kpa25 = R(2.5) * kpa, kpa50 = R(5) * kpa;
    if (qc > thresq) {
      R nufci, nucci, nuhci;
      if (t > tlow && t < t0) nufci = fminf(rwdt2 * (expf(R(-.66) * tcel) - R(1)) * qc * qc / ncc, qc);
      else nufci = R(0);
      const R tc = t;
      if (tc > tlow && tc < R(270.16)) {
        const R piv = R(1) / p;
        const R knd = cknd * piv * t;
        const R dar = cdar * tc * (R(1) + knd) / mu;
        const R f1 = cc45 * expf(R(1.3) * logf(R(270.16) - tc)) * diaqc;
        if (tc < t) {
          const R f2 = kpa * piv * (t - tc);
          const R ft = (kp + kpa25 * knd) * (R(.4) + R(.58) * knd + R(.16) * expf(R(-1) / knd)) /
                       ((R(1) + R(3) * knd) * (R(2) * kp + kpa50 * knd + kpa));
          nucci = f1 * f2 * (R(MP::rv) * t / lv + ft);
        } else nucci = R(0);
        nucci = (nucci + f1 * dar) * qc * dtb;
      } else nucci = R(0);
      if (t <= tlow) nuhci = qc; else nuhci = R(0);
      nuci = nufci + nucci + nuhci;
    } else nuci = R(0);
  }

  // ---- s_collect cphopt>=3 (collect.f90:160-190 constants, 1550-1981)
  R clcr, clcs, clcg, clri, clrs, clrg, clir, clis, clig, clsr, clsg, clrin, clrsn, clsrn, clsgn, ecs;
  {
    const R rwdv9 = R(MP::oned9) * R(MP::rhow);
    const R bur2 = R(2) + R(MP::bur), bus2 = R(2) + R(MP::bus), bug2 = R(2) + R(MP::bug);
    const R esgiv = R(1) / R(MP::esg);
    const R cclcr = R(.25) * R(MP::aur) * R(MP::gf3bur) * cc * dtb;
    const R cclcs = R(.25) * R(MP::aus) * R(MP::gf3bus) * cc * dtb;
    const R cclcg = R(.25) * R(MP::aug) * R(MP::gf3bug) * cc * dtb;
    const R cclri = R(.25) * R(MP::aur) * R(MP::gf3bur) * R(MP::eir) * cc * dtb;
    const R cclrs = R(MP::ers) * cc * cc * R(MP::rhow) * dtb;
    const R cclrg = R(MP::erg) * cc * cc * R(MP::rhow) * dtb;
    const R cclis = R(.25) * R(MP::aus) * R(MP::gf3bus) * R(MP::eis) * cc * dtb;
    const R cclig = R(.25) * R(MP::aug) * R(MP::gf3bug) * R(MP::eig) * cc * dtb;
    const R cclsr = R(MP::esr) * cc * cc * R(MP::rhos) * dtb;
    const R cclsg = R(MP::esg) * cc * cc * R(MP::rhos) * dtb;
    const R cclrsn = R(.5) * R(MP::ers) * cc * dtb;
    const R cclsgn = R(.5) * R(MP::esg) * cc * dtb;
    const R r0rsq = sqrtf(R(MP::r0) * rbr);
    R diaqr2, diaqr3, qr2b, diaqs2, diaqs3, qs2b, diaqg2, qg2b;
    if (qr > thresq) { diaqr2 = diaqr * diaqr; diaqr3 = diaqr * diaqr2; qr2b = r0rsq * expf(bur2 * logf(diaqr)); }
    else { diaqr2 = R(0); diaqr3 = R(0); qr2b = R(0); }
    if (qs > thresq) { diaqs2 = diaqs * diaqs; diaqs3 = diaqs * diaqs2; qs2b = r0rsq * expf(bus2 * logf(diaqs)); }
    else { diaqs2 = R(0); diaqs3 = R(0); qs2b = R(0); }
    if (qg > thresq) { diaqg2 = diaqg * diaqg; qg2b = r0rsq * expf(bug2 * logf(diaqg)); }
    else { diaqg2 = R(0); qg2b = R(0); }
    const R urq = c.urq, usq = c.usq, ugq = c.ugq, urn = c.urn, usn = c.usn, ugn = c.ugn;
    if (t > tlow) {
      if (qc > thresq) {
        const R cstk = rwdv9 * diaqc * diaqc;
        if (qr > thresq) {
          R a = cstk * urq / (diaqr * mu);
          const R b = a + R(.5);
          a = a * a / (b * b);
          clcr = cclcr * a * qr2b * ncr * qc;
        } else clcr = R(0);
        if (qs > thresq) {
          const R a = cstk * usq / (diaqs * mu);
          const R b = a + R(.5);
          ecs = a * a / (b * b);
          clcs = cclcs * qs2b * ecs * ncs * qc;
        } else { clcs = R(0); ecs = R(0); }
        if (qg > thresq) {
          R a = cstk * ugq / (diaqg * mu);
          const R b = a + R(.5);
          a = a * a / (b * b);
          clcg = cclcg * a * qg2b * ncg * qc;
        } else clcg = R(0);
        const R sink = clcr + clcs + clcg;
        if (qc < sink) { const R a = qc / sink; clcr = clcr * a; clcs = clcs * a; clcg = clcg * a; }
      } else { clcr = R(0); clcs = R(0); clcg = R(0); ecs = R(0); }
      if (qr > thresq) {
        if (qi > thresq) {
          if (t < t0) { clri = cclri * qr2b * ncr * qi; clir = clri; clrin = clri / mi; }
          else { clri = R(0); clir = R(0); clrin = R(0); }
        } else { clri = R(0); clir = R(0); clrin = R(0); }
        if (qs > thresq) {
          const R a = R(2) * diaqr * diaqs;
          const R b = ncr * ncs * rbr;
          R cv = urq - usq;
          cv = sqrtf(cv * cv + R(.04) * urq * usq);
          clrs = b * cv * cclrs * (R(5) * diaqr2 + a + R(.5) * diaqs2) * diaqr3;
          clsr = b * cv * cclsr * (R(5) * diaqs2 + a + R(.5) * diaqr2) * diaqs3;
          cv = urn - usn;
          clrsn = b * cclrsn * (diaqr2 + R(.5) * a + diaqs2) * sqrtf(cv * cv + R(.04) * urn * usn);
          clsrn = clrsn;
        } else { clrs = R(0); clsr = R(0); clrsn = R(0); clsrn = R(0); }
        if (qg > thresq) {
          const R a = R(5) * diaqr2 + R(2) * diaqr * diaqg + R(.5) * diaqg2;
          const R b = urq - ugq;
          clrg = a * cclrg * diaqr3 * ncr * ncg * rbr * sqrtf(b * b + R(.04) * urq * ugq);
        } else clrg = R(0);
        R sink = clri + clrs + clrg;
        if (qr < sink) { const R a = qr / sink; clri = clri * a; clrs = clrs * a; clrg = clrg * a; }
        sink = clrin + clrsn;
        if (ncr < sink) { const R a = ncr / sink; clrin = clrin * a; clrsn = clrsn * a; }
      } else {
        clri = R(0); clrs = R(0); clrg = R(0); clir = R(0); clsr = R(0);
        clrin = R(0); clrsn = R(0); clsrn = R(0);
      }
    } else {
      clcr = R(0); clcs = R(0); clcg = R(0); clri = R(0); clrs = R(0); clrg = R(0); clir = R(0);
      clsr = R(0); clrin = R(0); clrsn = R(0); clsrn = R(0); ecs = R(0);
    }
    if (qi > thresq) {
      if (t < t0) {
        if (qs > thresq) clis = cclis * qs2b * ncs * qi; else clis = R(0);
        if (qg > thresq) clig = cclig * qg2b * ncg * qi; else clig = R(0);
        const R sink = clir + clis + clig;
        if (qi < sink) { const R a = qi / sink; clir = clir * a; clis = clis * a; clig = clig * a; }
      } else { clis = R(0); clig = R(0); }
    } else { clis = R(0); clig = R(0); }
    if (qs > thresq) {
      if (qg > thresq) {
        const R a = diaqs * diaqg;
        R b = (t < t0) ? ncs * ncg * rbr : esgiv * ncs * ncg * rbr;
        R cv = usq - ugq;
        clsg = b * cclsg * (R(5) * diaqs2 + R(2) * a + R(.5) * diaqg2) * diaqs3 * sqrtf(cv * cv + R(.04) * usq * ugq);
        cv = usn - ugn;
        clsgn = b * cclsgn * (diaqs2 + a + diaqg2) * sqrtf(cv * cv + R(.04) * usn * ugn);
      } else { clsg = R(0); clsgn = R(0); }
      R sink = clsr + clsg;
      if (qs < sink) { const R a = qs / sink; clsr = clsr * a; clsg = clsg * a; }
      sink = clsrn + clsgn;
      if (ncs < sink) { const R a = ncs / sink; clsrn = clsrn * a; clsgn = clsgn * a; }
    } else { clsg = R(0); clsgn = R(0); }
  }

  // ---- s_prodctwg cphopt>=3 (prodctwg.f90:206-209, 302-389)
  R pgwet;
  {
    const R cc2dtn = R(-2) * cc * dtb;
    const R eigiv = R(1) / R(MP::eig), esgiv = R(1) / R(MP::esg);
    if (qg > thresq) {
      if (tcel < R(MP::t0cel)) {
        const R pgdry = clcg + clrg + clig + clsg;
        const R lfice = lf + R(MP::cw) * tcel;
        const R cligw = eigiv * clig, clsgw = esgiv * clsg;
        pgwet = cc2dtn * vntg * (lv * dv * rbr * qvsst0 + kp * tcel) / (lfice * rbr) +
                (cligw + clsgw) * (R(1) - R(MP::ci) * tcel / lfice);
        if (pgwet > R(0) && pgwet < pgdry) {
          clig = cligw;
          clsg = clsgw;
          clsgn = esgiv * clsgn;
          R sink = clir + clis + clig;
          if (qi < sink) { const R a = qi / sink; clir = clir * a; clis = clis * a; clig = clig * a; }
          sink = clsr + clsg;
          if (qs < sink) { const R a = qs / sink; clsr = clsr * a; clsg = clsg * a; }
          sink = clsrn + clsgn;
          if (ncs < sink) { const R a = ncs / sink; clsrn = clsrn * a; clsgn = clsgn * a; }
        } else pgwet = R(-1);
      } else pgwet = R(-1);
    } else pgwet = R(-1);
  }

  // ---- s_distrpg cphopt>=3 (distrpg.f90:148-149, 328-371)
  R clrsg;
  {
    const R rhos2 = R(MP::rhos) * R(MP::rhos), rhow2 = R(MP::rhow) * R(MP::rhow);
    if (qs > thresq) {
      if (t < t0) {
        R a = diaqs * diaqs, b = diaqr * diaqr;
        a = rhos2 * a * a * a;
        b = rhow2 * b * b * b;
        const R alpha = a / (a + b), alpha1 = R(1) - alpha;
        clrsg = alpha1 * clrs;
        clrs = alpha * clrs;
        clsr = alpha1 * clsr;
        clrsn = alpha1 * clrsn;
        clsrn = alpha1 * clsrn;
      } else { clrsg = clrs; clrs = R(0); }
    } else clrsg = R(0);
  }

  // ---- s_aggregat cphopt=3 (aggregat.f90:150-191, 434-469)
  R agin, agsn;
  {
    const R expo1 = oned3 * (R(2) + R(MP::bus)), expo2 = oned3 * (R(4) - R(MP::bus));
    const R cagin = R(MP::r0) * expf(R(3) * logf(R(.5) * R(MP::aui) * R(MP::eii) * R(MP::xl) / R(MP::rhoi) * dtb));
    const R cagsn = R(3.47222e-4) * R(MP::aus) * R(MP::ess) * R(MP::hfbus) * dtb *
                    expf(oned3 * (R(1) - R(MP::bus)) * logf(cc)) * expf(-oned3 * (R(2) + R(MP::bus)) * logf(R(MP::rhos)));
    if (qi > thresq) agin = rbr * nci * qi * expf(oned3 * logf(cagin * rbv)); else agin = R(0);
    if (qs > thresq) agsn = cagsn * rbr * expf(expo1 * logf(qs)) * expf(expo2 * logf(ncs)); else agsn = R(0);
  }

  // ---- s_melting (melting.f90:150, 278-360)
  R mlic, mlsr, mlgr;
  {
    const R cc2dt = R(2) * cc * dtb;
    const R cmlxr1 = cc2dt * rbv * (kp * tcel + lv * dv * rbr * qvsst0);
    const R cmlxr2 = R(MP::cw) * tcel;
    if (qi > thresq) mlic = (tcel >= R(MP::t0cel)) ? qi : R(0); else mlic = R(0);
    if (qs > thresq && tcel >= R(MP::t0cel)) mlsr = fmaxf((cmlxr1 * vnts + cmlxr2 * (clcs + clrs)) / lf, R(0));
    else mlsr = R(0);
    if (qg > thresq && tcel >= R(MP::t0cel)) mlgr = fmaxf((cmlxr1 * vntg + cmlxr2 * (clcg + clrg)) / lf, R(0));
    else mlgr = R(0);
  }

  // ---- s_depsit (depsit.f90:200-242, 427-600)
  R vdvr, vdvi, vdvs, vdvg;
  {
    const R ccdtb4 = R(2) * cc * dtb;
    const R t27311 = t0 - R(.01);
    if (t > tlow) {
      const R qvssw = qv - qvsw, qvssi = qv - qvsi;
      const R a = R(1) / (R(MP::rv) * kp * t * t);
      const R b = dv * rbr;
      const R cv = ccdtb4 * rbv;
      const R gi = R(1) / (ls * ls * a + R(1) / (b * qvsi));
      const R cvdvx1 = cv * (qv / qvsw - R(1)) / (lv * lv * a + R(1) / (b * qvsw));
      const R cvdvx2 = ccdtb4 * dv * qvsst0;
      const R cvdvx3 = cv * (qv / qvsi - R(1));
      const R cvdvx4 = a * ls * lf;
      if (qr > thresq && qv < qvsw) vdvr = fmaxf(cvdvx1 * vntr, qvssw); else vdvr = R(0);
      if (qi > thresq && t < t27311) {
        const int itsc = (int)(-tcel);
        vdvi = kKoeC[itsc] * (qv - qvsi) / (qvsw - qvsi) * nci * expf(kKoeP[itsc] * logf(mi)) * dtb;
      } else vdvi = R(0);
      if (qs > thresq) {
        if (t > t0) vdvs = (mlsr > R(0)) ? cvdvx2 * vnts : cvdvx1 * vnts;
        else vdvs = gi * (cvdvx3 * vnts - cvdvx4 * clcs);
      } else vdvs = R(0);
      if (qg > thresq) {
        if (t > t0) vdvg = (mlgr > R(0)) ? cvdvx2 * vntg : cvdvx1 * vntg;
        else vdvg = gi * (cvdvx3 * vntg - cvdvx4 * clcg);
      } else vdvg = R(0);
      const R sink = vdvi + vdvs + vdvg;
      if ((qvssi < sink && qvssi > R(0)) || (qvssi > sink && qvssi < R(0))) {
        const R aa = qvssi / sink;
        vdvi = vdvi * aa; vdvs = vdvs * aa; vdvg = vdvg * aa;
      }
    } else { vdvr = R(0); vdvi = R(0); vdvs = R(0); vdvg = R(0); }
  }

  // ---- s_convers cphopt>=3 (convers.f90:180-225, 604-719)
  R cncr, cnis, cnsg, cnsgn;
  {
    const R busm1 = R(MP::bus) - R(1);
    const R ms05 = R(.5) * R(MP::ms0);
    const R qccm = R(MP::oned6) * R(MP::rhow) * cc * R(MP::diaqcm) * R(MP::diaqcm) * R(MP::diaqcm);
    const R diaqs0 = expf(oned3 * logf(R(6) * R(MP::ms0) / (cc * R(MP::rhos))));
    const R cagin = R(MP::r0) * expf(R(3) * logf(R(.5) * oned3 * R(MP::aui) * R(MP::eii) * R(MP::xl) / R(MP::rhoi) * dtb));
    const R ccncr = R(.104) * R(kGrav) * R(MP::ecc) * expf(-oned3 * logf(R(MP::rhow))) * dtb;
    R ccnsgn = R(1) / (R(MP::rhog) - R(MP::rhos));
    const R ccnsg = R(MP::rhog) * ccnsgn;
    ccnsgn = R(1.5) * R(MP::aus) * R(MP::gfbus) * sqrtf(R(MP::r0)) * ccnsgn * dtb;
    if (qc > thresq) {
      const R qcm = qccm * ncc;
      if (t > tlow && qc >= qcm) cncr = ccncr * rbr * expf(-oned3 * logf(ncc)) * expf(R(MP::sevnd3) * logf(qc)) / mu;
      else cncr = R(0);
    } else cncr = R(0);
    if (t < t0) {
      if (qi > thresq) {
        cnis = rbr * expf(oned3 * logf(cagin * rbv)) * qi * qi / logf(diaqs0 / diaqi);
        if (vdvi >= R(0)) {
          if (mi < ms05) cnis = cnis + mi / (R(MP::ms0) - mi) * vdvi;
          else cnis = cnis + (vdvi + (R(1) - ms05 / mi) * qi);
        }
        cnis = fminf(cnis, qi);
      } else cnis = R(0);
      if (qs > thresq) {
        if (vdvs > R(0) && vdvs < clcs) {
          cnsg = fminf(ccnsg * clcs, qs);
          cnsgn = fminf(ccnsgn * ecs * qc * ncs * sqrtf(rbr) * expf(busm1 * logf(diaqs)), ncs);
        } else { cnsg = R(0); cnsgn = R(0); }
      } else { cnsg = R(0); cnsgn = R(0); }
    } else { cnis = R(0); cnsg = R(0); cnsgn = R(0); }
  }

  // ---- s_nuc2nd (nuc2nd.f90:100-101, 208-282)
  R spsi, spgi;
  {
    const R mi0352 = R(.5) * R(3.5e8) * R(MP::mi0), mi0353 = oned3 * R(3.5e8) * R(MP::mi0);
    if (pgwet > R(0)) {
      if (t > R(270.16)) spsi = R(0);
      else if (t > R(268.16) && t <= R(270.16)) spsi = (R(270.16) - t) * mi0352 * rbv * clcs;
      else if (t > R(265.16) && t <= R(268.16)) spsi = (t - R(265.16)) * mi0353 * rbv * clcs;
      else spsi = R(0);
      spgi = R(0);
    } else {
      if (t > R(270.16)) { spsi = R(0); spgi = R(0); }
      else if (t > R(268.16) && t <= R(270.16)) { const R a = (R(270.16) - t) * mi0352 * rbv; spsi = a * clcs; spgi = a * clcg; }
      else if (t > R(265.16) && t <= R(268.16)) { const R a = (t - R(265.16)) * mi0353 * rbv; spsi = a * clcs; spgi = a * clcg; }
      else { spsi = R(0); spgi = R(0); }
    }
  }

  // ---- s_freezing cphopt>=3 (freezing.f90:120-157, 316-366)
  R frrg, frrgn;
  {
    const R tclow = tlow - t0;
    const R cfrrg = R(20) * R(100) * cc * cc * R(MP::rhow) * dtb;
    const R cfrrgn = R(100) * cc * dtb;
    if (qr > thresq && tcel < R(MP::t0cel)) {
      if (tcel <= tclow) { frrg = qr; frrgn = ncr; }
      else {
        const R a = (expf(R(-.66) * tcel) - R(1)) * ncr;
        const R diaqr3 = diaqr * diaqr * diaqr;
        frrg = fminf(cfrrg * diaqr3 * diaqr3 * a, qr);
        frrgn = fminf(cfrrgn * diaqr3 * a, ncr);
      }
    } else { frrg = R(0); frrgn = R(0); }
  }

  // ---- s_shedding (shedding.f90:209-278)
  R shsr, shgr;
  if (qs > thresq && t >= t0) shsr = clcs + clrs; else shsr = R(0);
  if (qg > thresq) {
    if (t >= t0) shgr = clcg + clrg;
    else shgr = (pgwet > R(0)) ? (clcg + clrg + clig + clsg) - pgwet : R(0);
  } else shgr = R(0);

  // ---- s_more0q (more0q.f90:448-659), evapor_opt=1
  R& qcf = c.qcf; R& qrf = c.qrf; R& qif = c.qif; R& qsf = c.qsf; R& qgf = c.qgf;
  if (qc > thresq) {
    const R sink = nuci + clcr + clcs + clcg + cncr - mlic;
    if (qcf < sink) {
      const R h = qcf / sink;
      nuci *= h; clcr *= h; clcs *= h; clcg *= h; cncr *= h; mlic *= h;
    }
  }
  if (qi > thresq) {
    const R sink = clir + clis + clig + cnis + mlic - vdvi - nuvi - nuci - spsi - spgi;
    if (qif < sink) {
      const R h = qif / sink;
      clir *= h; clis *= h; clig *= h; cnis *= h; mlic *= h; vdvi *= h; nuvi *= h; nuci *= h; spsi *= h; spgi *= h;
    }
  }
  if (qr > thresq) {
    const R sink = clri + clrs + clrg + clrsg + frrg - vdvr - clcr - cncr - mlsr - mlgr - shsr - shgr;
    if (qrf < sink) {
      const R h = qrf / sink;
      clri *= h; clrs *= h; clrg *= h; clrsg *= h; frrg *= h; vdvr *= h; clcr *= h; cncr *= h;
      mlsr *= h; mlgr *= h; shsr *= h; shgr *= h;
    }
  }
  if (qs > thresq) {
    const R sink = clsr + clsg + cnsg + spsi + mlsr + shsr - vdvs - clcs - clrs - clis - cnis;
    if (qsf < sink) {
      const R h = qsf / sink;
      clsr *= h; clsg *= h; cnsg *= h; spsi *= h; mlsr *= h; shsr *= h; vdvs *= h; clcs *= h;
      clrs *= h; clis *= h; cnis *= h;
    }
  }
  if (qg > thresq) {
    const R sink = spgi + mlgr + shgr - vdvg - clri - clir - clsr - clcg - clrg - clig - clsg - clrsg - cnsg - frrg;
    if (qgf < sink) {
      const R h = qgf / sink;
      spgi *= h; mlgr *= h; shgr *= h; vdvg *= h; clri *= h; clir *= h; clsr *= h; clcg *= h;
      clrg *= h; clig *= h; clsg *= h; clrsg *= h; cnsg *= h; frrg *= h;
    }
  }

  // ---- s_newblk cphopt=3 (newblk.f90:300-374 constants, 1145-1343)
  {
    const R mi0iv = R(1) / R(MP::mi0), ms0iv = R(1) / R(MP::ms0);
    const R cppiv = R(1) / (R(kCpAir) * c.pi);
    const R clix = clir + clis + clig;
    const R spxi = spsi + spgi;
    const R cxcr = clcr + cncr;
    const R cxsg = clsr + clsg + cnsg;
    const R nmci = nuci - mlic;
    const R mssr = mlsr + shsr, msgr = mlgr + shgr;
    const R nuvdvx = vdvi + vdvs + vdvg + nuvi;
    const R clnmci = clcs + clcg + nmci;
    const R cfmsxr = clri + clrs + clrg + clrsg + frrg - mssr - msgr;
    c.ptpf = c.ptpf + (vdvr * lv + (clnmci + cfmsxr) * lf + nuvdvx * ls) * cppiv;
    R qvsink = nuvdvx + vdvr;
    R qxsink = cfmsxr - cxcr - vdvr;
    if (qrf < qxsink) { qxsink = cxcr + clnmci + (qxsink - qrf); qrf = R(0); }
    else { qrf = qrf - qxsink; qxsink = cxcr + clnmci; }
    if (qcf < qxsink) {
      const R dqv = qxsink - qcf;
      c.ptpf = c.ptpf + cppiv * dqv * lv;
      qvsink = qvsink + dqv;
      qcf = R(0);
    } else qcf = qcf - qxsink;
    qxsink = clix - spxi - nmci + cnis - vdvi - nuvi;
    if (qif < qxsink) {
      const R dqv = qxsink - qif;
      c.ptpf = c.ptpf + cppiv * dqv * ls;
      qvsink = qvsink + dqv;
      qif = R(0);
    } else qif = qif - qxsink;
    c.qvf = fmaxf(c.qvf - qvsink, R(0));
    qsf = fmaxf(qsf - (cxsg + mssr + spsi - vdvs - clcs - clrs - clis - cnis), R(0));
    qgf = fmaxf(qgf + (cxsg - msgr - spgi + vdvg + clri + clir + clcg + clrg + clig + clrsg + frrg), R(0));
    if (qc > thresq) c.ncif = c.ncif + nuci * ncc / qc;
    if (qi > thresq) {
      if (vdvi < R(0))
        c.ncif = c.ncif - (agin + (clix + mlic - vdvi) / mi - (spxi + nuvi) * mi0iv + cnis * ms0iv);
      else
        c.ncif = c.ncif - (agin + (clix + mlic) / mi - (spxi + nuvi) * mi0iv + cnis * ms0iv);
    } else c.ncif = c.ncif + (spxi + nuvi) * mi0iv;
    if (qs > thresq) {
      if (vdvs < R(0))
        c.ncsf = c.ncsf - (agsn - cnis * ms0iv + clsrn + clsgn + cnsgn + (mlsr - vdvs) * ncs / qs);
      else
        c.ncsf = c.ncsf - (agsn - cnis * ms0iv + clsrn + clsgn + cnsgn + mlsr * ncs / qs);
    } else c.ncsf = c.ncsf + cnis * ms0iv;
    if (qg > thresq) {
      if (vdvg < R(0))
        c.ncgf = c.ncgf + ((vdvg - mlgr) * ncg / qg + clrsn + clrin + cnsgn + frrgn);
      else
        c.ncgf = c.ncgf - (mlgr * ncg / qg - clrsn - clrin - cnsgn - frrgn);
    } else c.ncgf = c.ncgf + (clrsn + clrin + cnsgn + frrgn);
  }
}

// s_siadjst then s_swadjst (cphopt<=3 branch), SrcOrig/siadjst.f90:149-269,
// SrcOrig/swadjst.f90:198-310, called by s_satadjst (satadjst.f90:175-183).
__device__ inline void satadjst_cell(R thresq, R ptbr, R pi, R p, R& ptp, R& qv, R& qc, R& qi, R& nci) {
    const R t0 = R(MP::t0), tlow = R(MP::tlow);
  const R cwmci = R(MP::cw) - R(MP::ci);
  const R mi0iv = R(1) / R(MP::mi0);
  const R cp = R(kCpAir);
  // siadjst: two passes below tlow
  for (int pass = 0; pass < 2; ++pass) {
    const R t = (ptbr + ptp) * pi;
    if (!(t <= tlow)) break;
    const R tcel = t - t0;
    const R a = R(1) / (t - R(7.66));
    const R b = a * tcel;
    const R esi = R(MP::es0) * expf(R(21.875) * b);
    const R qvsi = R(MP::epsva) * esi / (p - esi);
    if (qi > thresq || qv > qvsi) {
      const R lscpi = (R(MP::lv0) * expf((R(.167) + R(3.67e-4) * t) * logf(t0 / t)) + (R(MP::lf0) + cwmci * tcel)) / (cp * pi);
      const R dqi = (qvsi - qv) / (R(1) + R(21.875) * a * (R(1) - b) * qvsi * lscpi * pi);
      if (qi > dqi) {
        if (qi > thresq) nci = nci - dqi * nci / qi; else nci = nci - dqi * mi0iv;
        ptp = ptp - dqi * lscpi;
        qv = qv + dqi;
        qi = qi - dqi;
      } else {
        nci = R(0);
        ptp = ptp - qi * lscpi;
        qv = qv + qi;
        qi = R(0);
      }
    }
    if (pass == 0) {
      // the second pass runs only when the first one ran (siadjst.f90:216-267)
    }
  }
  // swadjst (cphopt<=3): two passes
  for (int pass = 0; pass < 2; ++pass) {
    const R t = (ptbr + ptp) * pi;
    const R a = R(1) / (t - R(35.86));
    const R b = a * (t - t0);
    const R esw = R(MP::es0) * expf(R(17.269) * b);
    const R qvsw = R(MP::epsva) * esw / (p - esw);
    if (qc > thresq || qv > qvsw) {
      const R lvcpi = R(MP::lv0) * expf((R(.167) + R(3.67e-4) * t) * logf(t0 / t)) / (cp * pi);
      const R dqc = (qvsw - qv) / (R(1) + R(17.269) * a * (R(1) - b) * qvsw * lvcpi * pi);
      if (qc > dqc) {
        ptp = ptp - dqc * lvcpi;
        qv = qv + dqc;
        qc = qc - dqc;
      } else {
        ptp = ptp - qc * lvcpi;
        qv = qv + qc;
        qc = R(0);
      }
    } else if (pass == 0) {
      break;  // the second pass is nested in the first one's condition (swadjst.f90:252-308)
    }
  }
}

}  // namespace cress

// Oracle: Smagorinsky turbulence (tubopt=1) and the 1.5-order TKE closure
// (tubopt=2), isoopt=1, for flat terrain without map factors (trnopt=0,
// mfcopt=0), no surface fluxes (sfcopt=0),
// periodic lateral boundaries on one process (iwest=ieast=jsouth=jnorth=0),
// rigid bottom and top (bbc=tbc=2).
//
// TEST INFRASTRUCTURE ONLY (see arr.h).
#pragma once
#include <algorithm>
#include <cmath>
#include "small.h"

namespace oracle {

struct TurbConst {
  static constexpr double epsav = 1.6077;   // comphy.f90:82
  static constexpr double tlow = 233.16;    // comphy.f90:100
  static constexpr double lv0 = 2.50078e6, lf0 = 3.34e5, t0 = 273.16;
  static constexpr double cw = 4.218e3, ci = 2.106e3;
  static constexpr double ckm = .1, ckmin = 1.e-6;   // comphy.f90:341-344
  static constexpr double eps = 1.e-20;              // commath.f90:177
};

template <class R>
struct TurbWork {
  F3<R> nsq8w, t11, t22, t33, t12, t13, t23, t31, t32, ssq, rkh, rkv, priv, pt, ptv, a, tmp1, tmp2,
      tmp3, rkv8s, rkh8u, rkh8v, h1, h2, h3, jcbs;
  void resize(int ni, int nj, int nk) {
    for (F3<R>* x : {&nsq8w, &t11, &t22, &t33, &t12, &t13, &t23, &t31, &t32, &ssq, &rkh, &rkv, &priv, &pt,
                     &ptv, &a, &tmp1, &tmp2, &tmp3, &rkv8s, &rkh8u, &rkh8v, &h1, &h2, &h3, &jcbs})
      x->resize(ni, nj, nk);
  }
};

// s_bruntv, SrcOrig/bruntv.f90:212-345: squared Brunt-Vaisala frequency at
// w levels from the past level; dry, or moist with the saturated form
// where qall > thresq (cphopt != 0).
template <class R>
void bruntv(const Opts& o, bool moist, R thresq, const Base<R>& b, const F3<R>& ppp, const F3<R>& ptpp,
            const F3<R>* qvp, const F3<R>* qallp, TurbWork<R>& tw) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dziv = R(1) / R(o.dz);
  const R gdzv = R(Phys::g) * dziv, gdzv05 = R(.5) * R(Phys::g) * dziv;
  const R rddvcp = R(Phys::rd) / R(Phys::cp), cwmci = R(TurbConst::cw) - R(TurbConst::ci);
  const R p0iv = R(1) / R(Phys::p0);
  F3<R>& pt = tw.pt;
  F3<R>& ptv = tw.ptv;
  F3<R>& a = tw.a;
  F3<R>& nsq8w = tw.nsq8w;
  for (int k = 1; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) pt(i, j, k) = b.ptbr(i, j, k) + ptpp(i, j, k);
  if (!moist) {
    for (int k = 2; k <= nk - 1; ++k)
      for (int j = 1; j <= nj - 1; ++j)
        for (int i = 1; i <= ni - 1; ++i)
          nsq8w(i, j, k) = gdzv * (pt(i, j, k) - pt(i, j, k - 1)) /
                           (b.jcb8w(i, j, k) * (b.ptbr(i, j, k - 1) + b.ptbr(i, j, k)));
  } else {
    const F3<R>& qv = *qvp;
    const F3<R>& qall = *qallp;
    for (int k = 1; k <= nk - 1; ++k)
      for (int j = 1; j <= nj - 1; ++j)
        for (int i = 1; i <= ni - 1; ++i)
          ptv(i, j, k) = pt(i, j, k) * (R(1) + R(TurbConst::epsav) * qv(i, j, k)) / (R(1) + qv(i, j, k));
    for (int k = 1; k <= nk - 1; ++k)
      for (int j = 1; j <= nj - 1; ++j)
        for (int i = 1; i <= ni - 1; ++i) {
          const R t = pt(i, j, k) * std::exp(rddvcp * std::log(p0iv * (b.pbr(i, j, k) + ppp(i, j, k))));
          R av = R(TurbConst::lv0) * std::exp((R(.167) + R(3.67e-4) * t) * std::log(R(TurbConst::t0) / t));
          if (t <= R(TurbConst::tlow)) av = av + (R(TurbConst::lf0) + cwmci * (t - R(TurbConst::t0)));
          const R lhcpt = av / (R(Phys::cp) * t);
          pt(i, j, k) = pt(i, j, k) * std::exp(lhcpt * qv(i, j, k));
          av = av * qv(i, j, k) / (R(Phys::rd) * t);
          a(i, j, k) = (R(1) + av) / (R(1) + R(Phys::epsva) * lhcpt * av);
        }
    for (int k = 2; k <= nk - 1; ++k)
      for (int j = 1; j <= nj - 1; ++j)
        for (int i = 1; i <= ni - 1; ++i) {
          if (qall(i, j, k) > thresq)
            nsq8w(i, j, k) = gdzv05 * ((qall(i, j, k - 1) - qall(i, j, k)) +
                                       (pt(i, j, k) - pt(i, j, k - 1)) * (a(i, j, k - 1) + a(i, j, k)) /
                                           (b.ptbr(i, j, k - 1) + b.ptbr(i, j, k))) /
                             b.jcb8w(i, j, k);
          else
            nsq8w(i, j, k) = gdzv * (ptv(i, j, k) - ptv(i, j, k - 1)) /
                             (b.jcb8w(i, j, k) * (b.ptbr(i, j, k - 1) + b.ptbr(i, j, k)));
        }
  }
  for (int j = 1; j <= nj - 1; ++j)
    for (int i = 1; i <= ni - 1; ++i) {
      nsq8w(i, j, 1) = nsq8w(i, j, 2);
      nsq8w(i, j, nk) = nsq8w(i, j, nk - 1);
    }
}

// s_bcten, SrcOrig/bcten.f90:126-160 for rigid walls (bbc=tbc=2).
template <class R>
void bcten(const Opts& o, F3<R>& t) {
  for (int j = 0; j <= o.nj + 1; ++j)
    for (int i = 0; i <= o.ni + 1; ++i) {
      t(i, j, 1) = -t(i, j, 3);
      t(i, j, o.nk) = -t(i, j, o.nk - 2);
    }
}

// s_defomten, SrcOrig/defomten.f90:305-1106 (trnopt=0, mfcopt=0), and
// s_defomssq, SrcOrig/defomssq.f90:130-141: deformation tensor of the past
// winds into t11..t32 and its square into ssq.
template <class R>
void defomten(const Opts& o, const Base<R>& b, const F3<R>& u, const F3<R>& v, const F3<R>& w, TurbWork<R>& tw) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dxiv = R(1) / R(o.dx), dyiv = R(1) / R(o.dy), dziv = R(1) / R(o.dz);
  F3<R>&tmp1 = tw.tmp1, &tmp2 = tw.tmp2, &tmp3 = tw.tmp3;
  for (int k = 1; k <= nk - 1; ++k) {
    for (int j = 0; j <= nj; ++j)
      for (int i = 0; i <= ni + 1; ++i) tmp1(i, j, k) = u(i, j, k) * b.jcb8u(i, j, k);
    for (int j = 0; j <= nj + 1; ++j)
      for (int i = 0; i <= ni; ++i) tmp2(i, j, k) = v(i, j, k) * b.jcb8v(i, j, k);
  }
  for (int k = 1; k <= nk - 1; ++k)
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i)
        tmp3(i, j, k) =
            R(4) / ((b.jcb(i - 1, j - 1, k) + b.jcb(i, j, k)) + (b.jcb(i - 1, j, k) + b.jcb(i, j - 1, k)));
  for (int k = 1; k <= nk - 1; ++k) {
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni; ++i)
        tw.t12(i, j, k) = tmp3(i, j, k) * ((tmp1(i, j, k) - tmp1(i, j - 1, k)) * dyiv +
                                           (tmp2(i, j, k) - tmp2(i - 1, j, k)) * dxiv);
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) {
        tw.t11(i, j, k) = (tmp1(i + 1, j, k) - tmp1(i, j, k)) * dxiv;
        tw.t22(i, j, k) = (tmp2(i, j + 1, k) - tmp2(i, j, k)) * dyiv;
      }
  }
  for (int k = 1; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) {
        const R jcbiv2 = R(2) / b.jcb(i, j, k);
        tw.t11(i, j, k) = jcbiv2 * tw.t11(i, j, k);
        tw.t22(i, j, k) = jcbiv2 * tw.t22(i, j, k);
        tw.t33(i, j, k) = jcbiv2 * (w(i, j, k + 1) - w(i, j, k)) * dziv;
      }
  // x-z / z-x and y-z / z-y components (defomten.f90:763-1091)
  for (int k = 1; k <= nk; ++k)
    for (int j = 0; j <= nj; ++j)
      for (int i = 0; i <= ni; ++i) tmp1(i, j, k) = w(i, j, k) * b.jcb8w(i, j, k);
  for (int k = 1; k <= nk; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni; ++i) tmp3(i, j, k) = R(2) / (b.jcb8w(i - 1, j, k) + b.jcb8w(i, j, k));
  for (int k = 2; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni; ++i) {
        tw.t13(i, j, k) =
            ((tmp1(i, j, k) - tmp1(i - 1, j, k)) * dxiv + (u(i, j, k) - u(i, j, k - 1)) * dziv) * tmp3(i, j, k);
        tw.t31(i, j, k) = tw.t13(i, j, k);
      }
  for (int k = 1; k <= nk; ++k)
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni - 1; ++i) tmp3(i, j, k) = R(2) / (b.jcb8w(i, j - 1, k) + b.jcb8w(i, j, k));
  for (int k = 2; k <= nk - 1; ++k)
    for (int j = 1; j <= nj; ++j)
      for (int i = 1; i <= ni - 1; ++i) {
        tw.t23(i, j, k) =
            ((tmp1(i, j, k) - tmp1(i, j - 1, k)) * dyiv + (v(i, j, k) - v(i, j, k - 1)) * dziv) * tmp3(i, j, k);
        tw.t32(i, j, k) = tw.t23(i, j, k);
      }
  bcten(o, tw.t31);
  bcten(o, tw.t32);
  for (int k = 1; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) {
        const R s128s =
            (tw.t12(i, j, k) + tw.t12(i + 1, j + 1, k)) + (tw.t12(i + 1, j, k) + tw.t12(i, j + 1, k));
        const R s318s =
            (tw.t31(i, j, k) + tw.t31(i + 1, j, k + 1)) + (tw.t31(i, j, k + 1) + tw.t31(i + 1, j, k));
        const R s328s =
            (tw.t32(i, j, k) + tw.t32(i, j + 1, k + 1)) + (tw.t32(i, j + 1, k) + tw.t32(i, j, k + 1));
        tw.ssq(i, j, k) = R(.5) * (tw.t33(i, j, k) * tw.t33(i, j, k) +
                                   (tw.t11(i, j, k) * tw.t11(i, j, k) + tw.t22(i, j, k) * tw.t22(i, j, k))) +
                          R(.0625) * (s128s * s128s + (s318s * s318s + s328s * s328s));
      }
}

// s_eddyvis tubopt=1, isoopt=1, mfcopt=0 (SrcOrig/eddyvis.f90:213-268):
// rkv = rkh = rbr * min(cs^2 l^2 sqrt(max(ssq - N^2/Pr, 0)), ckmax l^2),
// l = (dx dy dz jcb)^(1/3), ckmax = 0.125/dtb, 1/Pr capped at 3.
template <class R>
void eddyvis(const Opts& o, R dtb, const Base<R>& b, TurbWork<R>& tw) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R ds3 = R(o.dx) * R(o.dy) * R(o.dz);
  R cpriv = R(1) / R(Phys::prnum);
  if (cpriv > R(3)) cpriv = R(3);
  const R ckmax = R(.125) / dtb;
  const R csnum2 = R(Phys::csnum) * R(Phys::csnum);
  const R oned3 = R(1) / R(3);
  for (int k = 1; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) {
        const R ln = std::exp(oned3 * std::log(ds3 * b.jcb(i, j, k)));
        const R ln2 = ln * ln;
        tw.priv(i, j, k) = cpriv;
        R kv = csnum2 * ln2 *
               std::sqrt(std::max(tw.ssq(i, j, k) - (tw.nsq8w(i, j, k) + tw.nsq8w(i, j, k + 1)) * cpriv, R(0)));
        kv = b.rbr(i, j, k) * std::min(kv, ckmax * ln2);
        tw.rkv(i, j, k) = kv;
        tw.rkh(i, j, k) = kv;
      }
}

// s_eddyvis tubopt>=2 (the Deardorff form), isoopt=1, mfcopt=0, sfcopt=0
// (SrcOrig/eddyvis.f90:448-481): the length scale l = l0 = (dx dy dz
// jcb)^(1/3) in unstable air, else max(0.1 l0, min(0.76 sqrt(e/N^2), l0));
// 1/Pr = 1 + 2 l/l0; rkv = rkh = rbr * min(K, ckmax l0^2) with
// K = ckm l sqrt(e), raised to ckmin l0^2 where 1/Pr N^2 < ssq.  tke is the
// past level.
template <class R>
void eddyvis_tke(const Opts& o, R dtb, const Base<R>& b, const F3<R>& tke, TurbWork<R>& tw) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R ds3 = R(o.dx) * R(o.dy) * R(o.dz);
  const R ckmax = R(.125) / dtb;
  const R oned3 = R(1) / R(3);
  const R ckm = R(TurbConst::ckm), ckmin = R(TurbConst::ckmin), eps = R(TurbConst::eps);
  for (int k = 1; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) {
        const R ln0 = std::exp(oned3 * std::log(ds3 * b.jcb(i, j, k)));
        const R ln02 = ln0 * ln0;
        const R nsq = tw.nsq8w(i, j, k) + tw.nsq8w(i, j, k + 1);
        const R e = tke(i, j, k);
        R ln;
        if (nsq < R(0))
          ln = ln0;
        else
          ln = std::max(R(.1) * ln0, std::min(R(.76) * std::sqrt(e / (nsq + eps)), ln0));
        const R priv = R(1) + R(2) * ln / ln0;
        tw.priv(i, j, k) = priv;
        R kv = ckm * ln * std::sqrt(e);
        if (priv * nsq < tw.ssq(i, j, k)) kv = std::max(kv, ckmin * ln02);
        kv = b.rbr(i, j, k) * std::min(kv, ckmax * ln02);
        tw.rkv(i, j, k) = kv;
        tw.rkh(i, j, k) = kv;
      }
}

// s_sheartke, SrcOrig/sheartke.f90:112-120: shear production jcb rkv ssq
// (rkv as s_eddyvis left it).
template <class R>
void sheartke(const Opts& o, const Base<R>& b, const TurbWork<R>& tw, F3<R>& tkefrc) {
  for (int k = 2; k <= o.nk - 2; ++k)
    for (int j = 2; j <= o.nj - 2; ++j)
      for (int i = 2; i <= o.ni - 2; ++i)
        tkefrc(i, j, k) = tkefrc(i, j, k) + b.jcb(i, j, k) * tw.rkv(i, j, k) * tw.ssq(i, j, k);
}

// s_disptke isoopt=1, mfcopt=0 (SrcOrig/disptke.f90:181-195): dissipation
// (0.37/Pr - 0.18) rst e^1.5 / l, with l = (1/Pr - 1)(dx dy dz jcb / 8)^(1/3)
// recovered from 1/Pr; tke is the past level.
template <class R>
void disptke(const Opts& o, const Base<R>& b, const TurbWork<R>& tw, const F3<R>& tke, F3<R>& tkefrc) {
  const R ds308 = R(.125) * R(o.dx) * R(o.dy) * R(o.dz);
  const R oned3 = R(1) / R(3);
  for (int k = 2; k <= o.nk - 2; ++k)
    for (int j = 2; j <= o.nj - 2; ++j)
      for (int i = 2; i <= o.ni - 2; ++i) {
        const R priv = tw.priv(i, j, k);
        const R ln = (priv - R(1)) * std::exp(oned3 * std::log(ds308 * b.jcb(i, j, k))) + R(TurbConst::eps);
        const R e = tke(i, j, k);
        tkefrc(i, j, k) = tkefrc(i, j, k) - (R(.37) * priv - R(.18)) * b.rst(i, j, k) * e * std::sqrt(e) / ln;
      }
}

// s_eddyvisj mfcopt=0 (SrcOrig/eddyvisj.f90:121-134): rkh, rkv divided by jcb.
template <class R>
void eddyvisj(const Opts& o, const Base<R>& b, TurbWork<R>& tw) {
  for (int k = 1; k <= o.nk - 1; ++k)
    for (int j = 1; j <= o.nj - 1; ++j)
      for (int i = 1; i <= o.ni - 1; ++i) {
        const R jcbiv = R(1) / b.jcb(i, j, k);
        tw.rkh(i, j, k) = jcbiv * tw.rkh(i, j, k);
        tw.rkv(i, j, k) = jcbiv * tw.rkv(i, j, k);
      }
}

// s_tkeflx (SrcOrig/tkeflx.f90:251-462, trnopt=0, mfcopt=0) and s_turbtke
// (SrcOrig/turbtke.f90:203-237): turbulent transport of the past-level
// TKE with twice the momentum diffusivity (the 2/dx of the divergence),
// added to tkefrc.
template <class R>
void turbtke(const Opts& o, const Base<R>& b, const F3<R>& tke, TurbWork<R>& tw, F3<R>& tkefrc) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dxiv = R(1) / R(o.dx), dyiv = R(1) / R(o.dy), dziv = R(1) / R(o.dz);
  const R dxv5 = R(.5) * dxiv, dyv5 = R(.5) * dyiv, dzv5 = R(.5) * dziv;
  const R dxiv2 = R(2) * dxiv, dyiv2 = R(2) * dyiv, dziv2 = R(2) * dziv;
  F3<R>& jt = tw.jcbs;
  for (int k = 1; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) jt(i, j, k) = tke(i, j, k) * b.jcb(i, j, k);
  for (int k = 1; k <= nk - 1; ++k) {
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i)
        tw.h1(i, j, k) = (tw.rkh(i - 1, j, k) + tw.rkh(i, j, k)) * (jt(i, j, k) - jt(i - 1, j, k)) * dxv5;
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        tw.h2(i, j, k) = (tw.rkh(i, j - 1, k) + tw.rkh(i, j, k)) * (jt(i, j, k) - jt(i, j - 1, k)) * dyv5;
  }
  for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        tw.h3(i, j, k) = (tw.rkv(i, j, k - 1) + tw.rkv(i, j, k)) * (tke(i, j, k) - tke(i, j, k - 1)) * dzv5;
  F3<R>&a = tw.tmp1, &c = tw.tmp2;
  for (int k = 2; k <= nk - 2; ++k) {
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i) a(i, j, k) = b.jcb8u(i, j, k) * tw.h1(i, j, k);
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i) c(i, j, k) = b.jcb8v(i, j, k) * tw.h2(i, j, k);
  }
  for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        tkefrc(i, j, k) = tkefrc(i, j, k) + ((tw.h3(i, j, k + 1) - tw.h3(i, j, k)) * dziv2 +
                                             ((a(i + 1, j, k) - a(i, j, k)) * dxiv2 + (c(i, j + 1, k) - c(i, j, k)) * dyiv2));
}

// s_eddydif tubopt>=2, isoopt=1 (SrcOrig/eddydif.f90:265-284, 333-359) after
// s_eddyvisj, and s_kh8uv mfcopt=0 (SrcOrig/kh8uv.f90:211-230): the scalar
// diffusivities rkh = 1/Pr rkv (rkv already divided by jcb), rkh8u, rkh8v,
// rkv8w (into rkv), and the half value 0.5 jcb rkh at scalar points
// (rkv8s) that the buoyancy production uses.
template <class R>
void eddydif_tke(const Opts& o, const Base<R>& b, TurbWork<R>& tw) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  for (int k = 1; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) {
        tw.rkv8s(i, j, k) = tw.priv(i, j, k) * tw.rkv(i, j, k);
        tw.rkh(i, j, k) = tw.rkv8s(i, j, k);
      }
  for (int k = 2; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) tw.rkv(i, j, k) = R(.5) * (tw.rkv8s(i, j, k - 1) + tw.rkv8s(i, j, k));
  for (int k = 1; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) tw.rkv8s(i, j, k) = R(.5) * b.jcb(i, j, k) * tw.rkv8s(i, j, k);
  for (int k = 1; k <= nk - 1; ++k) {
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 1; ++i) tw.rkh8u(i, j, k) = tw.rkh(i - 1, j, k) + tw.rkh(i, j, k);
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) tw.rkh8v(i, j, k) = tw.rkh(i, j - 1, k) + tw.rkh(i, j, k);
  }
}

// s_buoytke, SrcOrig/buoytke.f90:124-151: buoyancy production
// -(b(k) + b(k+1)) with b(k) = jcb8w N^2(k) (rkv8s(k-1) + rkv8s(k)).
template <class R>
void buoytke(const Opts& o, const Base<R>& b, TurbWork<R>& tw, F3<R>& tkefrc) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  F3<R>& t = tw.tmp1;
  for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        t(i, j, k) = b.jcb8w(i, j, k) * tw.nsq8w(i, j, k) * (tw.rkv8s(i, j, k - 1) + tw.rkv8s(i, j, k));
  for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) tkefrc(i, j, k) = tkefrc(i, j, k) - (t(i, j, k) + t(i, j, k + 1));
}

// s_strsten, SrcOrig/strsten.f90:150-262 (sfcopt=0): the stresses.
template <class R>
void strsten(const Opts& o, TurbWork<R>& tw) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const F3<R>&rkh = tw.rkh, &rkv = tw.rkv;
  for (int k = 1; k <= nk - 1; ++k) {
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) {
        tw.t11(i, j, k) = rkh(i, j, k) * tw.t11(i, j, k);
        tw.t22(i, j, k) = rkh(i, j, k) * tw.t22(i, j, k);
        tw.t33(i, j, k) = rkv(i, j, k) * tw.t33(i, j, k);
      }
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 1; ++i)
        tw.t12(i, j, k) = R(.25) * tw.t12(i, j, k) *
                          ((rkh(i - 1, j - 1, k) + rkh(i, j, k)) + (rkh(i - 1, j, k) + rkh(i, j - 1, k)));
  }
  for (int k = 2; k <= nk - 1; ++k) {
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i)
        tw.t13(i, j, k) = R(.25) * tw.t13(i, j, k) *
                          ((rkv(i - 1, j, k - 1) + rkv(i, j, k)) + (rkv(i - 1, j, k) + rkv(i, j, k - 1)));
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        tw.t23(i, j, k) = R(.25) * tw.t23(i, j, k) *
                          ((rkv(i, j - 1, k - 1) + rkv(i, j, k)) + (rkv(i, j - 1, k) + rkv(i, j, k - 1)));
  }
  for (int k = 2; k <= nk - 1; ++k) {
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i)
        tw.t31(i, j, k) = R(.25) * tw.t31(i, j, k) *
                          ((rkh(i - 1, j, k - 1) + rkh(i, j, k)) + (rkh(i - 1, j, k) + rkh(i, j, k - 1)));
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        tw.t32(i, j, k) = R(.25) * tw.t32(i, j, k) *
                          ((rkh(i, j - 1, k - 1) + rkh(i, j, k)) + (rkh(i, j - 1, k) + rkh(i, j, k - 1)));
  }
  bcten(o, tw.t31);
  bcten(o, tw.t32);
}

// s_turbuvw, SrcOrig/turbuvw.f90:284-1340 (trnopt=0, mfcopt=0, advopt<=3):
// the divergence of the stresses SETS ufrc, vfrc, wfrc on their ranges.
template <class R>
void turbuvw(const Opts& o, const Base<R>& b, TurbWork<R>& tw, F3<R>& ufrc, F3<R>& vfrc, F3<R>& wfrc) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dxiv = R(1) / R(o.dx), dyiv = R(1) / R(o.dy), dziv = R(1) / R(o.dz);
  const R dxiv05 = R(.5) * dxiv, dyiv05 = R(.5) * dyiv;
  F3<R>&a = tw.tmp1, &c = tw.tmp2;
  for (int k = 2; k <= nk - 2; ++k) {   // u, turbuvw.f90:288-333
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 1; i <= ni - 1; ++i) a(i, j, k) = b.jcb(i, j, k) * tw.t11(i, j, k);
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 1; ++i) c(i, j, k) = (b.jcb8u(i, j - 1, k) + b.jcb8u(i, j, k)) * tw.t12(i, j, k);
  }
  for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i)
        ufrc(i, j, k) = ((a(i, j, k) - a(i - 1, j, k)) * dxiv + (c(i, j + 1, k) - c(i, j, k)) * dyiv05) +
                        (tw.t13(i, j, k + 1) - tw.t13(i, j, k)) * dziv;
  for (int k = 2; k <= nk - 2; ++k) {   // v, turbuvw.f90:795-840
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i) a(i, j, k) = b.jcb(i, j, k) * tw.t22(i, j, k);
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 1; ++i) c(i, j, k) = (b.jcb8v(i - 1, j, k) + b.jcb8v(i, j, k)) * tw.t12(i, j, k);
  }
  for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        vfrc(i, j, k) = ((a(i, j, k) - a(i, j - 1, k)) * dyiv + (c(i + 1, j, k) - c(i, j, k)) * dxiv05) +
                        (tw.t23(i, j, k + 1) - tw.t23(i, j, k)) * dziv;
  for (int k = 2; k <= nk - 1; ++k) {   // w, turbuvw.f90:1300-1330
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i) a(i, j, k) = (b.jcb8u(i, j, k - 1) + b.jcb8u(i, j, k)) * tw.t31(i, j, k);
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i) c(i, j, k) = (b.jcb8v(i, j, k - 1) + b.jcb8v(i, j, k)) * tw.t32(i, j, k);
  }
  for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        wfrc(i, j, k) = (tw.t33(i, j, k) - tw.t33(i, j, k - 1)) * dziv +
                        ((a(i + 1, j, k) - a(i, j, k)) * dxiv05 + (c(i, j + 1, k) - c(i, j, k)) * dyiv05);
}

// s_eddydif tubopt=1, isoopt=1, mfcopt=0 (SrcOrig/eddydif.f90:154-260) and
// s_kh8uv mfcopt=0 (SrcOrig/kh8uv.f90:211-230): scalar diffusivities rkh
// (scalar points), rkh8u, rkh8v (u, v points) and rkv8w (w points, into rkv).
template <class R>
void eddydif(const Opts& o, const Base<R>& b, TurbWork<R>& tw) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  for (int k = 1; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) {
        tw.rkv8s(i, j, k) = tw.priv(i, j, k) * tw.rkv(i, j, k) / b.jcb(i, j, k);
        tw.rkh(i, j, k) = tw.rkv8s(i, j, k);
      }
  for (int k = 2; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) tw.rkv(i, j, k) = R(.5) * (tw.rkv8s(i, j, k - 1) + tw.rkv8s(i, j, k));
  for (int k = 1; k <= nk - 1; ++k) {
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 1; ++i) tw.rkh8u(i, j, k) = tw.rkh(i - 1, j, k) + tw.rkh(i, j, k);
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) tw.rkh8v(i, j, k) = tw.rkh(i, j - 1, k) + tw.rkh(i, j, k);
  }
}

// s_turbflx (SrcOrig/turbflx.f90:236-352, trnopt=0, sfcopt=0) and s_turbs
// (SrcOrig/turbs.f90:189-232, mfcopt=0): turbulent mixing of the scalar s,
// added to sfrc.
template <class R>
void turbs(const Opts& o, const Base<R>& b, const F3<R>& s, TurbWork<R>& tw, F3<R>& sfrc) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dxiv = R(1) / R(o.dx), dyiv = R(1) / R(o.dy), dziv = R(1) / R(o.dz);
  const R dxv05 = R(.5) * dxiv, dyv05 = R(.5) * dyiv;
  for (int k = 1; k <= nk - 1; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) tw.jcbs(i, j, k) = s(i, j, k) * b.jcb(i, j, k);
  for (int k = 1; k <= nk - 1; ++k) {
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i)
        tw.h1(i, j, k) = tw.rkh8u(i, j, k) * (tw.jcbs(i, j, k) - tw.jcbs(i - 1, j, k)) * dxv05;
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        tw.h2(i, j, k) = tw.rkh8v(i, j, k) * (tw.jcbs(i, j, k) - tw.jcbs(i, j - 1, k)) * dyv05;
  }
  for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) tw.h3(i, j, k) = tw.rkv(i, j, k) * (s(i, j, k) - s(i, j, k - 1)) * dziv;
  F3<R>&a = tw.tmp1, &c = tw.tmp2;
  for (int k = 2; k <= nk - 2; ++k) {
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i) a(i, j, k) = b.jcb8u(i, j, k) * tw.h1(i, j, k);
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i) c(i, j, k) = b.jcb8v(i, j, k) * tw.h2(i, j, k);
  }
  for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        sfrc(i, j, k) = sfrc(i, j, k) + ((tw.h3(i, j, k + 1) - tw.h3(i, j, k)) * dziv +
                                         ((a(i + 1, j, k) - a(i, j, k)) * dxiv + (c(i, j + 1, k) - c(i, j, k)) * dyiv));
}

}  // namespace oracle

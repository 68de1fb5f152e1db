// Oracle: the base state from a sounding (hydrostatic Exner integration,
// humidity iteration, interpolation to the model levels, base density and
// rho c^2) for a horizontally uniform grid.
//
// TEST INFRASTRUCTURE ONLY (see arr.h).  Each function restates one
// reference routine and cites it; R is float (the reference's default
// `real`) or double.
#pragma once
#include <cmath>
#include <vector>
#include "phys.h"

namespace oracle {

struct BaseConst {
  static constexpr double epsav = 1.6077;   // comphy.f90:82
  static constexpr double tlow = 233.16;    // comphy.f90:100
  static constexpr double eps = 1.e-20;     // commath.f90:177
  static constexpr double lim36 = 1.e36;    // commath.f90:183
};

// Sounding on levels kl = 0..nlev (level 0 is filled by vextlow).
template <class R>
struct Sounding {
  int nlev = 0;
  std::vector<R> z, u, v, p, pt, qv, t;
};

// s_set1d for height-level soundings (sndtyp(1:1) = 'z'), SrcOrig/set1d.f90:
// 278-452: potential temperature ('p') or temperature ('t') given,
// humidity as relative humidity in percent ('r') or mixing ratio; the
// hydrostatic integration (in Exner function or log p) and the humidity
// iterated until the mixing ratios change by less than 1e-5; then mixing
// ratios at or below thresq set to 0 (set1d.f90:536-540).  Returns 0, or 1
// when the integration reaches a non-positive pressure (set1d.f90:330-346).
template <class R>
int set1d_z(char tvar, char hvar, R psnd0, R thresq, Sounding<R>& s) {
  using std::exp; using std::log; using std::abs; using std::max; using std::min;
  const int nlev = s.nlev;
  const R g = R(Phys::g), cp = R(Phys::cp), rd = R(Phys::rd), p0 = R(Phys::p0);
  const R gdvcp2 = R(2) * g / cp, gdvrd2 = R(2) * g / rd, rddvcp = rd / cp, cpdvrd = cp / rd;
  const R p0iv = R(1) / p0, es001 = R(.01) * R(Phys::es0), qvveps = R(1.e-5);
  const R epsav = R(BaseConst::epsav), epsva = R(Phys::epsva), t0 = R(Phys::t0), tlow = R(BaseConst::tlow);
  const R eps = R(BaseConst::eps);
  std::vector<R> ltmp1(nlev + 1), ltmp2(nlev + 1);
  if (tvar == 't') {
    ltmp1[1] = log(psnd0);
    for (int kl = 1; kl <= nlev; ++kl) s.t[kl] = s.pt[kl];
  } else {
    ltmp1[1] = exp(rddvcp * log(p0iv * psnd0));
  }
  if (hvar == 'r') {
    for (int kl = 1; kl <= nlev; ++kl) { ltmp2[kl] = s.qv[kl]; s.qv[kl] = R(0); }
  }
  for (int it = 0; it < 1000; ++it) {
    R lpmin = R(BaseConst::lim36), pimin = R(BaseConst::lim36), itcon = R(0);
    if (tvar == 't') {
      for (int kl = 1; kl <= nlev; ++kl) s.pt[kl] = s.t[kl] * (R(1) + epsav * s.qv[kl]) / (R(1) + s.qv[kl]);
      for (int kl = 2; kl <= nlev; ++kl) {
        ltmp1[kl] = ltmp1[kl - 1] - gdvrd2 * (s.z[kl] - s.z[kl - 1]) / (s.pt[kl - 1] + s.pt[kl]);
        lpmin = min(ltmp1[kl], lpmin);
      }
      if (lpmin <= R(0)) return 1;
      for (int kl = 1; kl <= nlev; ++kl) {
        s.p[kl] = exp(ltmp1[kl]);
        s.pt[kl] = s.t[kl] * exp(rddvcp * log(p0 / s.p[kl]));
      }
    } else {
      for (int kl = 1; kl <= nlev; ++kl) s.t[kl] = s.pt[kl] * (R(1) + epsav * s.qv[kl]) / (R(1) + s.qv[kl]);
      for (int kl = 2; kl <= nlev; ++kl) {
        ltmp1[kl] = ltmp1[kl - 1] - gdvcp2 * (s.z[kl] - s.z[kl - 1]) / (s.t[kl - 1] + s.t[kl]);
        pimin = min(ltmp1[kl], pimin);
      }
      if (pimin <= R(0)) return 1;
      for (int kl = 1; kl <= nlev; ++kl) {
        s.p[kl] = p0 * exp(cpdvrd * log(ltmp1[kl]));
        s.t[kl] = s.pt[kl] * ltmp1[kl];
      }
    }
    if (hvar == 'r') {
      for (int kl = 1; kl <= nlev; ++kl) {
        const R tk = s.t[kl];
        const R ea = tk > tlow ? es001 * ltmp2[kl] * exp(R(17.269) * (tk - t0) / (tk - R(35.86)))
                               : es001 * ltmp2[kl] * exp(R(21.875) * (tk - t0) / (tk - R(7.66)));
        const R qvf = epsva * ea / (s.p[kl] - ea);
        const R dqv = abs((qvf + eps) / (s.qv[kl] + eps) - R(1));
        s.qv[kl] = qvf;
        itcon = max(dqv, itcon);
      }
    }
    if (itcon < qvveps) break;
  }
  for (int kl = 1; kl <= nlev; ++kl)
    if (s.qv[kl] <= thresq) s.qv[kl] = R(0);
  return 0;
}

// s_vextlow('oooooo'), SrcOrig/vextlow.f90:150-220: level 0 below the
// sounding, linear extrapolation of u, v, theta, qv and a hydrostatic p.
template <class R>
void vextlow(Sounding<R>& s) {
  using std::exp; using std::log; using std::min;
  const R g = R(Phys::g), cp = R(Phys::cp), rd = R(Phys::rd), p0 = R(Phys::p0);
  const R gdvcp2 = R(2) * g / cp, cpdvrd = cp / rd, rddvcp = rd / cp, p0iv = R(1) / p0;
  const R epsav = R(BaseConst::epsav);
  s.z[0] = min(R(2) * s.z[1] - s.z[2], R(0));
  auto ext = [&](std::vector<R>& a) {
    a[0] = ((s.z[2] - s.z[0]) * a[1] - (s.z[1] - s.z[0]) * a[2]) / (s.z[2] - s.z[1]);
  };
  ext(s.u); ext(s.v); ext(s.pt); ext(s.qv);
  const R ptv0 = s.pt[0] * (R(1) + s.qv[0]) / (R(1) + epsav * s.qv[0]);
  const R ptv1 = s.pt[1] * (R(1) + s.qv[1]) / (R(1) + epsav * s.qv[1]);
  const R pi0 = exp(rddvcp * log(p0iv * s.p[1])) + gdvcp2 * (s.z[1] - s.z[0]) / (ptv0 + ptv1);
  s.p[0] = p0 * exp(cpdvrd * log(pi0));
}

// s_vint13 at one height, SrcOrig/vint13.f90:120-170: linear in height
// between sounding levels, extrapolated below level 0 and above level nlev.
template <class R>
R vint13(const Sounding<R>& s, const std::vector<R>& var, R z) {
  const int nlev = s.nlev;
  R out = R(0);
  if (s.z[0] > z) {
    const R dk = (R(1) / (s.z[1] - s.z[0])) * (z - s.z[0]);
    out = (R(1) - dk) * var[0] + dk * var[1];
  } else if (s.z[nlev] <= z) {
    const R dk = (R(1) / (s.z[nlev] - s.z[nlev - 1])) * (z - s.z[nlev - 1]);
    out = (R(1) - dk) * var[nlev - 1] + dk * var[nlev];
  }
  for (int kl = 0; kl <= nlev - 1; ++kl)
    if (s.z[kl] <= z && s.z[kl + 1] > z) {
      const R dk = (z - s.z[kl]) / (s.z[kl + 1] - s.z[kl]);
      out = (R(1) - dk) * var[kl] + dk * var[kl + 1];
    }
  return out;
}

// Base-state columns, index k = 1..nk (position 0 unused).
template <class R>
struct BaseColumn {
  std::vector<R> ubr, vbr, pbr, ptbr, qvbr, rbr, ptvbr, pibr, rst, rst8w, rcsq;
};

// s_intrpsnd (intrpsnd.f90:190-230, height soundings), s_setbase
// (setbase.f90:153-189) with s_bcbase (bcbase.f90:150-210), s_baserho
// (baserho.f90:150-160: rst = |jcb| rbr; var8uvw.f90:190-196 and
// bc8w.f90:136,166 for rst8w) and s_sndwave (sndwave.f90:119: rcsq =
// cp/cv pbr) on one column of w-level heights zph(1..nk) and Jacobian
// jcb(1..nk).  Levels 1..nk-1 follow the reference; level nk, which the
// reference leaves unset, repeats level nk-1 (rst8w: bc8w's level nk-2).
template <class R>
void base_column(int nk, const R* zph, const R* jcb, const Sounding<R>& s, BaseColumn<R>& c) {
  using std::exp; using std::log; using std::abs;
  const R g = R(Phys::g), cp = R(Phys::cp), cv = R(Phys::cv), rd = R(Phys::rd), p0 = R(Phys::p0);
  const R gdvcp2 = R(2) * g / cp, cpdvrd = cp / rd, rddvcp = rd / cp, p0iv = R(1) / p0;
  const R epsav = R(BaseConst::epsav);
  for (auto* v : {&c.ubr, &c.vbr, &c.pbr, &c.ptbr, &c.qvbr, &c.rbr, &c.ptvbr, &c.pibr, &c.rst, &c.rst8w, &c.rcsq})
    v->assign(nk + 1, R(0));
  std::vector<R> z8s(nk + 1, R(0));
  for (int k = 1; k <= nk - 1; ++k) z8s[k] = R(.5) * (zph[k + 1] + zph[k]);   // setbase.f90:153
  for (int k = 2; k <= nk - 2; ++k) {
    c.ubr[k] = vint13(s, s.u, z8s[k]);
    c.vbr[k] = vint13(s, s.v, z8s[k]);
    c.pbr[k] = vint13(s, s.p, z8s[k]);
    c.ptbr[k] = vint13(s, s.pt, z8s[k]);
    c.qvbr[k] = vint13(s, s.qv, z8s[k]);
    c.ptvbr[k] = c.ptbr[k] * (R(1) + epsav * c.qvbr[k]) / (R(1) + c.qvbr[k]);
    c.pibr[k] = exp(rddvcp * log(p0iv * c.pbr[k]));
    c.rbr[k] = c.pbr[k] / (rd * c.ptvbr[k] * c.pibr[k]);
  }
  const int k1 = nk - 1, k2 = nk - 2;
  c.ubr[1] = c.ubr[2]; c.ubr[k1] = c.ubr[k2];
  c.vbr[1] = c.vbr[2]; c.vbr[k1] = c.vbr[k2];
  c.ptbr[1] = c.ptbr[2]; c.ptbr[k1] = c.ptbr[k2];
  c.qvbr[1] = c.qvbr[2]; c.qvbr[k1] = c.qvbr[k2];
  c.ptvbr[1] = c.ptvbr[2]; c.ptvbr[k1] = c.ptvbr[k2];
  c.pibr[1] = c.pibr[2] + gdvcp2 * (z8s[2] - z8s[1]) / (c.ptvbr[1] + c.ptvbr[2]);
  c.pibr[k1] = c.pibr[k2] - gdvcp2 * (z8s[k1] - z8s[k2]) / (c.ptvbr[k2] + c.ptvbr[k1]);
  for (int k : {1, k1}) {
    c.pbr[k] = p0 * exp(cpdvrd * log(c.pibr[k]));
    c.rbr[k] = c.pbr[k] / (rd * c.ptvbr[k] * c.pibr[k]);
  }
  for (int k = 1; k <= nk - 1; ++k) {
    c.rst[k] = abs(jcb[k]) * c.rbr[k];
    c.rcsq[k] = (cp / cv) * c.pbr[k];
  }
  for (int k = 2; k <= nk - 1; ++k) c.rst8w[k] = R(.5) * (c.rst[k - 1] + c.rst[k]);
  c.rst8w[1] = c.rst8w[3];
  c.rst8w[nk] = c.rst8w[nk - 2];
  for (auto* v : {&c.ubr, &c.vbr, &c.pbr, &c.ptbr, &c.qvbr, &c.rbr, &c.ptvbr, &c.pibr, &c.rst, &c.rcsq})
    (*v)[nk] = (*v)[nk - 1];
}

}  // namespace oracle

// Oracle: large-step forcing, leapfrog scalar step, Asselin filter and the
// periodic halo planes, for idealized runs (flat terrain, mfcopt=0,
// periodic lateral boundaries on one process, advopt=2, smtopt=2/3,
// vspopt=2, coropt=0/1, buyopt=1, gwmopt=0, impopt=1).
//
// TEST INFRASTRUCTURE ONLY (see arr.h).  Every routine restates the cited
// Fortran: same loop ranges, same parenthesisation.
#pragma once
#include <cmath>
#include <string>
#include "small.h"

namespace oracle {

struct LargeOpts {
  int advopt = 2;      // 2: 4th-order horizontal, 2nd-order vertical (advuvw.f90:292-397)
  int smtopt = 3;      // 2: horizontal 4th order; 3: + vertical (smoo4s.f90:248-296)
  double smhcoe = 0.001, smvcoe = 0.0004;
  int vspopt = 2;      // Rayleigh damping toward the base state (vsps.f90:181-198)
  std::string vspvar = "oooxoooooo";  // u v w p pt qv qw ... (vsps/vspuvw switches)
  int ksp0 = 2;        // first damped level (vspdmp.f90:222-232)
  int coropt = 0;      // 1: f-plane Coriolis on u, v (coriuv.f90:124-182)
  int tubopt = 0;      // 0: no turbulence; 1: Smagorinsky
  double filcoe = 0.1; // Asselin coefficient (timeflt.f90:335)
  int moist = 0;       // fmois: 0 'dry', 1 'moist'
};

// Full periodic wrap of both ghost layers (s_bcycle with the stepper
// arguments, bcycle.f90:159-225, then shift2nd.f90:4274-4300 for the second
// plane).  stag: 's' scalar/w, 'u', 'v'.
template <class R>
void halo_both(const Opts& o, char stag, F3<R>& a) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  if (stag == 'u') {
    bcycle(o, 3, 1, ni - 2, ni, 2, 1, nj - 2, nj - 1, nk, a);
    bcycle(o, 4, 0, ni - 3, ni + 1, 3, 0, nj - 3, nj, nk, a);
  } else if (stag == 'v') {
    bcycle(o, 2, 1, ni - 2, ni - 1, 3, 1, nj - 2, nj, nk, a);
    bcycle(o, 3, 0, ni - 3, ni, 4, 0, nj - 3, nj + 1, nk, a);
  } else {
    bcycle(o, 2, 1, ni - 2, ni - 1, 2, 1, nj - 2, nj - 1, nk, a);
    bcycle(o, 3, 0, ni - 3, ni, 3, 0, nj - 3, nj, nk, a);
  }
}

// s_rstuvwc, SrcOrig/rstuvwc.f90:172-210 (mfcopt=0, periodic: iwest=ieast=0).
template <class R>
void rstuvwc(const Opts& o, const Base<R>& b, const F3<R>& u, const F3<R>& v, const F3<R>& wc,
             F3<R>& rxu, F3<R>& rxv, F3<R>& rxw) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  OMP_FOR for (int k = 1; k <= nk - 1; ++k) {
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 0; i <= ni + 1; ++i) rxu(i, j, k) = b.rst8u(i, j, k) * u(i, j, k);
    for (int j = 0; j <= nj + 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) rxv(i, j, k) = b.rst8v(i, j, k) * v(i, j, k);
  }
  OMP_FOR for (int k = 1; k <= nk; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) rxw(i, j, k) = b.rst8w(i, j, k) * wc(i, j, k);
}

// s_advuvw advopt=2 or 3, SrcOrig/advuvw.f90:209-430 (u), 458-657 (v), 685-884 (w).
template <class R>
void advuvw(const Opts& o, const F3<R>& rxu, const F3<R>& rxv, const F3<R>& rxw, const F3<R>& u,
            const F3<R>& v, const F3<R>& w, F3<R>& ufrc, F3<R>& vfrc, F3<R>& wfrc, F3<R>& t1,
            F3<R>& t2, F3<R>& t3, F3<R>& hadv) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dxiv = R(1) / R(o.dx), dyiv = R(1) / R(o.dy), dziv = R(1) / R(o.dz);
  const R oned24 = R(1) / R(24), fourd3 = R(4) / R(3);   // commath.f90:63,75
  const R dxv25n = R(-.25) * dxiv, dyv25n = R(-.25) * dyiv, dzv25n = R(-.25) * dziv;
  const R dxv24 = oned24 * dxiv, dyv24 = oned24 * dyiv;
  const R dxv48 = R(.5) * dxv24, dyv48 = R(.5) * dyv24;
  const R dzv24 = oned24 * dziv, dzv48 = R(.5) * dzv24;
  const int iw = o.iw(), ie = o.ie();   // open x: 4th order away from the boundary columns
  // ---- u (advuvw.f90:231-397)
  OMP_FOR for (int k = 2; k <= nk - 2; ++k) {
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 1; i <= ni - 1; ++i)
        t1(i, j, k) = (rxu(i, j, k) + rxu(i + 1, j, k)) * (u(i + 1, j, k) - u(i, j, k)) * dxv25n;
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 1; ++i)
        t2(i, j, k) = (rxv(i - 1, j, k) + rxv(i, j, k)) * (u(i, j, k) - u(i, j - 1, k)) * dyv25n;
  }
  OMP_FOR for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i)
        t3(i, j, k) = (rxw(i - 1, j, k) + rxw(i, j, k)) * (u(i, j, k) - u(i, j, k - 1)) * dzv25n;
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i)
        hadv(i, j, k) = (t1(i - 1, j, k) + t1(i, j, k)) + (t2(i, j, k) + t2(i, j + 1, k));
  OMP_FOR for (int k = 2; k <= nk - 2; ++k) {
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 1 + iw; i <= ni - ie; ++i)
        t1(i, j, k) = (rxu(i - 1, j, k) + rxu(i + 1, j, k)) * (u(i + 1, j, k) - u(i - 1, j, k)) * dxv24;
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 2 + iw; i <= ni - 1 - ie; ++i)
        t2(i, j, k) = ((rxv(i - 1, j, k) + rxv(i, j, k)) + (rxv(i - 1, j + 1, k) + rxv(i, j + 1, k))) *
                      (u(i, j + 1, k) - u(i, j - 1, k)) * dyv48;
  }
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2 + iw; i <= ni - 1 - ie; ++i)
        hadv(i, j, k) = fourd3 * hadv(i, j, k) +
                        ((t1(i - 1, j, k) + t1(i + 1, j, k)) + (t2(i, j - 1, k) + t2(i, j + 1, k)));
  if (o.advopt == 3) {   // advuvw.f90:309-335, 399-430: 4th order in z on k = 3..nk-3
    F3<R> va(ni, nj, nk), tz(ni, nj, nk);
    for (int k = 2; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 1; ++i) {
          va(i, j, k) = t3(i, j, k) + t3(i, j, k + 1);
          tz(i, j, k) = ((rxw(i - 1, j, k) + rxw(i, j, k)) + (rxw(i - 1, j, k + 1) + rxw(i, j, k + 1))) *
                        (u(i, j, k + 1) - u(i, j, k - 1)) * dzv48;
        }
    for (int k = 3; k <= nk - 3; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 1; ++i) va(i, j, k) = fourd3 * va(i, j, k) + (tz(i, j, k - 1) + tz(i, j, k + 1));
    for (int k = 2; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 1; ++i) ufrc(i, j, k) = ufrc(i, j, k) + hadv(i, j, k) + va(i, j, k);
  } else {
    OMP_FOR for (int k = 2; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 1; ++i)
          ufrc(i, j, k) = ufrc(i, j, k) + hadv(i, j, k) + (t3(i, j, k) + t3(i, j, k + 1));
  }
  // ---- v (advuvw.f90:458-624)
  OMP_FOR for (int k = 2; k <= nk - 2; ++k) {
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 1; ++i)
        t1(i, j, k) = (rxu(i, j - 1, k) + rxu(i, j, k)) * (v(i, j, k) - v(i - 1, j, k)) * dxv25n;
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        t2(i, j, k) = (rxv(i, j, k) + rxv(i, j + 1, k)) * (v(i, j + 1, k) - v(i, j, k)) * dyv25n;
  }
  OMP_FOR for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        t3(i, j, k) = (rxw(i, j - 1, k) + rxw(i, j, k)) * (v(i, j, k) - v(i, j, k - 1)) * dzv25n;
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        hadv(i, j, k) = (t1(i, j, k) + t1(i + 1, j, k)) + (t2(i, j - 1, k) + t2(i, j, k));
  OMP_FOR for (int k = 2; k <= nk - 2; ++k) {
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 1 + iw; i <= ni - 1 - ie; ++i)
        t1(i, j, k) = ((rxu(i, j - 1, k) + rxu(i, j, k)) + (rxu(i + 1, j - 1, k) + rxu(i + 1, j, k))) *
                      (v(i + 1, j, k) - v(i - 1, j, k)) * dxv48;
    for (int j = 1; j <= nj; ++j)
      for (int i = 2 + iw; i <= ni - 2 - ie; ++i)
        t2(i, j, k) = (rxv(i, j - 1, k) + rxv(i, j + 1, k)) * (v(i, j + 1, k) - v(i, j - 1, k)) * dyv24;
  }
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2 + iw; i <= ni - 2 - ie; ++i)
        hadv(i, j, k) = fourd3 * hadv(i, j, k) +
                        ((t1(i - 1, j, k) + t1(i + 1, j, k)) + (t2(i, j - 1, k) + t2(i, j + 1, k)));
  if (o.advopt == 3) {   // advuvw.f90:536-562, 626-657
    F3<R> va(ni, nj, nk), tz(ni, nj, nk);
    for (int k = 2; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 1; ++j)
        for (int i = 2; i <= ni - 2; ++i) {
          va(i, j, k) = t3(i, j, k) + t3(i, j, k + 1);
          tz(i, j, k) = ((rxw(i, j - 1, k) + rxw(i, j, k)) + (rxw(i, j - 1, k + 1) + rxw(i, j, k + 1))) *
                        (v(i, j, k + 1) - v(i, j, k - 1)) * dzv48;
        }
    for (int k = 3; k <= nk - 3; ++k)
      for (int j = 2; j <= nj - 1; ++j)
        for (int i = 2; i <= ni - 2; ++i) va(i, j, k) = fourd3 * va(i, j, k) + (tz(i, j, k - 1) + tz(i, j, k + 1));
    for (int k = 2; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 1; ++j)
        for (int i = 2; i <= ni - 2; ++i) vfrc(i, j, k) = vfrc(i, j, k) + hadv(i, j, k) + va(i, j, k);
  } else {
    OMP_FOR for (int k = 2; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 1; ++j)
        for (int i = 2; i <= ni - 2; ++i)
          vfrc(i, j, k) = vfrc(i, j, k) + hadv(i, j, k) + (t3(i, j, k) + t3(i, j, k + 1));
  }
  // ---- w (advuvw.f90:685-852)
  OMP_FOR for (int k = 2; k <= nk - 1; ++k) {
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i)
        t1(i, j, k) = (rxu(i, j, k - 1) + rxu(i, j, k)) * (w(i, j, k) - w(i - 1, j, k)) * dxv25n;
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        t2(i, j, k) = (rxv(i, j, k - 1) + rxv(i, j, k)) * (w(i, j, k) - w(i, j - 1, k)) * dyv25n;
  }
  OMP_FOR for (int k = 1; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        t3(i, j, k) = (rxw(i, j, k) + rxw(i, j, k + 1)) * (w(i, j, k + 1) - w(i, j, k)) * dzv25n;
  OMP_FOR for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        hadv(i, j, k) = (t1(i, j, k) + t1(i + 1, j, k)) + (t2(i, j, k) + t2(i, j + 1, k));
  OMP_FOR for (int k = 2; k <= nk - 1; ++k) {
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 1 + iw; i <= ni - 1 - ie; ++i)
        t1(i, j, k) = ((rxu(i, j, k - 1) + rxu(i, j, k)) + (rxu(i + 1, j, k - 1) + rxu(i + 1, j, k))) *
                      (w(i + 1, j, k) - w(i - 1, j, k)) * dxv48;
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 2 + iw; i <= ni - 2 - ie; ++i)
        t2(i, j, k) = ((rxv(i, j, k - 1) + rxv(i, j, k)) + (rxv(i, j + 1, k - 1) + rxv(i, j + 1, k))) *
                      (w(i, j + 1, k) - w(i, j - 1, k)) * dyv48;
  }
  OMP_FOR for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2 + iw; i <= ni - 2 - ie; ++i)
        hadv(i, j, k) = fourd3 * hadv(i, j, k) +
                        ((t1(i - 1, j, k) + t1(i + 1, j, k)) + (t2(i, j - 1, k) + t2(i, j + 1, k)));
  if (o.advopt == 3) {   // advuvw.f90:763-789, 854-884
    F3<R> va(ni, nj, nk), tz(ni, nj, nk);
    for (int k = 2; k <= nk - 1; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 2; ++i) {
          va(i, j, k) = t3(i, j, k - 1) + t3(i, j, k);
          tz(i, j, k) = (rxw(i, j, k - 1) + rxw(i, j, k + 1)) * (w(i, j, k + 1) - w(i, j, k - 1)) * dzv24;
        }
    for (int k = 3; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 2; ++i) va(i, j, k) = fourd3 * va(i, j, k) + (tz(i, j, k - 1) + tz(i, j, k + 1));
    for (int k = 2; k <= nk - 1; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 2; ++i) wfrc(i, j, k) = wfrc(i, j, k) + hadv(i, j, k) + va(i, j, k);
  } else {
    OMP_FOR for (int k = 2; k <= nk - 1; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 2; ++i)
          wfrc(i, j, k) = wfrc(i, j, k) + hadv(i, j, k) + (t3(i, j, k - 1) + t3(i, j, k));
  }
}

// s_advs advopt=2 or 3, SrcOrig/advs.f90:189-416: sfrc = advection of s (set,
// not accumulated).  Also s_advp (advp.f90:249-620, diaopt=0) with the
// J-weighted fluxes passed as rxu/rxv/rxw.
template <class R>
void advs(const Opts& o, const F3<R>& rxu, const F3<R>& rxv, const F3<R>& rxw, const F3<R>& s,
          F3<R>& sfrc, F3<R>& t1, F3<R>& t2, F3<R>& t3) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dxiv = R(1) / R(o.dx), dyiv = R(1) / R(o.dy), dziv = R(1) / R(o.dz);
  const R oned24 = R(1) / R(24), fourd3 = R(4) / R(3);
  const R dxv05n = R(-.5) * dxiv, dyv05n = R(-.5) * dyiv, dzv05n = R(-.5) * dziv;
  const R dxv24 = oned24 * dxiv, dyv24 = oned24 * dyiv;
  const int iw = o.iw(), ie = o.ie();   // open x: 4th order away from the boundary columns
  OMP_FOR for (int k = 2; k <= nk - 2; ++k) {
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i) t1(i, j, k) = rxu(i, j, k) * (s(i, j, k) - s(i - 1, j, k)) * dxv05n;
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i) t2(i, j, k) = rxv(i, j, k) * (s(i, j, k) - s(i, j - 1, k)) * dyv05n;
  }
  OMP_FOR for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) t3(i, j, k) = rxw(i, j, k) * (s(i, j, k) - s(i, j, k - 1)) * dzv05n;
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        sfrc(i, j, k) = (t1(i, j, k) + t1(i + 1, j, k)) + (t2(i, j, k) + t2(i, j + 1, k));
  // keep the vertical part before t3 is reused below
  F3<R>& vt = t3;
  OMP_FOR for (int k = 2; k <= nk - 2; ++k) {
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 1 + iw; i <= ni - 1 - ie; ++i)
        t1(i, j, k) = (rxu(i, j, k) + rxu(i + 1, j, k)) * (s(i + 1, j, k) - s(i - 1, j, k)) * dxv24;
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 2 + iw; i <= ni - 2 - ie; ++i)
        t2(i, j, k) = (rxv(i, j, k) + rxv(i, j + 1, k)) * (s(i, j + 1, k) - s(i, j - 1, k)) * dyv24;
  }
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2 + iw; i <= ni - 2 - ie; ++i)
        sfrc(i, j, k) = fourd3 * sfrc(i, j, k) +
                        ((t1(i - 1, j, k) + t1(i + 1, j, k)) + (t2(i, j - 1, k) + t2(i, j + 1, k)));
  if (o.advopt == 3) {   // advs.f90:284-300, 372-416 (advp.f90:627-655 alike)
    const R dzv24 = oned24 * dziv;
    F3<R> va(ni, nj, nk), tz(ni, nj, nk);
    for (int k = 2; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 2; ++i) {
          va(i, j, k) = vt(i, j, k) + vt(i, j, k + 1);
          tz(i, j, k) = (rxw(i, j, k) + rxw(i, j, k + 1)) * (s(i, j, k + 1) - s(i, j, k - 1)) * dzv24;
        }
    for (int k = 3; k <= nk - 3; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 2; ++i) va(i, j, k) = fourd3 * va(i, j, k) + (tz(i, j, k - 1) + tz(i, j, k + 1));
    for (int k = 2; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 2; ++i) sfrc(i, j, k) = sfrc(i, j, k) + va(i, j, k);
  } else {
    OMP_FOR for (int k = 2; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 2; ++i) sfrc(i, j, k) = sfrc(i, j, k) + (vt(i, j, k) + vt(i, j, k + 1));
  }
}

// 4th-order numerical smoothing of one field, the operator shared by
// s_smoo4s (smoo4s.f90:184-296, applied to rbr*s), s_smoo4p (smoo4p.f90:
// 178-283, applied to p'), s_smoo4uvw (smoo4uvw.f90:220-568, applied to
// rst8*(u-ubr)/jcb8 etc.).  `a` is the smoothed quantity (tmp4 in the
// reference) already formed over its range; (ilo..ihi, jlo..jhi, klo..khi)
// is the output range of frc; `kw` marks the w-point variant (vertical
// ghost extension at nk instead of nk-1).
template <class R>
void smooth4(const Opts& o, int smtopt, double smhcoe_d, double smvcoe_d, const F3<R>& a, int ilo,
             int ihi, int jlo, int jhi, int klo, int khi, bool wpoint, F3<R>& frc, F3<R>& t1, F3<R>& t2,
             F3<R>& t3) {
  const R smhcoe = R(smhcoe_d), smvcoe = R(smvcoe_d);
  // open x: the 4th-order increments skip the boundary columns
  // (smoo4uvw.f90:286-330 etc., i = 2+iwest .. ni-1-ieast)
  const int i4lo = ilo + o.iw(), i4hi = ihi - o.ie();
  OMP_FOR for (int k = klo; k <= khi; ++k) {
    for (int j = jlo; j <= jhi; ++j)
      for (int i = ilo - 1 + o.iw(); i <= ihi + 1 - o.ie(); ++i)
        t1(i, j, k) = (a(i + 1, j, k) + a(i - 1, j, k)) - R(2) * a(i, j, k);
    for (int j = jlo - 1; j <= jhi + 1; ++j)
      for (int i = ilo; i <= ihi; ++i)
        t2(i, j, k) = (a(i, j + 1, k) + a(i, j - 1, k)) - R(2) * a(i, j, k);
    for (int j = jlo; j <= jhi; ++j)
      for (int i = ilo; i <= ihi; ++i)
        t3(i, j, k) = (a(i, j, k + 1) + a(i, j, k - 1)) - R(2) * a(i, j, k);
  }
  OMP_FOR for (int k = klo; k <= khi; ++k)
    for (int j = jlo; j <= jhi; ++j)
      for (int i = ilo; i <= ihi; ++i)
        frc(i, j, k) = frc(i, j, k) + smhcoe * (t1(i, j, k) + t2(i, j, k)) + smvcoe * t3(i, j, k);
  if (smtopt % 10 == 2) {
    OMP_FOR for (int k = klo; k <= khi; ++k)
      for (int j = jlo; j <= jhi; ++j)
        for (int i = i4lo; i <= i4hi; ++i)
          frc(i, j, k) = frc(i, j, k) + smhcoe * ((t1(i, j, k) - (t1(i + 1, j, k) + t1(i - 1, j, k))) +
                                                  (t2(i, j, k) - (t2(i, j + 1, k) + t2(i, j - 1, k))));
  } else {
    for (int j = jlo; j <= jhi; ++j)
      for (int i = i4lo; i <= i4hi; ++i) {
        t3(i, j, klo - 1) = t3(i, j, klo);
        t3(i, j, khi + 1) = t3(i, j, khi);
      }
    (void)wpoint;
    OMP_FOR for (int k = klo; k <= khi; ++k)
      for (int j = jlo; j <= jhi; ++j)
        for (int i = i4lo; i <= i4hi; ++i)
          frc(i, j, k) = frc(i, j, k) + (smvcoe * (t3(i, j, k) - (t3(i, j, k + 1) + t3(i, j, k - 1))) +
                                         smhcoe * ((t1(i, j, k) - (t1(i + 1, j, k) + t1(i - 1, j, k))) +
                                                   (t2(i, j, k) - (t2(i, j + 1, k) + t2(i, j - 1, k)))));
  }
}

}  // namespace oracle

namespace oracle {

// Rayleigh damping coefficient rbct(k,2) of s_vspdmp (vspdmp.f90:222-292)
// for vspopt=2, from the w-level heights zph (flat terrain: zph = zsth).
// Returns ksp0(2).
template <class R>
int vspdmp(const Opts& o, const std::vector<double>& zph, double vspbar, double botbar,
           std::vector<R>& rbct) {
  const int nk = o.nk;
  const R cc = R(3.141592);                 // commath.f90:42
  const R cbar05 = R(.5) * R(vspbar);       // vspdmp.f90:161
  rbct.assign(nk + 2, R(0));
  int ksp0 = 2;
  for (int k = 3; k <= nk; ++k)
    if (R(zph[k]) > R(botbar)) { ksp0 = k - 1; break; }
  for (int k = 2; k <= nk - 1; ++k) {
    const R z = R(zph[k]);
    if (z > R(botbar))
      rbct[k] = cbar05 * (R(1) - std::cos(cc * (z - R(botbar)) / (R(zph[nk - 1]) - R(botbar))));
    else
      rbct[k] = R(0);
  }
  return ksp0;
}

// s_vspuvw vspopt=2 (vspuvw.f90:230-408), s_vspp (vspp.f90:178-195),
// s_vsps (vsps.f90:181-198).  rbct is the 1-D coefficient above.
template <class R>
void vspuvw(const Opts& o, const LargeOpts& lo, const Base<R>& b, const std::vector<R>& rbct,
            const F3<R>& up, const F3<R>& vp, const F3<R>& wp, F3<R>& ufrc, F3<R>& vfrc, F3<R>& wfrc,
            F3<R>& r8s) {
  const int ni = o.ni, nj = o.nj, nk = o.nk, k0 = lo.ksp0;
  for (int k = k0 - 1; k <= nk - 2; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 1; i <= ni - 1; ++i) r8s(i, j, k) = R(.25) * (rbct[k] + rbct[k + 1]);
  if (lo.vspvar[0] == 'o')
    for (int k = k0 - 1; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 1; ++i)
          ufrc(i, j, k) = ufrc(i, j, k) - b.rst8u(i, j, k) * (r8s(i - 1, j, k) + r8s(i, j, k)) *
                                              (up(i, j, k) - b.ubr(i, j, k));
  if (lo.vspvar[1] == 'o')
    for (int k = k0 - 1; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 1; ++j)
        for (int i = 2; i <= ni - 2; ++i)
          vfrc(i, j, k) = vfrc(i, j, k) - b.rst8v(i, j, k) * (r8s(i, j - 1, k) + r8s(i, j, k)) *
                                              (vp(i, j, k) - b.vbr(i, j, k));
  if (lo.vspvar[2] == 'o')
    for (int k = k0; k <= nk - 1; ++k)
      for (int j = 2; j <= nj - 2; ++j)
        for (int i = 2; i <= ni - 2; ++i)
          wfrc(i, j, k) = wfrc(i, j, k) - rbct[k] * b.rst8w(i, j, k) * wp(i, j, k);
}

// s_vsps / s_vspp form: sfrc -= .5*(rbct(k)+rbct(k+1)) * wt * sp.
template <class R>
void vsp_scalar(const Opts& o, int ksp0, const std::vector<R>& rbct, const F3<R>& wt,
                const F3<R>& sp, F3<R>& sfrc) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  for (int k = ksp0 - 1; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        sfrc(i, j, k) = sfrc(i, j, k) - R(.5) * (rbct[k] + rbct[k + 1]) * wt(i, j, k) * sp(i, j, k);
}

// s_coriuv, SrcOrig/coriuv.f90:124-182 (fc = 0.5*omega*sin(lat), trilat.f90:118-134).
template <class R>
void coriuv(const Opts& o, R fc, const Base<R>& b, const F3<R>& u, const F3<R>& v, F3<R>& ufrc,
            F3<R>& vfrc, F3<R>& t1) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 1; i <= ni - 1; ++i) t1(i, j, k) = fc * b.rst(i, j, k) * (v(i, j, k) + v(i, j + 1, k));
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 1; ++i) ufrc(i, j, k) = ufrc(i, j, k) + (t1(i - 1, j, k) + t1(i, j, k));
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i) t1(i, j, k) = -fc * b.rst(i, j, k) * (u(i, j, k) + u(i + 1, j, k));
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 1; ++j)
      for (int i = 2; i <= ni - 2; ++i) vfrc(i, j, k) = vfrc(i, j, k) + (t1(i, j - 1, k) + t1(i, j, k));
}

// s_buoywb, SrcOrig/buoywb.f90:152-319 (gwmopt=0): dry, or moist with
// qall = total hydrometeor mixing ratio (cphopt != 0).
template <class R>
void buoywb(const Opts& o, bool moist, const Base<R>& b, const F3<R>& ptp, const F3<R>* qv,
            const F3<R>* qall, F3<R>& wfrc, F3<R>& wb8s) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R g05 = R(.5) * R(Phys::g), epsva = R(Phys::epsva);
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) {
        if (!moist) {
          wb8s(i, j, k) = g05 * b.rst(i, j, k) * ptp(i, j, k) / b.ptbr(i, j, k);
        } else {
          const R qvd = (*qv)(i, j, k) - b.qvbr(i, j, k);
          if (qall)
            wb8s(i, j, k) = g05 * b.rst(i, j, k) *
                            (qvd / (epsva + b.qvbr(i, j, k)) - (qvd + (*qall)(i, j, k)) / (R(1) + b.qvbr(i, j, k)) +
                             ptp(i, j, k) / b.ptbr(i, j, k));
          else
            wb8s(i, j, k) = g05 * b.rst(i, j, k) *
                            (qvd / (epsva + b.qvbr(i, j, k)) - qvd / (R(1) + b.qvbr(i, j, k)) +
                             ptp(i, j, k) / b.ptbr(i, j, k));
        }
      }
  OMP_FOR for (int k = 3; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) wfrc(i, j, k) = wfrc(i, j, k) + (wb8s(i, j, k - 1) + wb8s(i, j, k));
}

// s_advbspt gwmopt=0, SrcOrig/advbspt.f90:135-172: base-state theta advection.
template <class R>
void advbspt(const Opts& o, const Base<R>& b, const F3<R>& w, F3<R>& ptadv, F3<R>& pta8w) {
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dziv25 = R(.25) * (R(1) / R(o.dz));
  OMP_FOR for (int k = 2; k <= nk - 1; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i)
        pta8w(i, j, k) = (b.rbr(i, j, k - 1) + b.rbr(i, j, k)) * w(i, j, k) *
                         (b.ptbr(i, j, k - 1) - b.ptbr(i, j, k)) * dziv25;
  OMP_FOR for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      for (int i = 2; i <= ni - 2; ++i) ptadv(i, j, k) = ptadv(i, j, k) + (pta8w(i, j, k) + pta8w(i, j, k + 1));
}

}  // namespace oracle

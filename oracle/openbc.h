// Oracle: open (radiation) west and east boundaries, wbc = ebc in {4, 5, 7}
// with periodic y, advopt <= 3, no lateral damping (lbcvar all 'x', so
// the lbnews / lbnorm terms are multiplied by zero), no GPV nudging
// (nggopt = 0, lspopt = 0, exbopt = 0) and vspopt != 1.
//
// TEST INFRASTRUCTURE ONLY (see arr.h).
//
//   phase speeds  s_phasev -> s_phvuvw / s_phvs (phasev.f90:464-800,
//                 phvuvw.f90:300-1760, phvs.f90:200-560), called after the
//                 Asselin filter with the filtered present level, the past
//                 and the future level (intgdrv.f90:1023-1056)
//   small step    s_rbcu / s_rbcv (stepuv.f90:266-280, rbcu.f90:228-300,
//                 rbcv.f90:324-400), s_rbcw (stepwi.f90:296, rbcw.f90:401-483),
//                 s_rbcss (steppi.f90:199, rbcss.f90:392-472), applied to the
//                 substep's working arrays before their interior update
//   large step    s_rbcpt (steps.f90:1036, rbcpt.f90:626-760), s_rbcqv
//                 (steps.f90:1055, rbcqv.f90:627-800), s_rbcq for the mixing
//                 ratios and s_rbcs for the number concentrations
//                 (steps.f90:1077-1260, rbcq.f90:625-790, rbcs.f90:385-470),
//                 the leapfrog form (advopt <= 3)
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>
#include "arr.h"
#include "phys.h"

namespace oracle {

// Variables with phase speeds, in the C-ABI's field order.
enum RadVar { RV_U = 0, RV_V, RV_W, RV_P, RV_PT, RV_QV, RV_N = RV_QV + 9 };

// ucpx(1:nj,1:nk,1:2) and its siblings: side 0 west, 1 east.
template <class R>
struct Radiation {
  int nj = 0, nk = 0;
  std::vector<R> c;
  void resize(int nj_, int nk_) {
    nj = nj_; nk = nk_;
    c.assign((size_t)RV_N * 2 * (nk + 1) * (nj + 2), R(0));
  }
  R& operator()(int var, int side, int j, int k) {
    return c[(((size_t)var * 2 + side) * (nk + 1) + k) * (nj + 2) + j];
  }
  R operator()(int var, int side, int j, int k) const {
    return c[(((size_t)var * 2 + side) * (nk + 1) + k) * (nj + 2) + j];
  }
};

template <class R>
const Radiation<R>& rad_of(const Opts& o) { return *static_cast<const Radiation<R>*>(o.rad); }

// s_rbcu (rbcu.f90:228-300): u(1) and u(ni), j = 1..nj-1, k = 2..nk-2.
template <class R, class B>
void rbcu(const Opts& o, const B& b, F3<R>& u) {
  if (!o.obc) return;
  const Radiation<R>& cp = rad_of<R>(o);
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R ndmpdt = R(0);
  for (int k = 2; k <= nk - 2; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      u(1, j, k) = u(1, j, k) - cp(RV_U, 0, j, k) * (u(2, j, k) - u(1, j, k)) - ndmpdt * (u(1, j, k) - b.ubr(1, j, k));
  for (int k = 2; k <= nk - 2; ++k)
    for (int j = 1; j <= nj - 1; ++j)
      u(ni, j, k) = u(ni, j, k) + cp(RV_U, 1, j, k) * (u(ni - 1, j, k) - u(ni, j, k)) -
                    ndmpdt * (u(ni, j, k) - b.ubr(ni, j, k));
}

// s_rbcv (rbcv.f90:324-400): v(1) and v(ni-1), j = 2..nj-1, k = 2..nk-2.
template <class R, class B>
void rbcv(const Opts& o, const B& b, F3<R>& v) {
  if (!o.obc) return;
  const Radiation<R>& cp = rad_of<R>(o);
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R tdmpdt = R(0);
  for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 1; ++j)
      v(1, j, k) = v(1, j, k) - cp(RV_V, 0, j, k) * (v(2, j, k) - v(1, j, k)) - tdmpdt * (v(1, j, k) - b.vbr(1, j, k));
  for (int k = 2; k <= nk - 2; ++k)
    for (int j = 2; j <= nj - 1; ++j)
      v(ni - 1, j, k) = v(ni - 1, j, k) + cp(RV_V, 1, j, k) * (v(ni - 2, j, k) - v(ni - 1, j, k)) -
                        tdmpdt * (v(ni - 1, j, k) - b.vbr(ni - 1, j, k));
}

// s_rbcw (rbcw.f90:401-483) and s_rbcss (rbcss.f90:392-472): s(1) and
// s(ni-1), j = 2..nj-2, k = 2..kend (nk-1 for w, nk-2 for p').
template <class R>
void rbc_point(const Opts& o, int var, int kend, F3<R>& s) {
  if (!o.obc) return;
  const Radiation<R>& cp = rad_of<R>(o);
  const int ni = o.ni, nj = o.nj;
  const R dmpdt = R(0);
  for (int k = 2; k <= kend; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      s(1, j, k) = s(1, j, k) - cp(var, 0, j, k) * (s(2, j, k) - s(1, j, k)) - dmpdt * s(1, j, k);
  for (int k = 2; k <= kend; ++k)
    for (int j = 2; j <= nj - 2; ++j)
      s(ni - 1, j, k) = s(ni - 1, j, k) + cp(var, 1, j, k) * (s(ni - 2, j, k) - s(ni - 1, j, k)) -
                        dmpdt * s(ni - 1, j, k);
}

// Leapfrog radiation of a large-step scalar at i = 1 and ni-1 (j = 2..nj-2,
// k = 2..nk-2): sf = sp - gamma*(s(2) - sp) with gamma = 2c/(1-c) west and
// sf = sp + gamma*(s(ni-2) - sp) with gamma = 2c/(1+c) east.  kind 0:
// theta' (rbcpt), 1: qv, clipped at
// zero, damped toward qvbr (rbcqv), 2: mixing ratios, clipped (rbcq), 3:
// number concentrations (rbcs, the damping term last).
template <class R, class B>
void rbc_leapfrog(const Opts& o, const B& b, int var, int kind, const F3<R>& s, const F3<R>& sp, F3<R>& sf) {
  if (!o.obc) return;
  const Radiation<R>& cp = rad_of<R>(o);
  const int ni = o.ni, nj = o.nj, nk = o.nk;
  const R dmpdt = R(0);
  for (int side = 0; side < 2; ++side) {
    const int ib = side == 0 ? 1 : ni - 1, in = side == 0 ? 2 : ni - 2;
    for (int k = 2; k <= nk - 2; ++k)
      for (int j = 2; j <= nj - 2; ++j) {
        const R c = cp(var, side, j, k);
        const R gamma = side == 0 ? R(2) * c / (R(1) - c) : R(2) * c / (R(1) + c);
        const R p = sp(ib, j, k), d = s(in, j, k) - p;
        R v;
        if (kind == 1)
          v = side == 0 ? std::max(p - gamma * d - dmpdt * (p - b.qvbr(ib, j, k)), R(0))
                        : std::max(p + gamma * d - dmpdt * (p - b.qvbr(ib, j, k)), R(0));
        else if (kind == 2)
          v = side == 0 ? std::max(p - gamma * d - dmpdt * p, R(0)) : std::max(p + gamma * d - dmpdt * p, R(0));
        else if (kind == 3)
          v = side == 0 ? p - gamma * d - dmpdt * p : p + gamma * d - dmpdt * p;
        else
          v = side == 0 ? p - dmpdt * p - gamma * d : p - dmpdt * p + gamma * d;
        sf(ib, j, k) = v;
      }
  }
}

// Phase speed of one variable on both x boundaries (s_phvuvw / s_phvs):
// west c = min((sf(2)-sp(2)) / (sf(2)+sp(2)-2 s(3)), -gwave dtb/dx) for
// options 4 and 5 (5 then averages it over the column), -gwave dtb/dx for
// 7, clipped at -1; east mirrored with the points iw1 = ni-1 (u) or ni-2
// (v, w, scalars) and iw2 = iw1-1, clipped at +1.  Small-step variables
// are scaled by dts/dtb.  j = 1..jend, k = 2..kend; the column average
// divides by kend-1 levels.
template <class R>
void phase_var(const Opts& o, int var, bool sml, int ie1, int jend, int kend, R dtb, R dts, const F3<R>& s,
               const F3<R>& sp, const F3<R>& sf, Radiation<R>& cp) {
  const R eps = R(1.e-20);                 // commath.f90:177
  const R dxiv = R(1) / R(o.dx);
  const R gdxdt = R(o.gwave) * dtb * dxiv, gdxdtn = -(R(o.gwave) * dtb * dxiv);
  const R dtsdb = dts / dtb;
  const R nkv = R(1) / R(kend - 1);        // nkm3v (kend = nk-2) or nkm2v (kend = nk-1)
  for (int side = 0; side < 2; ++side) {
    const int i1 = side == 0 ? 2 : ie1, i2 = side == 0 ? 3 : ie1 - 1;
    for (int k = 2; k <= kend; ++k)
      for (int j = 1; j <= jend; ++j) {
        R c;
        if (o.obc == 4 || o.obc == 5) {
          R den = side == 0 ? sf(i1, j, k) + sp(i1, j, k) - R(2) * s(i2, j, k)
                            : R(2) * s(i2, j, k) - sf(i1, j, k) - sp(i1, j, k);
          if (std::fabs(den) < eps) den = std::copysign(eps, den);
          c = (sf(i1, j, k) - sp(i1, j, k)) / den;
          c = side == 0 ? std::min(c, gdxdtn) : std::max(c, gdxdt);
        } else {
          c = side == 0 ? gdxdtn : gdxdt;
        }
        cp(var, side, j, k) = c;
      }
    if (o.obc == 5)
      for (int j = 1; j <= jend; ++j) {
        R av = R(0);
        for (int k = 2; k <= kend; ++k) av = av + cp(var, side, j, k) * nkv;
        for (int k = 2; k <= kend; ++k) cp(var, side, j, k) = av;
      }
    for (int k = 2; k <= kend; ++k)
      for (int j = 1; j <= jend; ++j) {
        R c = cp(var, side, j, k);
        c = side == 0 ? std::max(c, R(-1)) : std::min(c, R(1));
        if (sml) c = c * dtsdb;
        cp(var, side, j, k) = c;
      }
  }
}

}  // namespace oracle

// Stencil helpers shared by the large-step kernels (internal): the
// 4th-order numerical smoothing and the turbulent mixing of a scalar,
// written over accessor functors so that every kernel that uses them forms
// the same terms in the same order, whatever memory its neighbours come
// from and whether it computes one point or a pair (F2).
#pragma once
#include "f2.cuh"
#include "hevi.cuh"

namespace cress {

// 4th-order smoothing increments (smoo4s.f90:199-296 and its u/v/w/p
// variants) added to frc at a point of level k: A(dx, dy, dz) returns the
// smoothed quantity at an offset, and may be evaluated at every dz in
// -2..2 (a shared-memory ring that holds those levels, whatever they
// contain at the ends of the column).  The reference clamps the vertical
// second difference at kmin and kmax (tmp3(kmin-1) = tmp3(kmin),
// tmp3(kmax+1) = tmp3(kmax)); here that is a selection, so every offset is
// a compile-time constant.
// T is float, or F2 (f2.cuh) for two points at once.  edge: the points
// (bit 0 first, bit 1 second) in an open-x boundary column, where only the
// 2nd-order part applies (smoo4uvw.f90:286-330 and the other smoo4*: the
// 4th-order loops run over i = 2+iwest .. with iwest = 1).
template <class T, class FA>
__device__ __forceinline__ T smooth_tile(T frc, int smtopt, float smhcoe, float smvcoe, int k, int kmin, int kmax,
                                         const FA& A, int edge = 0) {
  auto t1 = [&](int x) { return (A(x + 1, 0, 0) + A(x - 1, 0, 0)) - 2.f * A(x, 0, 0); };
  auto t2 = [&](int y) { return (A(0, y + 1, 0) + A(0, y - 1, 0)) - 2.f * A(0, y, 0); };
  auto t3 = [&](int z) { return (A(0, 0, z + 1) + A(0, 0, z - 1)) - 2.f * A(0, 0, z); };
  const T t10 = t1(0), t20 = t2(0), t30 = t3(0);
  frc = frc + smhcoe * (t10 + t20) + smvcoe * t30;
  const T frc2 = frc;
  if (smtopt % 10 == 2) {
    frc = frc + smhcoe * ((t10 - (t1(1) + t1(-1))) + (t20 - (t2(1) + t2(-1))));
  } else {
    const T t3p = k >= kmax ? t30 : t3(1);    // tmp3(kmax+1) = tmp3(kmax)
    const T t3m = k <= kmin ? t30 : t3(-1);   // tmp3(kmin-1) = tmp3(kmin)
    frc = frc + (smvcoe * (t30 - (t3p + t3m)) +
                 smhcoe * ((t10 - (t1(1) + t1(-1))) + (t20 - (t2(1) + t2(-1)))));
  }
  return edge ? sel2(edge, frc2, frc) : frc;
}

// Turbulent mixing of a scalar S (the full field at t-dt) at a point of
// level k: s_eddydif / s_kh8uv diffusivities (rkh8u = rkh(i-1)+rkh(i),
// rkv8w = (rkh(k-1)+rkh(k))/2; eddydif.f90:154-260, 319-340,
// kh8uv.f90:211-230) and the flux divergence of s_turbflx / s_turbs
// (turbflx.f90:236-352, turbs.f90:189-232), added to frc.  The scalar
// diffusivity rkh at an offset is formed from the staged field R: the
// Smagorinsky form rkh = cpriv*rkv/jcb from the eddy viscosity (kdiv = 0),
// or, with the TKE closure, R is already 1/Pr*rkv/jcb (kdiv = 1).
template <class T, class FC, class FR, class FS>
__device__ __forceinline__ T turb_scalar_at(T frc, const FC& C, int k, float cpriv, int kdiv, float dxiv,
                                            float dyiv, float dziv, const FR& R, const FS& S) {
  // R(dx, dy, dz): the staged viscosity or diffusivity, S(dx, dy, dz): the
  // scalar, at an offset from the point (only dz = -1, 0, 1 on the point's
  // own column)
  auto RKH = [&](int dx, int dy, int dz) {
    return kdiv ? R(dx, dy, dz) : cpriv * R(dx, dy, dz) * C(C_IJCB, k + dz);
  };
  const float jc = C(C_JCB, k);
  const float dxv05 = .5f * dxiv, dyv05 = .5f * dyiv;
  auto JS = [&](int dx, int dy) { return S(dx, dy, 0) * jc; };
  auto H1 = [&](int dx) { return (RKH(dx - 1, 0, 0) + RKH(dx, 0, 0)) * (JS(dx, 0) - JS(dx - 1, 0)) * dxv05; };
  auto H2 = [&](int dy) { return (RKH(0, dy - 1, 0) + RKH(0, dy, 0)) * (JS(0, dy) - JS(0, dy - 1)) * dyv05; };
  auto H3 = [&](int dz) {
    return (.5f * (RKH(0, 0, dz - 1) + RKH(0, 0, dz))) * (S(0, 0, dz) - S(0, 0, dz - 1)) * dziv;
  };
  const float j8u = C(C_JCB8U, k), j8v = C(C_JCB8V, k);
  return frc + ((H3(1) - H3(0)) * dziv + ((j8u * H1(1) - j8u * H1(0)) * dxiv + (j8v * H2(1) - j8v * H2(0)) * dyiv));
}

}  // namespace cress

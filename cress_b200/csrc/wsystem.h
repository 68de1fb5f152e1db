// Host-side set-up of the HE-VI substep shared by the context API
// (capi.cu) and the allocation-free entry point (hevi_noalloc.cu), so both
// launch the kernel with the same columns and elimination factors.
#pragma once
#include <cmath>
#include <cstddef>
#include "../../include/cress_b200.h"
#include "hevi.cuh"

namespace cress {

// Physical constants used on the host side (SrcOrig/comphy.f90:49, :459).
constexpr float kG = 9.8f;
constexpr float kDivndc = 0.05f;

// Where a base array first varies horizontally (n < 0: it does not).
struct NonUniform {
  int n = -1, i = 0, j = 0, k = 0;
  float x = 0.f, v = 0.f;
};

// 1-D base columns col[field * (nk+1) + k] of the 11 cress_set_base3d
// arrays (reference layout (0:ni+1, 0:nj+1, 1:nk)), taken at the domain
// centre, plus the reciprocals of the per-level divisors the kernels
// multiply by.  Every point the small step reads (i in 1..ni, j in 1..nj)
// must carry the centre's value; the first one that does not is returned.
inline NonUniform base_columns(const float* const* b3, int ni, int nj, int nk, float* col) {
  auto at = [&](const float* a, int i, int j, int k) {
    return a[(size_t)i + (size_t)(ni + 2) * ((size_t)j + (size_t)(nj + 2) * (size_t)(k - 1))];
  };
  const int map[CRESS_B_N] = {C_JCB, C_JCB8U, C_JCB8V, C_JCB8W, C_RBR, C_PTBR,
                              C_RST, C_RST8U, C_RST8V, C_RST8W, C_RCSQ};
  const int ic = ni / 2, jc = nj / 2;
  NonUniform bad;
  for (int n = 0; n < CRESS_B_N; ++n) {
    const float* a = b3[n];
    for (int k = 1; k <= nk; ++k) {
      const float v = at(a, ic, jc, k);
      col[(size_t)map[n] * (nk + 1) + k] = v;
      for (int j = 1; j <= nj; ++j)
        for (int i = 1; i <= ni; ++i) {
          const float x = at(a, i, j, k);
          if (x != v && !(std::isnan(x) && std::isnan(v))) {
            bad.n = n; bad.i = i; bad.j = j; bad.k = k; bad.x = x; bad.v = v;
            return bad;
          }
        }
    }
  }
  const int inv_src[6] = {C_RST8U, C_RST8V, C_JCB, C_RCSQ, C_RST8W, C_JCB8W};
  const int inv_dst[6] = {C_IRST8U, C_IRST8V, C_IJCB, C_IRCSQ, C_IRST8W, C_IJCB8W};
  for (int n = 0; n < 6; ++n)
    for (int k = 1; k <= nk; ++k) {
      const float v = col[(size_t)inv_src[n] * (nk + 1) + k];
      col[(size_t)inv_dst[n] * (nk + 1) + k] = (v != 0.f) ? 1.f / v : 0.f;
    }
  return bad;
}

// Coefficients of the w tridiagonal system of s_stepwi for buyopt = 0/1
// (SrcOrig/stepwi.f90:308-416), formed in float exactly as the reference
// does for a horizontally uniform base state, then the elimination factors
// of s_gaussel impopt=1 (SrcOrig/gaussel.f90:189-240) in double:
// rr[k] = a_k, aa[k] = 1/(b_k - a_k c'_{k-1}), cp[k] = c'_k for k = 3..nk-2;
// every array holds nk+2 entries and is zeroed first.  The factors depend
// on dts only through sbsqzi and sbsqg5.
inline void w_system_factors(const float* col, int nk, float dz, float weicoe, int buyopt, float dts,
                             float* rr, double* aa, double* cp, float* scratch4 /* 4*(nk+2) */) {
  auto C = [&](int f, int k) { return col[(size_t)f * (nk + 1) + k]; };
  float* fwc = scratch4;
  float* wcc = fwc + (nk + 2);
  float* ss = wcc + (nk + 2);
  float* tt = ss + (nk + 2);
  for (int k = 0; k < nk + 2; ++k) {
    fwc[k] = wcc[k] = ss[k] = tt[k] = rr[k] = 0.f;
    aa[k] = cp[k] = 0.0;
  }
  const float dziv = 1.f / dz, g05 = .5f * kG;
  const float sbsqzi = dts * dts * weicoe * weicoe * dziv;
  const float sbsqg5 = .5f * kG * dts * dts * weicoe * weicoe;
  for (int k = 2; k <= nk - 2; ++k) {
    const float t1 = g05 * C(C_RBR, k) / C(C_RCSQ, k);
    const float t2 = dziv / C(C_JCB, k);
    fwc[k] = t1 + t2;
    wcc[k] = t1 - t2;
  }
  for (int k = 3; k <= nk - 2; ++k) {
    if (buyopt == 0) {
      const float a = sbsqzi / C(C_RST8W, k);
      const float mm = a * C(C_RCSQ, k - 1);
      const float nn = a * C(C_RCSQ, k);
      rr[k] = -mm * fwc[k - 1];
      ss[k] = 1.f + (nn * fwc[k] - mm * wcc[k - 1]);
      tt[k] = nn * wcc[k];
    } else {
      const float rstiv = 1.f / C(C_RST8W, k);
      const float a = rstiv * sbsqzi;
      const float b = rstiv * sbsqg5;
      const float mm = b * C(C_RST, k - 1) - a * C(C_RCSQ, k - 1);
      const float nn = b * C(C_RST, k) + a * C(C_RCSQ, k);
      rr[k] = mm * fwc[k - 1];
      ss[k] = 1.f + (mm * wcc[k - 1] + nn * fwc[k]);
      tt[k] = nn * wcc[k];
    }
  }
  const int ks = 3, ke = nk - 2;
  aa[ks] = 1.0 / (double)ss[ks];
  cp[ks] = (double)tt[ks] * aa[ks];
  for (int k = ks + 1; k <= ke - 1; ++k) {
    aa[k] = 1.0 / ((double)ss[k] - (double)rr[k] * cp[k - 1]);
    cp[k] = (double)tt[k] * aa[k];
  }
  aa[ke] = 1.0 / ((double)ss[ke] - (double)rr[ke] * cp[ke - 1]);
}

// Rows k = 0..nk of the level table of the on-chip HE-VI kernel (tile
// 12) from the base columns and the w-system factors above.
inline void hevi_level_rows(const float* col, int nk, const float* rr, const double* aa, const double* cp,
                            HeviLevel* out) {
  auto C = [&](int f, int k) { return col[(size_t)f * (nk + 1) + k]; };
  for (int k = 0; k <= nk; ++k) {
    HeviLevel r{};
    auto set = [](float* d, float v) { d[0] = d[1] = v; };
    if (k >= 1) {
      set(r.rst8u, C(C_RST8U, k)); set(r.rst8v, C(C_RST8V, k)); set(r.rst8w, C(C_RST8W, k));
      set(r.ij8w, C(C_IJCB8W, k)); set(r.jcb, C(C_JCB, k)); set(r.ijcb, C(C_IJCB, k));
      set(r.irst8u, C(C_IRST8U, k)); set(r.irst8v, C(C_IRST8V, k)); set(r.jcb8u, C(C_JCB8U, k));
      set(r.jcb8v, C(C_JCB8V, k)); set(r.rcsq, C(C_RCSQ, k)); set(r.rst, C(C_RST, k)); set(r.rbr, C(C_RBR, k));
      set(r.ircsq, C(C_IRCSQ, k)); set(r.irst8w, C(C_IRST8W, k));
    }
    set(r.rr, rr[k]);
    r.aa = aa[k];
    r.cp = cp[k];
    out[k] = r;
  }
}

inline void hevi_level_rows1(const float* col, int nk, const float* rr, const double* aa, const double* cp,
                             HeviLevel1* out) {
  auto C = [&](int f, int k) { return col[(size_t)f * (nk + 1) + k]; };
  for (int k = 0; k <= nk; ++k) {
    HeviLevel1 r{};
    if (k >= 1) {
      r.rst8u = C(C_RST8U, k); r.rst8v = C(C_RST8V, k); r.rst8w = C(C_RST8W, k); r.ij8w = C(C_IJCB8W, k);
      r.jcb = C(C_JCB, k); r.ijcb = C(C_IJCB, k); r.irst8u = C(C_IRST8U, k); r.irst8v = C(C_IRST8V, k);
      r.jcb8u = C(C_JCB8U, k); r.jcb8v = C(C_JCB8V, k); r.rcsq = C(C_RCSQ, k); r.rst = C(C_RST, k);
      r.rbr = C(C_RBR, k); r.ircsq = C(C_IRCSQ, k); r.irst8w = C(C_IRST8W, k);
    }
    r.rr = rr[k];
    r.aa = aa[k];
    r.cp = cp[k];
    out[k] = r;
  }
}

}  // namespace cress

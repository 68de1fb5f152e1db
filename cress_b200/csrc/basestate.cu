// The base state from a height-level sounding, in FP64 on the device:
// the hydrostatic integration of the sounding with its humidity iteration
// (s_set1d, SrcOrig/set1d.f90:278-452, 536-540), the extension below it
// (s_vextlow, vextlow.f90:150-220), the interpolation to the model's scalar
// levels (s_intrpsnd / s_vint13, intrpsnd.f90:190-230, vint13.f90:120-170),
// the base density and Exner function with their boundary levels
// (s_setbase, setbase.f90:153-189; s_bcbase, bcbase.f90:150-210), rho*J
// and its w-point average (s_baserho, baserho.f90:150-160; var8uvw.f90:
// 190-196; bc8w.f90:136,166) and rho c^2 (s_sndwave, sndwave.f90:119).
//
// The grid is horizontally uniform (flat terrain), so the base state is one
// column: the sounding is integrated by one thread (a serial recurrence
// over levels, iterated to convergence), then the column's levels are
// formed by one thread each.
#include <cuda_runtime.h>
#include <cmath>
#include <vector>
#include "../../include/cress_b200.h"
#include "ctx.h"

namespace cress {
namespace {

// SrcOrig/comphy.f90 and commath.f90
constexpr double kGd = 9.8, kCp = 1004., kCv = 717., kRd = 287., kP0 = 1.e5, kEs0 = 610.78;
constexpr double kEpsva = .622, kEpsav = 1.6077, kT0 = 273.16, kTlow = 233.16, kEps = 1.e-20;
constexpr int kMaxIter = 1000;

struct SndArgs {
  int nlev;            // sounding levels 1..nlev (level 0 is formed here)
  int tvar, hvar;      // 'p' theta / 't' temperature; 'r' relative humidity (percent) / else mixing ratio
  double psnd0, thresq;
  double* z; double* u; double* v; double* p; double* pt; double* qv; double* t;   // [0..nlev]
  double* work;        // 2 (nlev+1): integrated Exner function (or log p), given humidity
  int* status;         // 0 ok, 1 non-positive pressure, 2 no convergence
};

// One thread: set1d (height levels) and vextlow('oooooo').
__global__ void k_sounding(SndArgs s) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int n = s.nlev;
  const double gdvcp2 = 2. * kGd / kCp, gdvrd2 = 2. * kGd / kRd, rddvcp = kRd / kCp, cpdvrd = kCp / kRd;
  const double p0iv = 1. / kP0, es001 = .01 * kEs0;
  double* x = s.work;            // Exner function ('p') or log p ('t') per level
  double* h = s.work + n + 1;    // the given humidity
  const bool tgiven = s.tvar == 't', rh = s.hvar == 'r';
  if (tgiven) {
    x[1] = log(s.psnd0);
    for (int k = 1; k <= n; ++k) s.t[k] = s.pt[k];
  } else {
    x[1] = exp(rddvcp * log(p0iv * s.psnd0));
  }
  if (rh)
    for (int k = 1; k <= n; ++k) { h[k] = s.qv[k]; s.qv[k] = 0.; }
  int it = 0;
  for (; it < kMaxIter; ++it) {
    double xmin = 1.e36, change = 0.;
    // the virtual temperature (or potential temperature) of the current
    // humidity, then the trapezoidal hydrostatic integration upward
    double* tv = tgiven ? s.pt : s.t;
    const double* base = tgiven ? s.t : s.pt;
    for (int k = 1; k <= n; ++k) tv[k] = base[k] * (1. + kEpsav * s.qv[k]) / (1. + s.qv[k]);
    const double c = tgiven ? gdvrd2 : gdvcp2;
    for (int k = 2; k <= n; ++k) {
      x[k] = x[k - 1] - c * (s.z[k] - s.z[k - 1]) / (tv[k - 1] + tv[k]);
      xmin = fmin(x[k], xmin);
    }
    if (xmin <= 0.) { *s.status = 1; return; }
    for (int k = 1; k <= n; ++k) {
      if (tgiven) {
        s.p[k] = exp(x[k]);
        s.pt[k] = s.t[k] * exp(rddvcp * log(kP0 / s.p[k]));
      } else {
        s.p[k] = kP0 * exp(cpdvrd * log(x[k]));
        s.t[k] = s.pt[k] * x[k];
      }
    }
    if (rh) {
      for (int k = 1; k <= n; ++k) {
        const double tk = s.t[k];
        // Tetens over water above tlow, over ice below (set1d.f90:419-440)
        const double ea = tk > kTlow ? es001 * h[k] * exp(17.269 * (tk - kT0) / (tk - 35.86))
                                     : es001 * h[k] * exp(21.875 * (tk - kT0) / (tk - 7.66));
        const double q = kEpsva * ea / (s.p[k] - ea);
        change = fmax(fabs((q + kEps) / (s.qv[k] + kEps) - 1.), change);
        s.qv[k] = q;
      }
    }
    if (change < 1.e-5) break;
  }
  if (it == kMaxIter) { *s.status = 2; return; }
  for (int k = 1; k <= n; ++k)
    if (s.qv[k] <= s.thresq) s.qv[k] = 0.;
  // vextlow: level 0 at min(2 z1 - z2, 0), linear in u, v, theta, qv,
  // hydrostatic in p
  s.z[0] = fmin(2. * s.z[1] - s.z[2], 0.);
  const double w1 = s.z[2] - s.z[0], w2 = s.z[1] - s.z[0], dz12 = s.z[2] - s.z[1];
  s.u[0] = (w1 * s.u[1] - w2 * s.u[2]) / dz12;
  s.v[0] = (w1 * s.v[1] - w2 * s.v[2]) / dz12;
  s.pt[0] = (w1 * s.pt[1] - w2 * s.pt[2]) / dz12;
  s.qv[0] = (w1 * s.qv[1] - w2 * s.qv[2]) / dz12;
  const double ptv0 = s.pt[0] * (1. + s.qv[0]) / (1. + kEpsav * s.qv[0]);
  const double ptv1 = s.pt[1] * (1. + s.qv[1]) / (1. + kEpsav * s.qv[1]);
  const double pi0 = exp(rddvcp * log(p0iv * s.p[1])) + gdvcp2 * (s.z[1] - s.z[0]) / (ptv0 + ptv1);
  s.p[0] = kP0 * exp(cpdvrd * log(pi0));
  *s.status = 0;
}

struct ColArgs {
  int nk, nlev;
  const double* zph; const double* jcb;   // [k], k = 1..nk
  const double* z; const double* u; const double* v; const double* p; const double* pt; const double* qv;
  double* out;                             // CRESS_BS_N columns of nk+1 (cress_b200.h order)
};

// vint13 at height zz: linear between the sounding levels that bracket it,
// extrapolated from the end intervals outside them.
__device__ double interp(const ColArgs& c, const double* var, double zz) {
  const int n = c.nlev;
  double r = 0.;
  if (c.z[0] > zz) {
    const double d = (1. / (c.z[1] - c.z[0])) * (zz - c.z[0]);
    r = (1. - d) * var[0] + d * var[1];
  } else if (c.z[n] <= zz) {
    const double d = (1. / (c.z[n] - c.z[n - 1])) * (zz - c.z[n - 1]);
    r = (1. - d) * var[n - 1] + d * var[n];
  }
  // the bracketing interval by bisection (the levels increase)
  if (c.z[0] <= zz && zz < c.z[n]) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (c.z[mid] <= zz) lo = mid; else hi = mid;
    }
    const double d = (zz - c.z[lo]) / (c.z[lo + 1] - c.z[lo]);
    r = (1. - d) * var[lo] + d * var[lo + 1];
  }
  return r;
}

// Level k of the column (k = 2..nk-2): the interpolated sounding, virtual
// potential temperature, Exner function and density.
__global__ void k_base_levels(ColArgs c) {
  const int k = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int nk = c.nk, m = nk + 1;
  if (k > nk - 2) return;
  const double zz = .5 * (c.zph[k + 1] + c.zph[k]);
  double* o = c.out;
  const double pb = interp(c, c.p, zz), th = interp(c, c.pt, zz), q = interp(c, c.qv, zz);
  const double ptv = th * (1. + kEpsav * q) / (1. + q);
  const double pi = exp((kRd / kCp) * log((1. / kP0) * pb));
  o[CRESS_BS_UBR * m + k] = interp(c, c.u, zz);
  o[CRESS_BS_VBR * m + k] = interp(c, c.v, zz);
  o[CRESS_BS_PBR * m + k] = pb;
  o[CRESS_BS_PTBR * m + k] = th;
  o[CRESS_BS_QVBR * m + k] = q;
  o[CRESS_BS_PTVBR * m + k] = ptv;
  o[CRESS_BS_PIBR * m + k] = pi;
  o[CRESS_BS_RBR * m + k] = pb / (kRd * ptv * pi);
}

// One thread: the boundary levels 1 and nk-1 (bcbase), rho*J, its w-point
// average with bc8w, rho c^2, and level nk repeating level nk-1.
__global__ void k_base_bounds(ColArgs c) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int nk = c.nk, m = nk + 1, k1 = nk - 1, k2 = nk - 2;
  double* o = c.out;
  auto F = [&](int f, int k) -> double& { return o[f * m + k]; };
  const double gdvcp2 = 2. * kGd / kCp, cpdvrd = kCp / kRd;
  const double z1 = .5 * (c.zph[2] + c.zph[1]), z2 = .5 * (c.zph[3] + c.zph[2]);
  const double zk1 = .5 * (c.zph[nk] + c.zph[k1]), zk2 = .5 * (c.zph[k1] + c.zph[k2]);
  for (int f : {CRESS_BS_UBR, CRESS_BS_VBR, CRESS_BS_PTBR, CRESS_BS_QVBR, CRESS_BS_PTVBR}) {
    F(f, 1) = F(f, 2);
    F(f, k1) = F(f, k2);
  }
  F(CRESS_BS_PIBR, 1) = F(CRESS_BS_PIBR, 2) + gdvcp2 * (z2 - z1) / (F(CRESS_BS_PTVBR, 1) + F(CRESS_BS_PTVBR, 2));
  F(CRESS_BS_PIBR, k1) =
      F(CRESS_BS_PIBR, k2) - gdvcp2 * (zk1 - zk2) / (F(CRESS_BS_PTVBR, k2) + F(CRESS_BS_PTVBR, k1));
  for (int k : {1, k1}) {
    F(CRESS_BS_PBR, k) = kP0 * exp(cpdvrd * log(F(CRESS_BS_PIBR, k)));
    F(CRESS_BS_RBR, k) = F(CRESS_BS_PBR, k) / (kRd * F(CRESS_BS_PTVBR, k) * F(CRESS_BS_PIBR, k));
  }
  for (int k = 1; k <= k1; ++k) {
    F(CRESS_BS_RST, k) = fabs(c.jcb[k]) * F(CRESS_BS_RBR, k);
    F(CRESS_BS_RCSQ, k) = (kCp / kCv) * F(CRESS_BS_PBR, k);
  }
  for (int k = 2; k <= k1; ++k) F(CRESS_BS_RST8W, k) = .5 * (F(CRESS_BS_RST, k - 1) + F(CRESS_BS_RST, k));
  F(CRESS_BS_RST8W, 1) = F(CRESS_BS_RST8W, 3);
  F(CRESS_BS_RST8W, nk) = F(CRESS_BS_RST8W, nk - 2);
  for (int f = 0; f < CRESS_BS_N; ++f)
    if (f != CRESS_BS_RST8W) F(f, nk) = F(f, k1);
}

}  // namespace
}  // namespace cress

using namespace cress;

extern "C" int cress_base_state(int nk, const double* zph, const double* jcb, int nlev, const double* sounding,
                                int tvar, int hvar, double psnd0, double thresq, double* columns, int device) {
  if (!zph || !jcb || !sounding || !columns) return set_error(CRESS_E_ARG, "cress_base_state: null argument");
  if (nk < 6 || nlev < 3) return set_error(CRESS_E_ARG, "cress_base_state: nk=%d nlev=%d", nk, nlev);
  if (!(tvar == 'p' || tvar == 't'))
    return set_error(CRESS_E_UNSUPPORTED, "cress_base_state: tvar must be 'p' (theta) or 't' (temperature)");
  for (int kl = 1; kl < nlev; ++kl)
    if (!(sounding[kl] > sounding[kl - 1]))
      return set_error(CRESS_E_ARG, "cress_base_state: sounding heights must increase (level %d)", kl + 1);
  for (int k = 2; k <= nk; ++k)
    if (!(zph[k] > zph[k - 1]))
      return set_error(CRESS_E_ARG, "cress_base_state: zph must increase (k=%d)", k);
  int rc = cuda_check(cudaSetDevice(device), "cudaSetDevice");
  if (rc) return rc;
  const size_t ns = (size_t)nlev + 1, nc = (size_t)nk + 1;
  // device memory: 7 sounding columns, the integration work, the grid, the
  // output columns and the status word, in one allocation
  const size_t nd = 7 * ns + 2 * ns + 2 * nc + CRESS_BS_N * nc + 1;
  double* d = nullptr;
  if ((rc = cuda_check(cudaMalloc(&d, nd * sizeof(double)), "cudaMalloc base state"))) return rc;
  std::vector<double> h(nd, 0.);
  for (int q = 0; q < 5; ++q)      // z, u, v, pt, qv at levels 1..nlev
    for (int kl = 1; kl <= nlev; ++kl) {
      const int slot = q < 3 ? q : q + 1;   // slot 3 is p
      h[slot * ns + kl] = sounding[(size_t)q * nlev + kl - 1];
    }
  double* dz_ = d + 0 * ns; double* du = d + 1 * ns; double* dv = d + 2 * ns; double* dp = d + 3 * ns;
  double* dpt = d + 4 * ns; double* dqv = d + 5 * ns; double* dt = d + 6 * ns; double* dw = d + 7 * ns;
  double* dzph = d + 9 * ns; double* djcb = dzph + nc; double* dout = djcb + nc;
  int* dstat = reinterpret_cast<int*>(dout + CRESS_BS_N * nc);
  for (int k = 0; k <= nk; ++k) { h[9 * ns + k] = zph[k]; h[9 * ns + nc + k] = jcb[k]; }
  cudaStream_t st = nullptr;
  int status = -1;
  if (!(rc = cuda_check(cudaMemcpyAsync(d, h.data(), nd * sizeof(double), cudaMemcpyHostToDevice, st),
                        "copy sounding"))) {
    SndArgs s{nlev, tvar, hvar, psnd0, thresq, dz_, du, dv, dp, dpt, dqv, dt, dw, dstat};
    k_sounding<<<1, 32, 0, st>>>(s);
    ColArgs c{nk, nlev, dzph, djcb, dz_, du, dv, dp, dpt, dqv, dout};
    k_base_levels<<<(nk + 127) / 128, 128, 0, st>>>(c);
    k_base_bounds<<<1, 32, 0, st>>>(c);
    if (!(rc = cuda_check(cudaGetLastError(), "base state launch")) &&
        !(rc = cuda_check(cudaMemcpyAsync(columns, dout, CRESS_BS_N * nc * sizeof(double), cudaMemcpyDeviceToHost, st),
                          "copy base state")) &&
        !(rc = cuda_check(cudaMemcpyAsync(&status, dstat, sizeof(int), cudaMemcpyDeviceToHost, st), "copy status")))
      rc = cuda_check(cudaStreamSynchronize(st), "base state sync");
  }
  cudaFree(d);
  if (rc) return rc;
  if (status == 1) return set_error(CRESS_E_ARG, "cress_base_state: the hydrostatic integration reached p <= 0");
  if (status == 2) return set_error(CRESS_E_ARG, "cress_base_state: the humidity iteration did not converge");
  return CRESS_OK;
}

// Large-step kernels (forcing, leapfrog scalar step, Asselin filter,
// periodic halo planes): internal interface.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"
#include "hevi.cuh"

namespace cress {

// 1-D columns beyond the HE-VI ones, appended after C_NFIELDS in the
// same table: the Rayleigh coefficient rbct(k) (vspdmp.f90:269-292).
enum ColFieldLarge { C_RBCT = C_NFIELDS, C_NFIELDS_ALL };

// Per-level values the large-step kernels read from a k-major table (the
// level table, table[k * kLevelStride + field], built on the host once per
// large-step length and kept on the device): the 1-D columns, quotients of
// constants by columns (the same IEEE divisions the stencils would repeat
// per point) and reciprocals of the per-level divisors of field values,
// which the stencils multiply by (a field value of exactly zero would
// otherwise send every such division through its slow path).
enum ColDerived {
  D_IJCB8U = C_NFIELDS_ALL, D_IJCB8V, D_IPTBR, D_IEPSQV, D_I1QV, D_DTDRST, D_2JCB, D_4JCB, D_2J8W, D_NFIELDS
};
static_assert(kLevelStride >= D_NFIELDS, "level table stride too small");

// Column field f (base or derived) of level kk; B(f, kk) reads a base column.
#pragma nv_exec_check_disable
template <class FB>
__host__ __device__ __forceinline__ float level_value(int f, int kk, const FB& B, float dtb2) {
  switch (f) {
    case D_IJCB8U: return 1.f / B(C_JCB8U, kk);
    case D_IJCB8V: return 1.f / B(C_JCB8V, kk);
    case D_IPTBR: return 1.f / B(C_PTBR, kk);
    case D_IEPSQV: return 1.f / (.622f + B(C_QVBR, kk));   // epsva = rd/rv, comphy.f90:79
    case D_I1QV: return 1.f / (1.f + B(C_QVBR, kk));
    case D_DTDRST: return dtb2 / B(C_RST, kk);             // steps.f90:528
    case D_2JCB: return 2.f / B(C_JCB, kk);                 // defomten.f90:471-500
    case D_4JCB: {
      const float jc = B(C_JCB, kk);
      return 4.f / ((jc + jc) + (jc + jc));                 // defomten.f90:336-352
    }
    case D_2J8W: {
      const float j8w = B(C_JCB8W, kk);
      return 2.f / (j8w + j8w);                             // defomten.f90:763-833
    }
    default: return B(f, kk);
  }
}

struct ForceArgs {
  Grid g;
  const float* col;           // 1-D columns, C_NFIELDS_ALL x (nk+1)
  const float* lvl;           // level table (nk+1) x kLevelStride for this dtb
  // present level t
  const float* u; const float* v; const float* w; const float* pp; const float* ptp;
  // past level t-dt
  const float* up; const float* vp; const float* wp; const float* ppp; const float* ptpp;
  // outputs
  float* ufrc; float* vfrc; float* wfrc; float* pfrc;
  float* ptpf;                // future theta' (s_steps)
  float dxiv, dyiv, dziv;
  float smhcoe, smvcoe;
  float fc;                   // 0.5*omega*sin(lat) when coropt=1
  float dtb2;                 // 2*dtb
  int smtopt, vspopt, coropt, sthopt, ksp0;
  int advopt;                 // 2, or 3: 4th order in z too (advuvw.f90:309, advs.f90:284)
  int vsp_u, vsp_v, vsp_w, vsp_p, vsp_pt;  // vspvar switches
  // moist buoyancy (buoywb.f90:202-299, cphopt != 0): qv and the five
  // hydrometeor mixing ratios at t; null qv = dry buoyancy
  const float* qv; const float* qc; const float* qr; const float* qi; const float* qs; const float* qg;
  // turbulence (tubopt 1, 2): eddy viscosity at scalar points from
  // k_turb_visc (null: no turbulence) and 1/Pr (capped at 3); rks: the
  // field the theta' mixing stages (rkv, or with the TKE closure the scalar
  // diffusivity 1/Pr*rkv/jcb, kdiv = 1)
  const float* rkv;
  const float* rks;
  float cpriv;
  int kdiv;
  int* err;                   // device error word (a bounded wait gave up)
};

// The forcing runs as two kernels over 32 x kForceTY tiles: the momentum
// kernel (output groups u, v, w in one block) and the scalar kernel
// (groups p' and theta').  Each stages its fields (slots) level by level
// by TMA into a shared-memory ring: boxes kHeviBoxX wide, x from the
// tile's i0-2, rows from j0 + force_slot_r0 on, force_slot_rows of them.
constexpr int kForceTY = 8;
constexpr int kForceSlots = 8;
enum ForceBuf { FB_U, FB_V, FB_W, FB_PP, FB_PTP, FB_UP, FB_VP, FB_WP, FB_PPP, FB_PTPP, FB_RKV, FB_NONE };
// staged fields of kernel sg (0 momentum, 1 scalar), with turbulence: turb
__host__ __device__ constexpr int force_nslots(int sg, bool turb) { return sg == 0 ? (turb ? 7 : 6) : (turb ? 8 : 7); }
// momentum: u, v, w, up, vp, wp | rkv       scalar: pp, ptp, ppp, ptpp, u, v, w | rkv
__host__ __device__ constexpr int force_slot_buf(int sg, int s) {
  return sg == 0 ? (s == 0 ? FB_U : s == 1 ? FB_V : s == 2 ? FB_W : s == 3 ? FB_UP : s == 4 ? FB_VP : s == 5 ? FB_WP : FB_RKV)
                 : (s == 0 ? FB_PP : s == 1 ? FB_PTP : s == 2 ? FB_PPP : s == 3 ? FB_PTPP : s == 4 ? FB_U
                    : s == 5 ? FB_V : s == 6 ? FB_W : FB_RKV);
}
// first box row relative to j0 and the number of rows: the momentum slots
// and the scalars' own variables carry two rows of y halo; the scalars'
// winds and viscosity what their stencils reach
__host__ __device__ constexpr int force_slot_r0(int sg, int s) {
  return (sg == 0 || s < 4) ? -2 : (s == 4 || s == 6) ? 0 : -1;
}
__host__ __device__ constexpr int force_slot_rows(int sg, int s) {
  return kForceTY + ((sg == 0 || s < 4) ? 4 : (s == 4 || s == 6) ? 0 : s == 5 ? 3 : 2);
}
struct ForceMaps {
  CUtensorMap m[2][kForceSlots];
};

int launch_force(const ForceArgs& a, const ForceMaps& maps, cudaStream_t st);

// Eddy viscosity (s_turbdrv up to s_eddyvis: bruntv, defomten, defomssq,
// eddyvis, isoopt=1, flat terrain) from the past level into rkv at the
// scalar points i, j = 1..n-1, k = 1..nk-1: the Smagorinsky form
// (tubopt=1), or the Deardorff form from the past TKE (tkep non-null,
// tubopt=2), which also writes the TKE closure's fields rks, nsq, shr, dsp
// (Ctx::rks_d ...).
struct TurbArgs {
  Grid g;
  const float* col;
  const float* lvl;           // a level table (rows 0..nk, kLevelStride floats; its dtb is not used)
  const float *up, *vp, *wp, *ptpp, *ppp;                  // t-dt
  const float *qvp, *qcp, *qrp, *qip, *qsp, *qgp;          // t-dt moist species (null: dry)
  float* rkv;
  float dxiv, dyiv, dziv, ds3, ckmax, cpriv, thresq;
  const float* tkep;                                       // TKE at t-dt (tubopt=2) or null
  float *rks, *nsq, *shr, *dsp;
  float ds308;                                             // dx*dy*dz/8
};
int launch_turb_visc(const TurbArgs& a, cudaStream_t st);

// Forcing and leapfrog step of the nine moist scalars qv, qc, qr, qi, qs,
// qg, ni, ns, ng (s_forceqv, s_forceq, s_steps).
constexpr int kMoistN = 9;
struct MoistScalarArgs {
  Grid g;
  const float* col;
  const float* lvl;           // level table (nk+1) x kLevelStride for this dtb
  const float* u; const float* v; const float* w;   // present winds (flux rst*u etc.)
  const float* s[kMoistN];    // present level t
  const float* sp[kMoistN];   // past level t-dt
  float* sf[kMoistN];         // future level t+dt (output)
  float dxiv, dyiv, dziv, smhcoe, smvcoe, dtb2;
  int smtopt, vspopt, sthopt, ksp0, advopt;
  int vsp_qv, vsp_q;          // vspvar(6:6), vspvar(7:7)
  const float* rkv;           // staged viscosity (tubopt 1: rkv; 2: the diffusivity rks) or null
  float cpriv;
  int kdiv;                   // 1: the staged field is already 1/Pr*rkv/jcb (TKE closure)
  int* err;                   // device error word (a bounded wait gave up)
};

// The scalar kernel stages 32 x kScalarTY tiles of every input level by
// TMA (boxes kHeviBoxX wide, x from the tile's i0-2): the species at t and
// t-dt and the eddy viscosity with two rows of y halo, u on the tile rows,
// v from one row south to two rows north, w on the tile rows.
constexpr int kScalarTY = 8;
struct ScalarRows {
  static constexpr int s = kScalarTY + 4, u = kScalarTY, v = kScalarTY + 3, w = kScalarTY, r = kScalarTY + 4;
};
struct MoistMaps {
  CUtensorMap s[kMoistN], sp[kMoistN];
  CUtensorMap u, v, w, rkv;   // rkv only with turbulence
};
int launch_moist_scalars(const MoistScalarArgs& a, const MoistMaps& maps, cudaStream_t st);

struct FilterArgs {
  Grid g;
  float* u; float* v; float* w; float* pp; float* ptp;                      // t (filtered in place)
  const float* uf; const float* vf; const float* wf; const float* ppf; const float* ptpf;
  const float* up; const float* vp; const float* wp; const float* ppp; const float* ptpp;
  float filcoe;
  float* tke; const float* tkef; const float* tkep;   // TKE (tubopt=2) or null
};
int launch_timeflt(const FilterArgs& a, cudaStream_t st);

// Fill both periodic ghost layers of up to kHaloMax fields (stag per field).
constexpr int kHaloMax = 32;
struct HaloArgs {
  Grid g;
  float* f[kHaloMax];
  int stag[kHaloMax];
  int n;
};
int launch_halo(const HaloArgs& a, cudaStream_t st);
// Copy `rows` rows of `w` floats between pitches (floats): the host
// layout (pitch ni+2, contiguous) and the device layout (pitch px).
int launch_repitch(const float* src, int src_pitch, float* dst, int dst_pitch, int w, long long rows,
                   cudaStream_t st);

}  // namespace cress

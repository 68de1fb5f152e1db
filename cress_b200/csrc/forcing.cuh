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

struct ForceArgs {
  Grid g;
  const float* col;           // 1-D columns, C_NFIELDS_ALL x (nk+1)
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
  int vsp_u, vsp_v, vsp_w, vsp_p, vsp_pt;  // vspvar switches
};

int launch_force(const ForceArgs& a, cudaStream_t st);

struct FilterArgs {
  Grid g;
  float* u; float* v; float* w; float* pp; float* ptp;                      // t (filtered in place)
  const float* uf; const float* vf; const float* wf; const float* ppf; const float* ptpf;
  const float* up; const float* vp; const float* wp; const float* ppp; const float* ptpp;
  float filcoe;
};
int launch_timeflt(const FilterArgs& a, cudaStream_t st);

// Fill both periodic ghost layers of up to 8 fields (stag per field).
struct HaloArgs {
  Grid g;
  float* f[16];
  int stag[16];
  int n;
};
int launch_halo(const HaloArgs& a, cudaStream_t st);

}  // namespace cress

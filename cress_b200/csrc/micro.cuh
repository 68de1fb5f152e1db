// Cold-rain microphysics kernels (internal interface).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include "common.cuh"
#include "hevi.cuh"

namespace cress {

struct MicroArgs {
  Grid g;
  const float* col;  // 1-D base columns (C_PTBR, C_RBR, C_PBR, C_JCB, C_RST used)
  // past level t-dt (pp: pressure perturbation for p and the Exner function)
  const float *ptpp, *qvp, *qcp, *qrp, *qip, *qsp, *qgp, *nip, *nsp, *ngp, *ppp;
  // future level t+dt (updated)
  float *ptpf, *qvf, *qcf, *qrf, *qif, *qsf, *qgf, *nif, *nsf, *ngf;
  float* prec;       // 10 planes (px*py): prc, prr, pri, prs, prg x (rate, accumulated)
  float* uspd;       // 8 fall-speed fields (past level), written by the process-rate kernels
  int* dtp_bits;     // domain minimum of the sedimentation step (float bits, positive)
  float dtb;         // microphysics step = 2*dtb of the leapfrog (cloudphy.f90:282)
  float dz, thresq;
  int defer_adjstni; // 1: the final adjstni is left to k_moist_post (large step)
};

// Koenig table upload (once per device); returns a CRESS status.
int micro_init_tables();
// s_cloudphy for cphopt=3: source terms and sedimentation; or the two
// halves (process rates with the sub-step minimum, then sedimentation).
int launch_cloudphy(const MicroArgs& a, cudaStream_t st);
int launch_cloudphy_src(const MicroArgs& a, cudaStream_t st);
int launch_cloudphy_fall(const MicroArgs& a, cudaStream_t st);

struct SatArgs {
  Grid g;
  const float* col;  // C_PTBR, C_PBR
  const float* pp;
  float *ptp, *qv, *qc, *qi, *ni;
  float thresq;
};
int launch_satadjst(const SatArgs& a, cudaStream_t st);

// After the moist step's s_cloudphy: the Asselin filter of the nine moist
// fields (when `filter`) and s_satadjst on t and t+dt, pointwise in one
// pass.  Field order qv, qc, qr, qi, qs, qg, ni, ns, ng.
struct MoistPostArgs {
  Grid g;
  const float* col;
  float* c[9];          // t (filtered in place, then adjusted)
  float* f[9];          // t+dt (adjusted)
  const float* p[9];    // t-dt
  float* ptpc; const float* ppc;   // theta', p' at t (already filtered)
  float* ptpf; const float* ppf;   // theta', p' at t+dt
  float filcoe, thresq;
  int filter;
  int adjstni;          // 1: apply cloudphy's final adjstni to t+dt first (coldblk.f90:469)
};
int launch_moist_post(const MoistPostArgs& a, cudaStream_t st);

// Learned form of the process-rate part (the MLP of mlp.cu).
struct Mlp;
struct LearnedBuffers {
  bool fused = false;             // one persistent fused kernel (fb_list holds every cell)
  int chunk = 0;                  // cells per inference chunk (multiple of 128), chunked path
  __nv_bfloat16* xb = nullptr;    // [chunk][64] standardized inputs
  __nv_bfloat16* h0 = nullptr;    // [chunk][256] activations (ping)
  __nv_bfloat16* h1 = nullptr;    // [chunk][256] activations (pong)
  float* y = nullptr;             // [chunk][64] outputs
  unsigned char* env = nullptr;   // [chunk] inside the training envelope
  int* fb_list = nullptr;         // [chunk] cells sent to the plain scheme
  int* fb_count = nullptr;
  unsigned long long* stats = nullptr;   // MLP cells, fallback cells
  int* err = nullptr;
};
int launch_cloudphy_learned(const MicroArgs& a, const float* w, Mlp* m, const LearnedBuffers& L, float resid_tol,
                            cudaStream_t st, long long* launches);
int launch_cloudphy_fused(const MicroArgs& a, const float* w, Mlp* m, const LearnedBuffers& L, float resid_tol,
                          cudaStream_t st, long long* launches);
int launch_collect_tuples(const MicroArgs& a, const float* w, Mlp* m, int stride, float keep_zero,
                          unsigned long long seed, unsigned long long* count_d, cudaStream_t st);

}  // namespace cress

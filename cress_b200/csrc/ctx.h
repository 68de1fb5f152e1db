// Context object behind the opaque cress_ctx handle (internal).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <map>
#include <string>
#include <vector>
#include "../../include/cress_b200.h"
#include "common.cuh"
#include "hevi.cuh"
#include "micro.cuh"
#include "slab.h"

namespace cress {

int set_error(int code, const char* fmt, ...);
int cuda_check(cudaError_t e, const char* what);

// Elimination factors of the w system for one dts (device arrays indexed by k).
struct ThomasSet {
  float* rr = nullptr;
  double* aa = nullptr;
  double* cp = nullptr;
  HeviLevel* lvl3 = nullptr;   // level table of the on-chip kernel (rows 0..nk)
  HeviLevel1* lvl4 = nullptr;  // the same once per value (one-column-per-thread kernel)
};

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;      // stream all work is ordered on
  cudaStream_t own_stream = nullptr;  // the context's own stream (destroyed with it)
  cress_cfg cfg{};
  Grid g{};
  // Device state: lev[field][CRESS_PAST/NOW/FUTURE/FORCING]; spare[] is the
  // ping-pong partner of the future level during the small-step loop.
  float* lev[CRESS_NFIELD][4];
  float* spare[CRESS_NFIELD];
  // HE-VE (impopt=0): contravariant w of levels 2 and nk-1, two planes per
  // buffer, ping-pong between substeps
  float* wcside[2] = {nullptr, nullptr};
  std::vector<float> col_h;   // 1-D base columns on the host
  float* col_d = nullptr;
  bool base_set = false;
  std::map<uint32_t, ThomasSet> thomas;
  std::map<std::pair<const void*, int>, CUtensorMap> tmaps;  // (buffer, box rows) -> map
  int* err_d = nullptr;                                       // device error word
  std::vector<void*> owned;
  long long launches = 0;

  float* alloc_field();
  float* stage_d = nullptr;   // one field in host layout (host<->device transfers)
  int stage();
  int put_host(float* dst, const float* host);
  int get_host(float* host, const float* src);
  // asynchronous read-back (cress_get_fields_async): each field is
  // repitched on `stream` into its own host-layout buffer, then copied to
  // the host on copy_stream, so the copy overlaps later work on `stream`.
  // Two sets of buffers: read-back n uses set n % 2, and its repitch waits
  // (on the device) only for the copies of read-back n-2.
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_out[2] = {}, ev_done[2] = {};
  float* stage_out[CRESS_NFIELD][2] = {};
  long long out_issued = 0, out_waited = 0;   // read-backs issued / seen complete on the host
  int* err_h = nullptr;   // page-locked: the device error word as each set's read-back saw it
  int get_async(int level, int n, const int* fields, float* const* host);
  int wait_async(int keep);   // until at most `keep` read-backs are in flight
  // asynchronous input (cress_put_fields_async): the host->device copies
  // run on in_stream into one host-layout buffer per field and level; the
  // repitch into the level runs on `stream` once they have landed
  // (ev_in[level]); the next copies into a level's buffers wait for the
  // repitch that read them (ev_in_free[level])
  cudaStream_t in_stream = nullptr;
  cudaEvent_t ev_in[4] = {}, ev_in_free[4] = {};
  bool in_used[4] = {};
  float* stage_in[CRESS_NFIELD][4] = {};
  int put_async(int level, int n, const int* fields, const float* const* host);
  // y-slab decomposition (slab.h): the link to the other ranks, or null
  SlabLink* slab = nullptr;
  // byte stream of the dump and restart records (records.cu), kept and
  // grown as needed
  void* rec_d = nullptr;
  long long rec_bytes = 0;
  int thomas_for(float dts, const ThomasSet** out);
  std::map<uint32_t, float*> level_tables;   // level table per 2*dtb (bits)
  int level_table(float dtb2, const float** out);
  int small_steps(int nsstp, float dts);
  // phase 0: the whole step; 1: up to the forcing; 2: from the moist
  // scalars on (an ensemble runs every member's small steps in between)
  int large_step(bool filter, float dtb, int nsstp, float dts, int phase = 0);
  // jobs != null: instead of launching, append every substep's arguments
  // and maps (HE-VI, tile 0) for an ensemble launch; the pointer swaps that
  // make the result the future level are done either way
  int small_steps(int nsstp, float dts, std::vector<HeviJob>* jobs);
  int ksp0 = 2;            // first Rayleigh-damped level
  bool large_set = false;  // cress_set_base_large was called
  bool moist_set = false;  // cress_set_base_moist was called
  float* prec_d = nullptr; // surface precipitation planes (10 x px*py)
  float* uspd_d = nullptr; // fall speeds (8 fields)
  float* rkv_d = nullptr;  // eddy viscosity rbr*K at scalar points (tubopt 1 and 2)
  // TKE closure (tubopt=2), written by the eddy-viscosity kernel from the
  // past level: the scalar diffusivity 1/Pr*rkv/jcb, N^2 at w level k, and
  // the shear production and dissipation of the TKE at scalar points
  float* rks_d = nullptr;
  float* nsq_d = nullptr;
  float* shr_d = nullptr;
  float* dsp_d = nullptr;
  int* dtp_d = nullptr;    // sedimentation sub-step minimum (float bits)
  // defer_adjstni: leave the final adjstni to the moist post kernel (large step)
  int cloudphy(float dtb, float thresq, bool defer_adjstni = false);
  // learned microphysics (MLP in place of the process rates) and tuple
  // sampling of the plain scheme for its training
  Mlp* mlp = nullptr;
  float resid_tol = 0.5f;
  LearnedBuffers lb{};
  std::vector<void*> lb_owned;
  Mlp* sampler = nullptr;
  int sample_stride = 64;
  float sample_keep_zero = 0.1f;
  unsigned long long sample_seed = 1;
  unsigned long long* count_d = nullptr;
  long long sampled = 0;
  void free_learned();
  // CUDA graphs of whole large steps, keyed by the time-level pointer state
  // and the step parameters; each remembers the pointer state it leaves.
  struct GraphRec {
    cudaGraphExec_t exec = nullptr;
    long long nlaunch = 0;
    std::vector<float*> post;
  };
  bool graphs = false;
  std::map<std::string, GraphRec> grec;
  std::map<std::string, int> gseen;
  std::vector<float*> pointer_state() const;
  void set_pointer_state(const std::vector<float*>& s);
  int step(bool filter, float dtb, int nsstp, float dts);
  void free_graphs();
  int satadjst(int level, float thresq);
  int tmap(const float* buf, int rows, CUtensorMap* out);
  int check_device_error();
  void* diag_d = nullptr;
  float* rad_d = nullptr;   // open x: phase speeds (openbc.cuh layout)
  uint32_t spin_limit = kSpinLimit;   // probes per HE-VI ring wait (cress_set_spin_limit)
  int diagnostics(int level, double* out);
  int autotune(int nsstp, float dts, int reps, int* best, float* ms);
  ~Ctx();
};

}  // namespace cress

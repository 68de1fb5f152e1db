// HE-VI substep kernel interface (internal to the library).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include "common.cuh"
#include "status.h"
#include "tma.cuh"

namespace cress {

// 1-D base-state / metric columns of a horizontally uniform base state,
// stored as col[field*(nk+1) + k], k = 1..nk.
enum ColField {
  C_JCB = 0, C_JCB8U, C_JCB8V, C_JCB8W, C_RBR, C_PTBR, C_RST, C_RST8U, C_RST8V, C_RST8W, C_RCSQ,
  C_PBR, C_QVBR, C_UBR, C_VBR, C_ZPH8S,
  // reciprocals (float) of per-level divisors, so the kernels multiply
  C_IRST8U, C_IRST8V, C_IJCB, C_IRCSQ, C_IRST8W, C_IJCB8W, C_NFIELDS
};

// Stride (floats) of the k-major level table (table[k * kLevelStride +
// field]) the large-step kernels and the global-table HE-VI variant read:
// the ColField columns, then the derived values of forcing.cuh.
constexpr int kLevelStride = 32;

// Width (floats) of every TMA box of the HE-VI kernel: x from i0-2 (a
// multiple of 32, so 16-byte aligned) to i0+33, covering the 32-column
// tile with the x halos the stencils need.
constexpr int kHeviTX = 32;
constexpr int kHeviBoxX = 36;

// Rows of the staged boxes (tile height TY): old u, v, w, p' carry y halos.
template <int TY> struct HeviRows {
  static constexpr int u = TY + 2, v = TY + 3, w = TY + 2, p = TY + 2;
  static constexpr int uf = TY, vf = TY + 1, wf = TY, pf = TY;
};

// Tensor maps of the eight staged fields (3-D: x = i, y = j, z = k-1).
struct HeviMaps {
  CUtensorMap u, v, w, p, uf, vf, wf, pf;
};

// One row per level k of the level table of the on-chip HE-VI kernel
// (tile 12): the base-state columns and reciprocals a substep reads, the
// sub-diagonal a_k of the w system (float, as stepwi forms it) and the
// FP64 elimination factors aa_k = 1/(b_k - a_k c'_{k-1}), cp_k = c'_k.
// Every float is stored twice, so a 16-byte load yields two ready operand
// pairs of the packed FP32x2 arithmetic (f2.cuh); nine 16-byte vectors per
// level.
struct alignas(16) HeviLevel {
  float rst8u[2], rst8v[2];     // vector 0
  float rst8w[2], ij8w[2];      // vector 1
  float jcb[2], ijcb[2];        // vector 2
  float irst8u[2], irst8v[2];   // vector 3
  float jcb8u[2], jcb8v[2];     // vector 4
  float rcsq[2], rst[2];        // vector 5
  float rbr[2], ircsq[2];       // vector 6
  float irst8w[2], rr[2];       // vector 7
  double aa, cp;                // vector 8
};
static_assert(sizeof(HeviLevel) == 144, "HeviLevel is nine 16-byte vectors");

// The same values once each (five 16-byte vectors per level), for the
// one-column-per-thread on-chip kernel (tile 13).
struct alignas(16) HeviLevel1 {
  float rst8u, rst8v, rst8w, ij8w;
  float jcb, ijcb, irst8u, irst8v;
  float jcb8u, jcb8v, rcsq, rst;
  float rbr, ircsq, irst8w, rr;
  double aa, cp;
};
static_assert(sizeof(HeviLevel1) == 80, "HeviLevel1 is five 16-byte vectors");

// Largest nk the on-chip kernels hold: the eliminated right-hand sides of
// levels 3..nk-2 of two columns in FP64 fill 4 (nk - 4) <= 256 tensor-memory
// columns per thread.
constexpr int kHevi3MaxNk = 68;

struct HeviArgs {
  Grid g;
  const float* u_old; const float* v_old; const float* p_old;
  float* u_new; float* v_new; float* w_new; float* p_new;
  const float* col;       // 1-D base columns
  const float* lvl;       // the same k-major (level table, stride kLevelStride) or null
  const float* thom_rr;   // [k] sub-diagonal a_k of the w system (float, as formed by stepwi)
  const double* thom_aa;  // [k] 1/(b_k - a_k c'_{k-1})
  const double* thom_cp;  // [k] c'_k
  const HeviLevel* lvl3;  // level table of tile 12 (rows k = 0..nk), or null
  const HeviLevel1* lvl4; // level table of tile 13 (rows k = 0..nk), or null
  int* err;               // device error word (nonzero: a bounded wait gave up)
  // HE-VE only: the contravariant w of levels 2 and nk-1 (two planes of
  // px*py each), which the reference keeps from the explicit update while
  // the rigid lid sets w itself to 0 there; read from wc_old (or formed
  // from w_old when wc_from_w), written to wc_new
  const float* wc_old;
  float* wc_new;
  int wc_from_w;
  float dts, dxiv, dyiv, dziv, divch, divcv, weicoe, dtdzw, dtw, g05, g05n;
  int divopt, buyopt, sthopt, bbc;
  // probes of each ring wait of the k_hevi2 level loop before it gives up
  // (a test of the failure path sets it to 0; the drain keeps kSpinLimit)
  uint32_t spin = kSpinLimit;
};

// Tile heights the kernel is instantiated for.
int hevi_tile_rows(int tile);
// The on-chip kernel (tile 12); needs a.lvl3 and nk <= kHevi3MaxNk.
int launch_hevi3(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st);
// The on-chip kernel with one column per thread (tile 13); needs a.lvl4.
int launch_hevi4(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st);
// Launch one substep; `maps` must describe the buffers in `a` with the
// box rows of HeviRows<hevi_tile_rows(tile)>.
int launch_hevi_substep(const HeviArgs& a, const HeviMaps& maps, int tile, cudaStream_t st);
// One member's substep in an ensemble launch (tile 0's or tile 13's kernel
// over every member's tiles); 64-byte aligned for the tensor maps, in
// block order.
struct alignas(64) HeviJob {
  HeviMaps maps;
  HeviArgs args;
  int first_block, tiles_x;
};
// Tiles of tile shape 0 for a member's grid.
void hevi_job_tiles(const Grid& g, int* tx, int* ty);
// One launch for njobs members (jobs in device memory, nblocks tiles in
// all); every member uses divopt, sthopt != 0 (sth), buyopt == 1 (buy).
int launch_hevi_batch(const HeviJob* jobs_d, int njobs, int nblocks, int nk_max, int divopt, bool sth, bool buy,
                      cudaStream_t st);
// The same with the one-column-per-thread on-chip kernel (tile 13: the same
// 32 x 8 tiles; every member's args.lvl4 set, nk <= kHevi3MaxNk).
int launch_hevi4_batch(const HeviJob* jobs_d, int njobs, int nblocks, int nk_max, int divopt, bool sth, bool buy,
                       cudaStream_t st);

// One HE-VE substep (impopt=0, s_heve); the maps are those of tile 0's
// box rows (HeviRows<8>) and a.lvl must hold the level table.
int launch_heve_substep(const HeviArgs& a, const HeviMaps& maps, cudaStream_t st);

}  // namespace cress

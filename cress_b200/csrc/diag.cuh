// Domain diagnostics (internal interface): FP64 budget sums, maxima and the
// non-finite count of one time level.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"
#include "status.h"

namespace cress {

struct DiagAcc {
  double sum[3];              // water, precipitated water, mass (kg)
  unsigned int maxbits[4];    // max |u|, |v|, |w|, |theta'| as float bits
  unsigned long long nonfinite;
};

struct DiagArgs {
  Grid g;
  const float* col;
  const float *u, *v, *w, *pp, *ptp;
  const float* q[6];          // qv, qc, qr, qi, qs, qg (null: dry)
  const float* n[3];          // ni, ns, ng
  const float* prec;          // precipitation planes (null: none)
  double dv, dxdy;            // dx*dy*dz, dx*dy
  DiagAcc* acc;               // zeroed by the caller
};

int launch_diag(const DiagArgs& a, cudaStream_t st);

}  // namespace cress

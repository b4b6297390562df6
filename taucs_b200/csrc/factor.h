// The factor handle returned through the C ABI.
#pragma once

#include <cuda_runtime.h>

#include "internal.h"
#include "kernels.h"

namespace tb {

struct Factor {
  int flags = TAUCS_DOUBLE;   // first member, as in the reference's handle (src/taucs_sn_llt.c:603-605)
  int n = 0;
  int device = -1;
  Symbolic sym;
  Plan plan;
  DevPlan dp;
  bool dev_ready = false;
  std::vector<int> colptr, rowind;   // the pattern the plan was built for

  // device buffers
  double* dL = nullptr;        // L arena (FP64)
  double* dU = nullptr;        // update arena
  double* dA = nullptr;        // A values
  int* dstatus = nullptr;
  double* dW = nullptr;        // solve work vectors (v_len * SOLVE_NRHS)
  double* dpart = nullptr;     // backward-solve partial sums (plan.part_len)
  double* dX = nullptr;        // solve staging (n * SOLVE_NRHS)
  int* hstatus = nullptr;      // pinned status readback (2 ints: factor, solve)
  double* dDinv = nullptr;     // inverses of the big fronts' 64x64 diagonal blocks
  int* dflags = nullptr;       // solve handshake flags (plan.n_blk)
  int epoch = 0;               // last epoch written into dflags
  bool has_numeric = false;
  int precision = 0;           // 0 FP64, 1 FP32 fronts

  // FP32 path
  float* dL32 = nullptr;
  float* dU32 = nullptr;
  double* dscale = nullptr;    // diagonal scaling (n)
  int* dcolptr = nullptr;      // device copy of the permuted pattern (for SpMV)
  int* drowind = nullptr;
};

cudaStream_t current_stream();

}  // namespace tb

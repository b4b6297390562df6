// The factor handle returned through the C ABI.
#pragma once

#include <array>
#include <cstdint>
#include <functional>
#include <map>
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

  // FP32 fronts (precision 1) and iterative refinement
  float* dL32 = nullptr;
  float* dSp32 = nullptr;      // split arena: split copies of a level's panels (Plan::sp_len)
  int sp_fmt = 1;              // split format of the tensor-core products: 0 TF32 x3, 1 FP16 x3
  float* dU32 = nullptr;
  float* dDinv32 = nullptr;
  float* dA32 = nullptr;       // scaled values D A D in FP32
  float* dW32 = nullptr;       // solve work vectors (FP32)
  float* dpart32 = nullptr;
  float* dV32 = nullptr;       // FP32 right-hand sides / corrections (n x SOLVE_NRHS)
  double* dscale = nullptr;    // D = diag(A)^-1/2 (n)
  bool has_numeric32 = false;
  int* dcolptr = nullptr;      // device copy of the permuted pattern
  int* drowind = nullptr;
  int* dcolidx = nullptr;      // column of every entry (nnz)
  int* ddiagpos = nullptr;     // position of each column's diagonal entry (n)
  int* dcsr_ptr = nullptr;     // full symmetric CSR of the pattern, for the FP64 residual
  int* dcsr_col = nullptr;
  int* dcsr_val = nullptr;     // index of each CSR entry in A's value array
  double* dR = nullptr;        // residual (n x SOLVE_NRHS)
  double* dXi = nullptr;       // the iterate, row-interleaved (n rows of SOLVE_NRHS), for the residual's gathers
  double* dXr = nullptr;       // refined solution (n x SOLVE_NRHS)
  double* dBr = nullptr;       // right-hand sides (n x SOLVE_NRHS)
  unsigned long long* dnorm = nullptr;  // 2 x SOLVE_NRHS inf-norm bit patterns
  unsigned long long* hnorm = nullptr;  // pinned readback
  bool refine_ready = false;
  // PCG fallback of the refinement (preconditioned by the FP32 factor):
  // p, q, z (3 x n x SOLVE_NRHS), per-block dot partials and the dot results
  double* dpcg = nullptr;
  double* ddot_part = nullptr;
  double* ddot = nullptr;
  double* hdot = nullptr;              // pinned readback of ddot
  int pcg_maxits = 100;                // 0: no PCG, stalled refinement refactors in FP64
  int refine_method = 0;               // 0: refinement steps (PCG on stall), 1: PCG from the first step
  int last_fallback = 0;               // last refinement: 0 FP32 steps, 1 PCG, 2 FP64 refactor
  int last_pcg_its = 0;
  const double* dvals_cur = nullptr;   // values of the last numeric factorization (device)
  // independent systems held in one factor (a batch): row ranges seg_ptr[s]
  // .. seg_ptr[s+1]; refinement measures every segment's scaled residual on
  // its own.  Empty: one segment (the whole matrix).
  std::vector<int> seg_ptr;
  int* dseg = nullptr;                 // row -> segment (batches only)
  int nseg() const { return seg_ptr.empty() ? 1 : (int) seg_ptr.size() - 1; }
  // batch of systems: combined value k comes from value vmap[k] of system
  // s (nnz_off[s] <= k < nnz_off[s+1]); combined row seg_ptr[s] + i is row
  // perm[seg_ptr[s] + i] of system s
  struct BatchMap {
    std::vector<int64_t> nnz_off;
    std::vector<int> perm, vmap;
    // device side of taucs_b200_batch_factor / _solve: the systems' values
    // and vectors travel as they are given, concatenated, and are permuted on
    // the device: combined value k = raw[cvmap[k]], combined row i = raw row
    // cperm[i]; pinned host staging for both
    int* d_cvmap = nullptr;
    int* d_cperm = nullptr;
    double* d_raw = nullptr;     // max(nnz, n)
    double* d_b = nullptr;       // n
    double* d_x = nullptr;       // n
    double* h_raw = nullptr;     // pinned, max(nnz, n)
  } batch;

  // recorded launch sequences (numeric factorization, solves, refinement
  // steps), keyed by what they were recorded for; replayed as CUDA graphs
  struct Graph {
    cudaGraphExec_t exec = nullptr;
    long launches = 0;    // kernel launches inside the graph
    bool seen = false;    // the first run of a key is eager (one-time setup)
  };
  std::map<std::array<uint64_t, 6>, Graph> graphs;
  cudaStream_t cap_stream = nullptr;
  // record a key's graph on its first run instead of its second: for factors
  // whose buffers are reused by construction (request server instances), so
  // the one eager pass buys nothing
  bool graph_first_use = false;
};

using GraphKey = std::array<uint64_t, 6>;
// Enqueues record(stream) on st: the first time for a key eagerly (unless
// F->graph_first_use), then recorded once into a CUDA graph and replayed.  Eager whenever per-launch
// profiling is on or TAUCS_B200_NO_GRAPHS is set.  Returns record's result
// (0 or a cudaError_t).
int run_graphed(Factor* F, const GraphKey& key, cudaStream_t st, const std::function<int(cudaStream_t)>& record);
void drop_graphs(Factor* F);

cudaStream_t current_stream();
bool cuda_ok(cudaError_t e, const char* what);
int ensure_device(Factor* F);
void free_numeric(Factor* F);
// marks the numeric factors stale without freeing their buffers
void invalidate_numeric(Factor* F);
int numeric_fp64_device(Factor* F, const double* d_vals, bool wait);
// FP32 fronts: 0 on success, 1 on a nonpositive pivot (the caller may
// refactor in FP64), -1 on any other failure (message set)
int numeric_fp32_device(Factor* F, const double* d_vals);
// Reads a numeric factorization's status word: 0 (INT_MAX, success), 1 (a
// nonpositive pivot; its column is logged) or -1 (NUMERIC_TIMEOUT: a bounded
// device wait gave up).  Sets the error message for both failures.
int numeric_status_check(int word, const char* what);

}  // namespace tb

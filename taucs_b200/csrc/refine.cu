// Mixed precision: FP32 fronts with FP64 iterative refinement.
//
// The reference's precedent (progs/direct.c:656-663) is one refinement step
// with everything in FP32 and an FP64-accumulated SpMV
// (taucs_sccs_times_vec_dacc, src/taucs_ccs_ops.c:348-386).  Here:
//   * the matrix is scaled symmetrically, A_s = D A D with D = diag(A)^-1/2,
//     and A_s is factored with FP32 fronts (TF32x3 tensor products, FP32
//     POTRF); a nonpositive FP32 pivot refactors in FP64;
//   * refinement keeps x, b and the residual r = b - A x in FP64 on the device
//     (symmetric CSR SpMV over the lower-triangle values, each row summed by
//     one thread in a fixed order), solves L_s L_s^T d_s = D r in FP32 and
//     updates x += D d_s, until the scaled residual
//     ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf) reaches the target; when a
//     step fails to halve the residual twice in a row, or the step limit is
//     reached, it refactors in FP64 and finishes with the FP64 factor.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "factor.h"

namespace tb {

namespace {

__global__ void k_diag_scale(int n, const int* __restrict__ diagpos, const double* __restrict__ vals,
                             double* __restrict__ scale, int* status) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double d = diagpos[j] >= 0 ? vals[diagpos[j]] : 0.0;
  if (!(d > 0.0)) {
    atomicMin(status, j);
    scale[j] = 1.0;
  } else {
    scale[j] = rsqrt(d);
  }
}

__global__ void k_scaled_f32(long nnz, const int* __restrict__ rowind, const int* __restrict__ colidx,
                             const double* __restrict__ vals, const double* __restrict__ scale,
                             float* __restrict__ out) {
  const long k = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  out[k] = (float) (vals[k] * scale[rowind[k]] * scale[colidx[k]]);
}

// non-negative doubles order like their bit patterns
__device__ __forceinline__ void max_abs(unsigned long long* slot, double v) {
  atomicMax(slot, (unsigned long long) __double_as_longlong(fabs(v)));
}

// warp-level max into a segment's slot: one atomic per warp when the warp's
// rows lie in one segment, one per row otherwise
__device__ __forceinline__ void seg_max(unsigned long long* slots, int sg, int stride, double v) {
  const int lane = threadIdx.x & 31;
  const int sg0 = __shfl_sync(0xffffffffu, sg, 0);
  if (__all_sync(0xffffffffu, sg == sg0)) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) max_abs(slots + (size_t) sg0 * stride, v);
  } else {
    max_abs(slots + (size_t) sg * stride, v);
  }
}

// R = B - A X (FP64; X and B with leading dimension ld, R with ldr);
// inf-norms of R and X per column and segment: norms[(s * SOLVE_NRHS + q) * 2]
// (r) and [.. + 1] (x); seg == NULL: one segment
__global__ void k_residual(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           const int* __restrict__ vi, const double* __restrict__ vals,
                           const double* __restrict__ X, const double* __restrict__ B, double* __restrict__ R,
                           int ld, int ldr, int nrhs, const int* __restrict__ seg, unsigned long long* norms) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int sg = (seg && i < n) ? seg[i] : 0;
  // the row's entries eight at a time, then every column's products with
  // all loads in flight together; per column the entries are subtracted in
  // row order
  double acc[SOLVE_NRHS];
#pragma unroll
  for (int q = 0; q < SOLVE_NRHS; q++) acc[q] = (i < n && q < nrhs) ? B[i + (size_t) q * ld] : 0.0;
  const int e0 = (i < n) ? rp[i] : 0, e1 = (i < n) ? rp[i + 1] : 0;
  for (int eb = e0; eb < e1; eb += 8) {
    int c[8];
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) c[u] = (eb + u < e1) ? ci[eb + u] : -1;
#pragma unroll
    for (int u = 0; u < 8; u++) v[u] = (c[u] >= 0) ? vals[vi[eb + u]] : 0.0;
#pragma unroll
    for (int q = 0; q < SOLVE_NRHS; q++) {
      if (q >= nrhs) break;
      double xv[8];
#pragma unroll
      for (int u = 0; u < 8; u++) xv[u] = (c[u] >= 0) ? X[c[u] + (size_t) q * ld] : 0.0;
#pragma unroll
      for (int u = 0; u < 8; u++)
        if (c[u] >= 0) acc[q] -= v[u] * xv[u];
    }
  }
#pragma unroll
  for (int q = 0; q < SOLVE_NRHS; q++) {
    if (q >= nrhs) break;
    double r = 0.0, x = 0.0;
    if (i < n) {
      R[i + (size_t) q * ldr] = acc[q];
      r = fabs(acc[q]);
      x = fabs(X[i + (size_t) q * ld]);
    }
    seg_max(norms + 2 * q, sg, 2 * SOLVE_NRHS, r);
    seg_max(norms + 2 * q + 1, sg, 2 * SOLVE_NRHS, x);
  }
}

// the iterate's rows interleaved: Xi[i][q] = X[i + q ld] (zero past nrhs), so
// that the residual gathers one 64-byte row per matrix entry instead of
// eight scattered values
__global__ void k_interleave(int n, const double* __restrict__ X, int ld, int nrhs, double* __restrict__ Xi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v[SOLVE_NRHS];
#pragma unroll
  for (int q = 0; q < SOLVE_NRHS; q++) v[q] = (q < nrhs) ? X[i + (size_t) q * ld] : 0.0;
  double2* o = reinterpret_cast<double2*>(Xi + (size_t) i * SOLVE_NRHS);
#pragma unroll
  for (int q = 0; q < SOLVE_NRHS; q += 2) o[q / 2] = make_double2(v[q], v[q + 1]);
}

// k_residual over the interleaved iterate (same results, bit for bit: the
// entries of a row are subtracted in the same order)
constexpr int RES_THREADS = 256;   // the block size k_residual_i is launched with

__global__ void __launch_bounds__(RES_THREADS) k_residual_i(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                             const int* __restrict__ vi, const double* __restrict__ vals,
                             const double* __restrict__ Xi, const double* __restrict__ B, double* __restrict__ R,
                             int ld, int ldr, int nrhs, const int* __restrict__ seg, unsigned long long* norms) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int sg = (seg && i < n) ? seg[i] : 0;
  double acc[SOLVE_NRHS];
#pragma unroll
  for (int q = 0; q < SOLVE_NRHS; q++) acc[q] = (i < n && q < nrhs) ? B[i + (size_t) q * ld] : 0.0;
  const int e0 = (i < n) ? rp[i] : 0, e1 = (i < n) ? rp[i + 1] : 0;
  for (int eb = e0; eb < e1; eb += 4) {
    int c[4];
    double v[4];
#pragma unroll
    for (int u = 0; u < 4; u++) c[u] = (eb + u < e1) ? ci[eb + u] : -1;
#pragma unroll
    for (int u = 0; u < 4; u++) v[u] = (c[u] >= 0) ? vals[vi[eb + u]] : 0.0;
    double2 xr[4][SOLVE_NRHS / 2];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const double2* row = reinterpret_cast<const double2*>(Xi + (size_t) max(c[u], 0) * SOLVE_NRHS);
#pragma unroll
      for (int h = 0; h < SOLVE_NRHS / 2; h++) xr[u][h] = (c[u] >= 0) ? row[h] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (c[u] >= 0) {
#pragma unroll
        for (int h = 0; h < SOLVE_NRHS / 2; h++) {
          acc[2 * h] -= v[u] * xr[u][h].x;
          acc[2 * h + 1] -= v[u] * xr[u][h].y;
        }
      }
  }
  double xs[SOLVE_NRHS];
  {
    const double2* row = reinterpret_cast<const double2*>(Xi + (size_t) (i < n ? i : 0) * SOLVE_NRHS);
#pragma unroll
    for (int h = 0; h < SOLVE_NRHS / 2; h++) {
      const double2 t = row[h];
      xs[2 * h] = t.x;
      xs[2 * h + 1] = t.y;
    }
  }
  // the norms: when every row of the block lies in one segment (the usual
  // case) the block reduces them first and issues one atomic per norm --
  // one per warp would queue thousands of atomics on the same few words
  __shared__ int sg_blk;
  __shared__ double red[RES_THREADS / 32][2 * SOLVE_NRHS];
  if (threadIdx.x == 0) sg_blk = sg;
  __syncthreads();
  const bool uni = __syncthreads_and(sg == sg_blk) != 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < SOLVE_NRHS; q++) {
    if (q >= nrhs) break;
    double r = 0.0, x = 0.0;
    if (i < n) {
      R[i + (size_t) q * ldr] = acc[q];
      r = fabs(acc[q]);
      x = fabs(xs[q]);
    }
    if (uni) {
      for (int o = 16; o > 0; o >>= 1) {
        r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
        x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
      }
      if (lane == 0) {
        red[warp][2 * q] = r;
        red[warp][2 * q + 1] = x;
      }
    } else {
      seg_max(norms + 2 * q, sg, 2 * SOLVE_NRHS, r);
      seg_max(norms + 2 * q + 1, sg, 2 * SOLVE_NRHS, x);
    }
  }
  if (uni) {
    __syncthreads();
    const int t = threadIdx.x;
    if (t < 2 * nrhs) {
      double m = 0.0;
#pragma unroll
      for (int w = 0; w < RES_THREADS / 32; w++) m = fmax(m, red[w][t]);
      max_abs(norms + (size_t) sg_blk * 2 * SOLVE_NRHS + t, m);
    }
  }
}

__global__ void k_scale_down(int n, const double* __restrict__ R, const double* __restrict__ scale,
                             float* __restrict__ out, int ld, int nrhs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int q = 0; q < nrhs; q++) out[i + (size_t) q * n] = (float) (R[i + (size_t) q * ld] * scale[i]);
}

__global__ void k_update32(int n, double* __restrict__ X, const float* __restrict__ D, const double* __restrict__ scale,
                           int ld, int nrhs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int q = 0; q < nrhs; q++) X[i + (size_t) q * ld] += scale[i] * (double) D[i + (size_t) q * n];
}

// value k of P A P^T is value vmap[k] of A as given (the value map of
// taucs_ccs_permute_symmetrically, src/taucs_ccs_ops.c:174-257, precomputed
// once per pattern)
__global__ void k_gather_values(long nnz, const int* __restrict__ vmap, const double* __restrict__ raw,
                                double* __restrict__ out) {
  for (long k = (long) blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (long) gridDim.x * blockDim.x)
    out[k] = raw[vmap[k]];
}

// P b and its inverse (src/taucs_vec_base.c:194-206): dst[i] = src[perm[i]]
// and dst[perm[i]] = src[i], nq columns, original-order vectors with ld n
__global__ void k_perm_gather(int n, int nq, const int* __restrict__ perm, const double* __restrict__ src,
                              double* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int pi = perm[i];
  for (int q = 0; q < nq; q++) dst[i + (size_t) q * n] = src[pi + (size_t) q * n];
}

__global__ void k_perm_scatter(int n, int nq, const int* __restrict__ perm, const double* __restrict__ src,
                               double* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int pi = perm[i];
  for (int q = 0; q < nq; q++) dst[pi + (size_t) q * n] = src[i + (size_t) q * n];
}

__global__ void k_update64(int n, double* __restrict__ X, const double* __restrict__ D, int ld, int ldd, int nrhs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int q = 0; q < nrhs; q++) X[i + (size_t) q * ld] += D[i + (size_t) q * ldd];
}

// ---- preconditioned conjugate gradients (fallback of the refinement)

constexpr int DOT_BLOCKS = 296;   // fixed grid, so the summation order never changes
constexpr int PCG_STALL = 10;     // iterations over which PCG must at least halve its residual

struct Coef {
  double v[SOLVE_NRHS];
};

// Y = A X for nq columns (symmetric CSR of both triangles; leading dimension n)
__global__ void k_spmv(int n, const int* __restrict__ rp, const int* __restrict__ ci, const int* __restrict__ vi,
                       const double* __restrict__ vals, const double* __restrict__ X, double* __restrict__ Y, int nq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int q = 0; q < nq; q++) {
    double acc = 0.0;
    for (int e = rp[i]; e < rp[i + 1]; e++) acc += vals[vi[e]] * X[ci[e] + (size_t) q * n];
    Y[i + (size_t) q * n] = acc;
  }
}

// Z = D d: an FP32 correction scaled back to A's variables
__global__ void k_scale_up(int n, const float* __restrict__ D, const double* __restrict__ scale, double* __restrict__ Z,
                           int nq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int q = 0; q < nq; q++) Z[i + (size_t) q * n] = scale[i] * (double) D[i + (size_t) q * n];
}

// a_q . b_q for nq columns in two fixed-order stages: every block sums a
// fixed set of rows with a shared-memory tree, then one thread per column
// adds the block sums in block order
__global__ void __launch_bounds__(256) k_dot_part(int n, int nq, const double* __restrict__ A,
                                                  const double* __restrict__ B, double* __restrict__ part) {
  __shared__ double sh[256];
  for (int q = 0; q < nq; q++) {
    double acc = 0.0;
    for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256)
      acc += A[i + (size_t) q * n] * B[i + (size_t) q * n];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x * SOLVE_NRHS + q] = sh[0];
    __syncthreads();
  }
}

__global__ void k_dot_final(int nblocks, int nq, const double* __restrict__ part, double* __restrict__ out) {
  const int q = threadIdx.x;
  if (q >= nq) return;
  double acc = 0.0;
  for (int b = 0; b < nblocks; b++) acc += part[b * SOLVE_NRHS + q];
  out[q] = acc;
}

// search direction: P = Z + beta P (P = Z on a (re)start)
__global__ void k_pcg_dir(int n, int nq, const double* __restrict__ Z, double* __restrict__ Pd, Coef beta, int restart) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int q = 0; q < nq; q++) {
    const size_t k = i + (size_t) q * n;
    Pd[k] = restart ? Z[k] : Z[k] + beta.v[q] * Pd[k];
  }
}

// X += alpha P, R -= alpha Q, and the inf-norms of R and X per column (the
// one-segment layout of k_residual's norms)
__global__ void k_pcg_step(int n, int nq, double* __restrict__ X, int ld, double* __restrict__ R,
                           const double* __restrict__ Pd, const double* __restrict__ Q, Coef alpha,
                           unsigned long long* norms) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  for (int q = 0; q < nq; q++) {
    double r = 0.0, x = 0.0;
    if (i < n) {
      const size_t k = i + (size_t) q * n;
      const double xi = X[i + (size_t) q * ld] + alpha.v[q] * Pd[k];
      const double ri = R[k] - alpha.v[q] * Q[k];
      X[i + (size_t) q * ld] = xi;
      R[k] = ri;
      r = fabs(ri);
      x = fabs(xi);
    }
    seg_max(norms + 2 * q, 0, 2 * SOLVE_NRHS, r);
    seg_max(norms + 2 * q + 1, 0, 2 * SOLVE_NRHS, x);
  }
}

__global__ void k_init_status2(int* s) { *s = INT_MAX; }

// ||A||_inf of the full symmetric matrix from the CSR of both triangles
// ||A||_inf per segment: out[s]
__global__ void k_anorm(int n, const int* __restrict__ rp, const int* __restrict__ vi, const double* __restrict__ vals,
                        const int* __restrict__ seg, unsigned long long* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int sg = (seg && i < n) ? seg[i] : 0;
  double a = 0.0;
  if (i < n)
    for (int e = rp[i]; e < rp[i + 1]; e++) a += fabs(vals[vi[e]]);
  seg_max(out, sg, 1, a);
}

inline int nblk(long n, int b) { return (int) ((n + b - 1) / b); }

}  // namespace

// norm slots: 2 x SOLVE_NRHS per segment
static size_t norm_bytes(const Factor* F) {
  return sizeof(unsigned long long) * 2 * SOLVE_NRHS * (size_t) F->nseg();
}

// pattern-derived arrays for scaling and the FP64 residual
static int ensure_refine(Factor* F) {
  if (F->refine_ready) return 0;
  if (ensure_device(F)) return -1;
  const int n = F->n;
  const long nnz = F->colptr[n];
  std::vector<int> colidx(std::max(nnz, 1L)), diagpos(std::max(n, 1), -1), cnt(n + 1, 0);
  for (int j = 0; j < n; j++)
    for (int ip = F->colptr[j]; ip < F->colptr[j + 1]; ip++) {
      const int i = F->rowind[ip];
      colidx[ip] = j;
      if (i == j && diagpos[j] < 0) diagpos[j] = ip;
      cnt[i + 1]++;
      if (i != j) cnt[j + 1]++;
    }
  for (int i = 0; i < n; i++) cnt[i + 1] += cnt[i];
  const long ne = cnt[n];
  std::vector<int> ccol(std::max(ne, 1L)), cval(std::max(ne, 1L)), fill(cnt.begin(), cnt.end() - 1);
  for (int j = 0; j < n; j++)
    for (int ip = F->colptr[j]; ip < F->colptr[j + 1]; ip++) {
      const int i = F->rowind[ip];
      ccol[fill[i]] = j; cval[fill[i]] = ip; fill[i]++;
      if (i != j) { ccol[fill[j]] = i; cval[fill[j]] = ip; fill[j]++; }
    }
  cudaStream_t st = current_stream();
  auto up = [&](int** d, const std::vector<int>& h) {
    return cuda_ok(tb::dmalloc(d, sizeof(int) * h.size()), "cudaMalloc") &&
           cuda_ok(cudaMemcpyAsync(*d, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, st), "copy");
  };
  const size_t nv = (size_t) n * SOLVE_NRHS;
  if (!F->seg_ptr.empty()) {
    std::vector<int> seg(std::max(n, 1));
    for (int sg = 0; sg < F->nseg(); sg++)
      for (int i = F->seg_ptr[sg]; i < F->seg_ptr[sg + 1]; i++) seg[i] = sg;
    if (!up(&F->dseg, seg)) return -1;
  }
  bool ok = up(&F->dcolidx, colidx) && up(&F->ddiagpos, diagpos) && up(&F->dcsr_ptr, cnt) && up(&F->dcsr_col, ccol) &&
            up(&F->dcsr_val, cval) &&
            cuda_ok(tb::dmalloc(&F->dscale, sizeof(double) * std::max(n, 1)), "cudaMalloc") &&
            cuda_ok(tb::dmalloc(&F->dR, sizeof(double) * nv), "cudaMalloc") &&
            cuda_ok(tb::dmalloc(&F->dXi, sizeof(double) * nv), "cudaMalloc") &&
            cuda_ok(tb::dmalloc(&F->dXr, sizeof(double) * nv), "cudaMalloc") &&
            cuda_ok(tb::dmalloc(&F->dBr, sizeof(double) * nv), "cudaMalloc") &&
            cuda_ok(tb::dmalloc(&F->dV32, sizeof(float) * nv), "cudaMalloc") &&
            cuda_ok(tb::dmalloc(&F->dnorm, norm_bytes(F)), "cudaMalloc") &&
            cuda_ok(tb::hmalloc(&F->hnorm, norm_bytes(F)), "cudaMallocHost") &&
            cuda_ok(cudaStreamSynchronize(st), "refine setup");
  if (!ok) return -1;
  F->refine_ready = true;
  return 0;
}

int numeric_fp32_device(Factor* F, const double* d_vals) {
  if (ensure_device(F) || ensure_refine(F)) return -1;
  const Plan& P = F->plan;
  cudaStream_t st = current_stream();
  auto al = [&](float** d, size_t n, const char* w) { return *d || cuda_ok(tb::dmalloc(d, sizeof(float) * std::max<size_t>(n, 1)), w); };
  if (!al(&F->dL32, P.l_len, "cudaMalloc(L32)") || !al(&F->dU32, P.u_len, "cudaMalloc(U32)") ||
      !al(&F->dSp32, P.sp_len, "cudaMalloc(split arena)") ||
      !al(&F->dDinv32, P.dinv_len, "cudaMalloc(Dinv32)") || !al(&F->dA32, P.nnz, "cudaMalloc(A32)") ||
      !al(&F->dW32, (size_t) P.v_len * SOLVE_NRHS, "cudaMalloc(W32)") || !al(&F->dpart32, P.part_len, "cudaMalloc(part32)")) {
    free_numeric(F);
    return -1;
  }
  F->dvals_cur = d_vals;
  k_init_status2<<<1, 1, 0, st>>>(F->dstatus);
  k_diag_scale<<<nblk(F->n, 256), 256, 0, st>>>(F->n, F->ddiagpos, d_vals, F->dscale, F->dstatus);
  k_scaled_f32<<<nblk(P.nnz, 256), 256, 0, st>>>(P.nnz, F->drowind, F->dcolidx, d_vals, F->dscale, F->dA32);
  count_launch(3);
  cudaMemcpyAsync(F->hstatus, F->dstatus, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (!cuda_ok(cudaStreamSynchronize(st), "scaling")) return -1;
  if (*F->hstatus != INT_MAX) {
    tprintf("\t\tscaling: nonpositive diagonal in column %d\n", *F->hstatus);
    return 1;
  }
  int e = run_graphed(F, GraphKey{2, (uint64_t) F->dA32, 0, 0, 0, 0}, st, [&](cudaStream_t s) {
    return launch_numeric_fp32(P, F->dp, F->dA32, F->dL32, F->dU32, F->dDinv32, F->dSp32, F->sp_fmt, F->dstatus, s);
  });
  if (!cuda_ok((cudaError_t) e, "numeric launch")) return -1;
  cudaMemcpyAsync(F->hstatus, F->dstatus, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (!cuda_ok(cudaStreamSynchronize(st), "numeric factorization (FP32)")) return -1;
  const int rc = numeric_status_check(*F->hstatus, "FP32 fronts");
  if (rc != 0) return rc;
  F->has_numeric32 = true;
  return 0;
}

// Refines X (device, n x nrhs, ld) for B; returns the number of correction
// steps or -1; res (host, nrhs) gets the final scaled residuals.
// Preconditioned conjugate gradients for the nq columns of one refinement
// block, after taucs_conjugate_gradients (src/taucs_iter.c:66-223) with the
// refinement's scaled-residual test in place of its relative 2-norm test.
// Starts from the current X; the preconditioner is the FP32 factor applied as
// the refinement's correction, z = D (L32 L32^T)^-1 D r.  The iteration runs
// on the recursively updated residual; when every column meets tol there,
// b - A x confirms it (otherwise all columns restart from the true residual).
// alpha and beta come from fixed-order dot products, so a rerun gives the same
// result bit for bit.  A column whose r.z or p.Ap is not positive (the FP32
// preconditioner is not exactly symmetric) is frozen.  Returns the iterations
// used; -1 when some column is not within tol after F->pcg_maxits iterations,
// or when the worst scaled residual has not at least halved over the last
// PCG_STALL iterations (each costs about one FP32 solve, so a stagnating PCG
// hands over to the FP64 refactorization early); X then holds the last
// iterate and F->dR, F->hnorm its true residual.  -2 on a CUDA error.
static int pcg_fp32(Factor* F, int nq, double* X, const double* B, int ld, double tol, double anorm,
                    const double* bnorm, double* res_q) {
  const Plan& P = F->plan;
  const int n = F->n;
  cudaStream_t st = current_stream();
  const size_t nv = (size_t) n * SOLVE_NRHS;
  if (!F->dpcg && !(cuda_ok(tb::dmalloc(&F->dpcg, sizeof(double) * 3 * nv), "cudaMalloc(pcg)") &&
                    cuda_ok(tb::dmalloc(&F->ddot_part, sizeof(double) * DOT_BLOCKS * SOLVE_NRHS), "cudaMalloc(pcg)") &&
                    cuda_ok(tb::dmalloc(&F->ddot, sizeof(double) * 2 * SOLVE_NRHS), "cudaMalloc(pcg)") &&
                    cuda_ok(tb::hmalloc(&F->hdot, sizeof(double) * 2 * SOLVE_NRHS), "cudaMallocHost(pcg)")))
    return -2;
  double* Pd = F->dpcg;
  double* Q = Pd + nv;
  double* Z = Q + nv;
  double* R = F->dR;
  auto dots = [&](const double* a, const double* b, int slot) {
    k_dot_part<<<DOT_BLOCKS, 256, 0, st>>>(n, nq, a, b, F->ddot_part);
    k_dot_final<<<1, 32, 0, st>>>(DOT_BLOCKS, nq, F->ddot_part, F->ddot + slot * SOLVE_NRHS);
    count_launch(2);
  };
  auto fetch = [&](void* h, const void* d, size_t bytes) {
    return cuda_ok(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, st), "pcg readback");
  };
  auto true_residual = [&]() {
    cudaMemsetAsync(F->dnorm, 0, norm_bytes(F), st);
    k_residual<<<nblk(n, 256), 256, 0, st>>>(n, F->dcsr_ptr, F->dcsr_col, F->dcsr_val, F->dvals_cur, X, B, R, ld, n,
                                             nq, nullptr, F->dnorm);
    count_launch();
    return fetch(F->hnorm, F->dnorm, norm_bytes(F)) && cuda_ok(cudaStreamSynchronize(st), "pcg residual");
  };
  // worst scaled residual over the columns, from the norms in F->hnorm
  auto scaled = [&](double* out) {
    double worst = 0.0;
    for (int q = 0; q < nq; q++) {
      double rn, xn;
      memcpy(&rn, &F->hnorm[(size_t) q * 2], 8);
      memcpy(&xn, &F->hnorm[(size_t) q * 2 + 1], 8);
      const double den = anorm * xn + bnorm[q];
      const double v = den > 0 ? rn / den : 0.0;
      if (out) out[q] = v;
      worst = std::max(worst, std::isnan(v) ? INFINITY : v);
    }
    return worst;
  };
  if (!true_residual()) return -2;
  std::vector<double> rho(nq), rho_old(nq, 0.0), hist;   // hist: worst scaled residual per iteration
  hist.push_back(scaled(nullptr));
  bool restart = true;
  for (int it = 0; it < F->pcg_maxits;) {
    // z = M^-1 r and rho = r.z
    k_scale_down<<<nblk(n, 256), 256, 0, st>>>(n, R, F->dscale, F->dV32, n, nq);
    int e = launch_solve_fp32(P, F->dp, F->dL32, F->dDinv32, nq, F->dV32, F->dV32, n, F->dW32, F->dpart32, F->dflags,
                              &F->epoch, F->dstatus + 1, st);
    k_scale_up<<<nblk(n, 256), 256, 0, st>>>(n, F->dV32, F->dscale, Z, nq);
    count_launch(2);
    if (e) return -2;
    dots(R, Z, 0);
    if (!fetch(F->hdot, F->ddot, sizeof(double) * SOLVE_NRHS) || !cuda_ok(cudaStreamSynchronize(st), "pcg")) return -2;
    Coef beta{}, alpha{};
    for (int q = 0; q < nq; q++) {
      rho[q] = F->hdot[q];
      beta.v[q] = (!restart && rho_old[q] > 0 && rho[q] > 0) ? rho[q] / rho_old[q] : 0.0;
    }
    // p = z + beta p, q = A p, alpha = rho / p.q
    k_pcg_dir<<<nblk(n, 256), 256, 0, st>>>(n, nq, Z, Pd, beta, restart ? 1 : 0);
    k_spmv<<<nblk(n, 256), 256, 0, st>>>(n, F->dcsr_ptr, F->dcsr_col, F->dcsr_val, F->dvals_cur, Pd, Q, nq);
    count_launch(2);
    dots(Pd, Q, 1);
    if (!fetch(F->hdot + SOLVE_NRHS, F->ddot + SOLVE_NRHS, sizeof(double) * SOLVE_NRHS) ||
        !cuda_ok(cudaStreamSynchronize(st), "pcg"))
      return -2;
    for (int q = 0; q < nq; q++) {
      const double pq = F->hdot[SOLVE_NRHS + q];
      alpha.v[q] = (rho[q] > 0 && pq > 0) ? rho[q] / pq : 0.0;
    }
    // x += alpha p, r -= alpha q, and the norms of the updated residual
    cudaMemsetAsync(F->dnorm, 0, norm_bytes(F), st);
    k_pcg_step<<<nblk(n, 256), 256, 0, st>>>(n, nq, X, ld, R, Pd, Q, alpha, F->dnorm);
    count_launch();
    if (!fetch(F->hnorm, F->dnorm, norm_bytes(F)) || !cuda_ok(cudaStreamSynchronize(st), "pcg")) return -2;
    rho_old = rho;
    restart = false;
    it++;
    const double worst = scaled(nullptr);
    if (worst <= tol) {
      if (!true_residual()) return -2;
      if (scaled(res_q) <= tol) return it;
      restart = true;   // the recursive residual drifted: go on from b - A x
    }
    hist.push_back(worst);
    if (it >= PCG_STALL && !(worst <= 0.5 * hist[hist.size() - 1 - PCG_STALL])) break;
  }
  if (!true_residual()) return -2;
  scaled(res_q);
  return -1;
}

static int refine_device(Factor* F, int nrhs, double* dX, const double* dB, int ld, double tol, int maxits,
                         const std::vector<double>& anorm, double* res) {
  const Plan& P = F->plan;
  const int n = F->n, ns = F->nseg();
  cudaStream_t st = current_stream();
  int total = 0;
  F->last_fallback = 0;
  F->last_pcg_its = 0;
  for (int q0 = 0; q0 < nrhs; q0 += SOLVE_NRHS) {
    const int nq = std::min(SOLVE_NRHS, nrhs - q0);
    double* X = dX + (size_t) q0 * ld;
    const double* B = dB + (size_t) q0 * ld;
    std::vector<double> bnorm((size_t) nq * ns, 0.0);
    // r = b - A x and the inf-norms of r and x per segment, read back
    auto residual = [&](cudaStream_t s) {
      cudaMemsetAsync(F->dnorm, 0, norm_bytes(F), s);
      k_interleave<<<nblk(n, 256), 256, 0, s>>>(n, X, ld, nq, F->dXi);
      k_residual_i<<<nblk(n, RES_THREADS), RES_THREADS, 0, s>>>(n, F->dcsr_ptr, F->dcsr_col, F->dcsr_val, F->dvals_cur, F->dXi, B,
                                                F->dR, ld, n, nq, F->dseg, F->dnorm);
      count_launch(2);
      cudaMemcpyAsync(F->hnorm, F->dnorm, norm_bytes(F), cudaMemcpyDeviceToHost, s);
      return (int) cudaGetLastError();
    };
    // one correction step x += A~^-1 r, then the next residual
    auto correction = [&](cudaStream_t s, bool u64) {
      int e;
      if (u64) {
        e = launch_solve_fp64(P, F->dp, F->dL, F->dDinv, nq, F->dR, F->dR, n, F->dW, F->dpart, F->dflags, &F->epoch,
                              F->dstatus + 1, s);
        k_update64<<<nblk(n, 256), 256, 0, s>>>(n, X, F->dR, ld, n, nq);
      } else {
        k_scale_down<<<nblk(n, 256), 256, 0, s>>>(n, F->dR, F->dscale, F->dV32, n, nq);
        e = launch_solve_fp32(P, F->dp, F->dL32, F->dDinv32, nq, F->dV32, F->dV32, n, F->dW32, F->dpart32,
                              F->dflags, &F->epoch, F->dstatus + 1, s);
        k_update32<<<nblk(n, 256), 256, 0, s>>>(n, X, F->dV32, F->dscale, ld, nq);
      }
      count_launch(2);
      return e ? e : residual(s);
    };
    // ||b||_inf per column, from a residual pass with X = 0
    cudaMemsetAsync(X, 0, sizeof(double) * ((size_t) ld * (nq - 1) + n), st);
    if (run_graphed(F, GraphKey{6, (uint64_t) nq, (uint64_t) X, (uint64_t) B, (uint64_t) ld, 0}, st, residual))
      return -1;
    bool use64 = !F->has_numeric32;
    double prev_worst = INFINITY;
    int slow = 0, steps = 0;
    bool done = false;
    if (!use64 && ns == 1 && F->refine_method == 1 && F->pcg_maxits > 0) {
      // conjugate gradients preconditioned by the FP32 factor from the start
      // (from x = 0); the FP64 refactorization below only if they fail
      if (!cuda_ok(cudaStreamSynchronize(st), "refinement")) return -1;
      for (int q = 0; q < nq; q++) memcpy(&bnorm[q], &F->hnorm[(size_t) q * 2], 8);
      std::vector<double> rq(nq, 0.0);
      const int its = pcg_fp32(F, nq, X, B, ld, tol, anorm[0], bnorm.data(), rq.data());
      if (its == -2) return -1;
      if (res)
        for (int q = 0; q < nq; q++) res[q0 + q] = rq[q];
      F->last_pcg_its += std::max(its, 0);
      if (its >= 0) {
        F->last_fallback = std::max(F->last_fallback, 1);
        total = std::max(total, its);
        continue;
      }
      tprintf("\t\tPCG did not reach the tolerance; refactoring in FP64\n");
      if (!F->has_numeric && numeric_fp64_device(F, F->dvals_cur, true)) return -1;
      F->last_fallback = 2;
      use64 = true;
      cudaMemsetAsync(X, 0, sizeof(double) * ((size_t) ld * (nq - 1) + n), st);
      if (run_graphed(F, GraphKey{6, (uint64_t) nq, (uint64_t) X, (uint64_t) B, (uint64_t) ld, 0}, st, residual))
        return -1;
    }
    for (int it = 0; !done; it++) {
      if (!cuda_ok(cudaStreamSynchronize(st), "refinement")) return -1;
      double worst = 0.0;
      for (int sg = 0; sg < ns; sg++)
        for (int q = 0; q < nq; q++) {
          double rn, xn;
          memcpy(&rn, &F->hnorm[((size_t) sg * SOLVE_NRHS + q) * 2], 8);
          memcpy(&xn, &F->hnorm[((size_t) sg * SOLVE_NRHS + q) * 2 + 1], 8);
          if (it == 0) bnorm[(size_t) sg * nq + q] = rn;   // X = 0: r = b
          const double den = anorm[sg] * xn + bnorm[(size_t) sg * nq + q];
          const double rq = den > 0 ? rn / den : 0.0;
          if (res) res[(size_t) sg * nrhs + q0 + q] = rq;
          worst = std::max(worst, rq);
        }
      if (it > 0 && worst <= tol) break;
      if (it > 0) {
        if (worst > 0.5 * prev_worst) slow++;
        else slow = 0;
        if (!use64 && (slow >= 2 || steps >= maxits)) {
          // refinement stalled with the FP32 factor: first preconditioned
          // conjugate gradients on that factor (one system only), then an
          // FP64 refactorization
          if (ns == 1 && F->pcg_maxits > 0) {
            tprintf("\t\trefinement stalled at %.3e after %d steps; PCG on the FP32 factor\n", worst, steps);
            std::vector<double> rq(nq, 0.0);
            const int its = pcg_fp32(F, nq, X, B, ld, tol, anorm[0], bnorm.data(), rq.data());
            if (its == -2) return -1;
            if (res)
              for (int q = 0; q < nq; q++) res[q0 + q] = rq[q];
            F->last_pcg_its += std::max(its, 0);
            if (its >= 0) {
              F->last_fallback = std::max(F->last_fallback, 1);
              steps += its;
              done = true;
              continue;
            }
            tprintf("\t\tPCG did not reach the tolerance (stalled, or %d iterations)\n", F->pcg_maxits);
          }
          tprintf("\t\trefinement stalled at %.3e after %d steps; refactoring in FP64\n", worst, steps);
          if (!F->has_numeric && numeric_fp64_device(F, F->dvals_cur, true)) return -1;
          F->last_fallback = 2;
          use64 = true;
          slow = 0;
        } else if (use64 && (slow >= 2 || steps >= maxits + 5)) {
          done = true;
          total = -1;
          continue;
        }
      }
      prev_worst = worst;
      const bool u64 = use64;
      if (run_graphed(F, GraphKey{u64 ? 5u : 4u, (uint64_t) nq, (uint64_t) X, (uint64_t) B, (uint64_t) ld, 0}, st,
                      [&](cudaStream_t s) { return correction(s, u64); }))
        return -1;
      steps++;
    }
    if (total >= 0) total = std::max(total, steps);
  }
  return total;
}

// ||A||_inf of the factored values per segment, computed on the device
static int device_anorm(Factor* F, std::vector<double>* anorm) {
  cudaStream_t st = current_stream();
  const int ns = F->nseg();
  cudaMemsetAsync(F->dnorm, 0, sizeof(unsigned long long) * ns, st);
  k_anorm<<<nblk(F->n, 256), 256, 0, st>>>(F->n, F->dcsr_ptr, F->dcsr_val, F->dvals_cur, F->dseg, F->dnorm);
  count_launch();
  cudaMemcpyAsync(F->hnorm, F->dnorm, sizeof(unsigned long long) * ns, cudaMemcpyDeviceToHost, st);
  if (!cuda_ok(cudaStreamSynchronize(st), "norm")) return -1;
  anorm->resize(ns);
  for (int s = 0; s < ns; s++) memcpy(&(*anorm)[s], &F->hnorm[s], 8);
  return 0;
}

int gather_values_device(long nnz, const int* d_vmap, const double* d_raw, double* d_out) {
  if (nnz <= 0) return 0;
  const int grid = (int) std::min<long>(nblk(nnz, 256), 148L * 16);
  k_gather_values<<<grid, 256, 0, current_stream()>>>(nnz, d_vmap, d_raw, d_out);
  count_launch();
  return cuda_ok(cudaGetLastError(), "value gather") ? 0 : -1;
}

int perm_gather_device(int n, const int* d_perm, const double* src, double* dst) {
  if (n <= 0) return 0;
  k_perm_gather<<<nblk(n, 256), 256, 0, current_stream()>>>(n, 1, d_perm, src, dst);
  count_launch();
  return cuda_ok(cudaGetLastError(), "permutation") ? 0 : -1;
}

int perm_scatter_device(int n, const int* d_perm, const double* src, double* dst) {
  if (n <= 0) return 0;
  k_perm_scatter<<<nblk(n, 256), 256, 0, current_stream()>>>(n, 1, d_perm, src, dst);
  count_launch();
  return cuda_ok(cudaGetLastError(), "permutation") ? 0 : -1;
}

int solve_refine_permuted(Factor* F, int nrhs, double* d_x, const double* d_b, const int* d_perm, double tol,
                          int maxits, double* res) {
  if (!F || (!F->has_numeric && !F->has_numeric32)) { set_error("solve_refine: no numeric factor"); return -1; }
  if (F->nseg() > 1) { set_error("solve_refine: a batch handle solves through taucs_b200_batch_solve"); return -1; }
  if (ensure_refine(F)) return -1;
  const int n = F->n;
  std::vector<double> anorm;
  if (device_anorm(F, &anorm)) return -1;
  cudaStream_t st = current_stream();
  int worst_steps = 0;
  for (int q0 = 0; q0 < nrhs; q0 += SOLVE_NRHS) {
    const int nq = std::min(SOLVE_NRHS, nrhs - q0);
    k_perm_gather<<<nblk(n, 256), 256, 0, st>>>(n, nq, d_perm, d_b + (size_t) q0 * n, F->dBr);
    count_launch();
    const int s = refine_device(F, nq, F->dXr, F->dBr, n, tol, maxits, anorm, res ? res + q0 : nullptr);
    k_perm_scatter<<<nblk(n, 256), 256, 0, st>>>(n, nq, d_perm, F->dXr, d_x + (size_t) q0 * n);
    count_launch();
    if (!cuda_ok(cudaGetLastError(), "permute")) return -1;
    if (s < 0) worst_steps = -1;
    else if (worst_steps >= 0) worst_steps = std::max(worst_steps, s);
  }
  return worst_steps;
}

int solve_refine_device(Factor* F, int nrhs, double* dX, const double* dB, int ld, double tol, int maxits,
                        double* res) {
  if (!F || (!F->has_numeric && !F->has_numeric32)) { set_error("solve_refine: no numeric factor"); return -1; }
  if (ensure_refine(F)) return -1;
  std::vector<double> anorm;
  if (device_anorm(F, &anorm)) return -1;
  return refine_device(F, nrhs, dX, dB, ld, tol, maxits, anorm, res);
}

int solve_refine_host(Factor* F, taucs_ccs_matrix* A, int nrhs, double* X, const double* B, double tol, int maxits,
                      double* res) {
  if (!F || (!F->has_numeric && !F->has_numeric32)) { set_error("solve_refine: no numeric factor"); return -1; }
  if (F->nseg() > 1) { set_error("solve_refine: a batch handle solves through taucs_b200_batch_solve"); return -1; }
  if (ensure_refine(F)) return -1;
  const int n = F->n;
  // A, when given, has the factored pattern and values; the norm comes from
  // the device copy
  (void) A;
  std::vector<double> anorm;
  if (device_anorm(F, &anorm)) return -1;
  cudaStream_t st = current_stream();
  int worst_steps = 0;
  for (int q0 = 0; q0 < nrhs; q0 += SOLVE_NRHS) {
    const int nq = std::min(SOLVE_NRHS, nrhs - q0);
    if (!cuda_ok(cudaMemcpyAsync(F->dBr, B + (size_t) q0 * n, sizeof(double) * (size_t) n * nq, cudaMemcpyHostToDevice, st), "rhs"))
      return -1;
    const int s = refine_device(F, nq, F->dXr, F->dBr, n, tol, maxits, anorm, res ? res + q0 : nullptr);
    if (!cuda_ok(cudaMemcpyAsync(X + (size_t) q0 * n, F->dXr, sizeof(double) * (size_t) n * nq, cudaMemcpyDeviceToHost, st), "x"))
      return -1;
    if (!cuda_ok(cudaStreamSynchronize(st), "solve_refine")) return -1;
    if (s < 0) worst_steps = -1;
    else if (worst_steps >= 0) worst_steps = std::max(worst_steps, s);
  }
  return worst_steps;
}

}  // namespace tb

using namespace tb;

extern "C" int taucs_b200_set_precision(void* L, int precision) {
  if (!L || (precision != 0 && precision != 1)) return -1;
  ((Factor*) L)->precision = precision;
  return 0;
}

extern "C" int taucs_b200_set_split_format(void* L, int fmt) {
  if (!L || fmt < 0 || fmt > 1) return -1;
  Factor* F = (Factor*) L;
  if (F->sp_fmt != fmt) drop_graphs(F);
  F->sp_fmt = fmt;
  return 0;
}

extern "C" int taucs_b200_set_refinement(void* L, int method) {
  if (!L || method < 0 || method > 1) return -1;
  ((Factor*) L)->refine_method = method;
  return 0;
}

extern "C" int taucs_b200_set_pcg(void* L, int maxits) {
  if (!L || maxits < 0) return -1;
  ((Factor*) L)->pcg_maxits = maxits;
  return 0;
}

extern "C" int taucs_b200_refine_report(void* L, int* fallback, int* pcg_iterations) {
  if (!L) return -1;
  if (fallback) *fallback = ((Factor*) L)->last_fallback;
  if (pcg_iterations) *pcg_iterations = ((Factor*) L)->last_pcg_its;
  return 0;
}

extern "C" int taucs_b200_solve_refine_device(void* L, int nrhs, double* d_X, const double* d_B, int ld, double tol,
                                              int maxits, double* res_out) {
  if (!L || nrhs < 0 || (nrhs > 0 && (!d_X || !d_B))) return -1;
  if (nrhs == 0) return 0;
  Factor* F = (Factor*) L;
  if (ld < F->n) { set_error("taucs_b200_solve_refine_device: ld < n"); return -1; }
  return solve_refine_device(F, nrhs, d_X, d_B, ld, tol, maxits < 0 ? 0 : maxits, res_out);
}

extern "C" int taucs_b200_solve_refine(void* L, taucs_ccs_matrix* A, int nrhs, double* X, const double* B,
                                       double tol, int maxits, double* res_out) {
  if (!L || nrhs < 0 || (nrhs > 0 && (!X || !B))) return -1;
  if (nrhs == 0) return 0;
  return solve_refine_host((Factor*) L, A, nrhs, X, B, tol, maxits < 0 ? 0 : maxits, res_out);
}

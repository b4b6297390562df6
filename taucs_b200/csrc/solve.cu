// FP64 supernodal triangular solve on sm_100a, level scheduled.
//
// The reference solves one right-hand side per call by recursion
// (src/taucs_sn_llt.c:2596-2885): forward in postorder -- gather b at the
// supernode's columns, TRSM with L11, GEMM with L21, scatter-subtract into b
// at the update rows -- and backward in preorder with L21^T and L11^T.
//
// Here the forward pass is written multifrontally so that no two CTAs ever
// write the same vector entry: each front owns a work vector of f entries
// per right-hand side (W, at the front's row offset).  A front's forward step
// gathers b at its columns, adds its children's update vectors (their W rows
// s..f-1) through the child->parent maps in the fixed child order, solves
// with L11 and leaves y in W[0..s) and the update vector u = w2 - L21 y in
// W[s..f).  The backward pass runs the levels in reverse: gather x at the
// update rows (written by ancestors in earlier launches), r = y - L21^T x2,
// then the L11^T substitution, and scatter x at the columns.  Up to
// SOLVE_NRHS right-hand sides share every read of L.
#include "kernels.h"

namespace tb {

namespace {

constexpr int SB = 32;   // substitution block (one warp)

__global__ void __launch_bounds__(256)
k_fwd(int fbegin, const FrontDesc* __restrict__ fronts, const int* __restrict__ children,
      const int* __restrict__ maps, const int* __restrict__ rows, const double* __restrict__ L,
      const double* __restrict__ B, int ldb, double* __restrict__ W, int nrhs) {
  __shared__ double xs[SB][SOLVE_NRHS];
  const FrontDesc F = fronts[fbegin + blockIdx.x];
  const int f = F.f, s = F.s;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  double* Wf = W + F.v_off * SOLVE_NRHS;
  const int* rw = rows + F.rows_off;
  const double* P = L + F.l_off;

  for (int k = tid; k < f * nrhs; k += nt) {
    const int r = k % f, q = k / f;
    Wf[k] = (r < s) ? B[rw[r] + (size_t) q * ldb] : 0.0;
  }
  __syncthreads();
  for (int ci = F.child_begin; ci < F.child_end; ci++) {
    const FrontDesc C = fronts[children[ci]];
    const int mc = C.f - C.s;
    const int* mp = maps + C.map_off;
    const double* Wc = W + C.v_off * SOLVE_NRHS;
    for (int k = tid; k < mc * nrhs; k += nt) {
      const int i = k % mc, q = k / mc;
      Wf[mp[i] + q * f] += Wc[C.s + i + q * C.f];
    }
    __syncthreads();
  }
  for (int jb = 0; jb < s; jb += SB) {
    const int bw = min(SB, s - jb);
    if (warp == 0) {
      for (int q = 0; q < nrhs; q++) {
        double v = (lane < bw) ? Wf[jb + lane + q * f] : 0.0;
        for (int j = 0; j < bw; j++) {
          const double xj = __shfl_sync(0xffffffffu, v, j) / P[(jb + j) + (size_t) (jb + j) * f];
          if (lane == j) v = xj;
          if (lane > j && lane < bw) v -= P[(jb + lane) + (size_t) (jb + j) * f] * xj;
        }
        if (lane < bw) {
          Wf[jb + lane + q * f] = v;
          xs[lane][q] = v;
        }
      }
    }
    __syncthreads();
    for (int r = jb + bw + tid; r < f; r += nt) {
      double acc[SOLVE_NRHS];
#pragma unroll
      for (int q = 0; q < SOLVE_NRHS; q++) acc[q] = 0.0;
      for (int j = 0; j < bw; j++) {
        const double l = P[r + (size_t) (jb + j) * f];
#pragma unroll
        for (int q = 0; q < SOLVE_NRHS; q++)
          if (q < nrhs) acc[q] += l * xs[j][q];
      }
      for (int q = 0; q < nrhs; q++) Wf[r + q * f] -= acc[q];
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256)
k_bwd(int fbegin, const FrontDesc* __restrict__ fronts, const int* __restrict__ rows,
      const double* __restrict__ L, double* __restrict__ X, int ldx, double* __restrict__ W,
      int nrhs) {
  __shared__ double xs[SB][SOLVE_NRHS];
  const FrontDesc F = fronts[fbegin + blockIdx.x];
  const int f = F.f, s = F.s;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  double* Wf = W + F.v_off * SOLVE_NRHS;
  const int* rw = rows + F.rows_off;
  const double* P = L + F.l_off;

  // x at the update rows (final: written by ancestors)
  for (int k = tid; k < (f - s) * nrhs; k += nt) {
    const int i = k % (f - s), q = k / (f - s);
    Wf[s + i + q * f] = X[rw[s + i] + (size_t) q * ldx];
  }
  __syncthreads();
  // r_j = y_j - sum_{i >= s} L[i,j] x_i
  for (int j = warp; j < s; j += nw) {
    double acc[SOLVE_NRHS];
#pragma unroll
    for (int q = 0; q < SOLVE_NRHS; q++) acc[q] = 0.0;
    const double* pj = P + (size_t) j * f;
    for (int i = s + lane; i < f; i += 32) {
      const double l = pj[i];
#pragma unroll
      for (int q = 0; q < SOLVE_NRHS; q++)
        if (q < nrhs) acc[q] += l * Wf[i + q * f];
    }
#pragma unroll
    for (int q = 0; q < SOLVE_NRHS; q++) {
      double v = acc[q];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      acc[q] = v;
    }
    if (lane == 0)
      for (int q = 0; q < nrhs; q++) Wf[j + q * f] -= acc[q];
  }
  __syncthreads();
  // L11^T substitution, blocks from the end
  const int nblk = (s + SB - 1) / SB;
  for (int b = nblk - 1; b >= 0; b--) {
    const int jb = b * SB, bw = min(SB, s - jb), je = jb + bw;
    // contributions of the already solved x in rows [je, s)
    if (je < s) {
      for (int j = jb + warp; j < je; j += nw) {
        double acc[SOLVE_NRHS];
#pragma unroll
        for (int q = 0; q < SOLVE_NRHS; q++) acc[q] = 0.0;
        const double* pj = P + (size_t) j * f;
        for (int i = je + lane; i < s; i += 32) {
          const double l = pj[i];
#pragma unroll
          for (int q = 0; q < SOLVE_NRHS; q++)
            if (q < nrhs) acc[q] += l * Wf[i + q * f];
        }
#pragma unroll
        for (int q = 0; q < SOLVE_NRHS; q++) {
          double v = acc[q];
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          acc[q] = v;
        }
        if (lane == 0)
          for (int q = 0; q < nrhs; q++) Wf[j + q * f] -= acc[q];
      }
      __syncthreads();
    }
    if (warp == 0) {
      for (int q = 0; q < nrhs; q++) {
        double v = (lane < bw) ? Wf[jb + lane + q * f] : 0.0;
        for (int j = bw - 1; j >= 0; j--) {
          const double xj = __shfl_sync(0xffffffffu, v, j) / P[(jb + j) + (size_t) (jb + j) * f];
          if (lane == j) v = xj;
          if (lane < j) v -= P[(jb + j) + (size_t) (jb + lane) * f] * xj;
        }
        if (lane < bw) xs[lane][q] = v;
      }
    }
    __syncthreads();
    for (int k = tid; k < bw * nrhs; k += nt) {
      const int l = k % bw, q = k / bw;
      Wf[jb + l + q * f] = xs[l][q];
    }
    __syncthreads();
  }
  for (int k = tid; k < s * nrhs; k += nt) {
    const int r = k % s, q = k / s;
    X[rw[r] + (size_t) q * ldx] = Wf[r + q * f];
  }
}

}  // namespace

int launch_solve_fp64(const Plan& P, const DevPlan& D, const double* L, int nrhs, double* X,
                      const double* B, int ld, double* W, double* Y, cudaStream_t st) {
  (void) Y;
  for (int q0 = 0; q0 < nrhs; q0 += SOLVE_NRHS) {
    const int nq = std::min(SOLVE_NRHS, nrhs - q0);
    const double* Bq = B + (size_t) q0 * ld;
    double* Xq = X + (size_t) q0 * ld;
    for (int h = 0; h < P.n_levels; h++) {
      const LevelPlan& LP = P.levels[h];
      const int cnt = LP.front_end - LP.front_begin;
      if (cnt <= 0) continue;
      k_fwd<<<cnt, 256, 0, st>>>(LP.front_begin, D.fronts, D.children, D.maps, D.rows, L, Bq, ld, W, nq);
      count_launch();
    }
    for (int h = P.n_levels - 1; h >= 0; h--) {
      const LevelPlan& LP = P.levels[h];
      const int cnt = LP.front_end - LP.front_begin;
      if (cnt <= 0) continue;
      k_bwd<<<cnt, 256, 0, st>>>(LP.front_begin, D.fronts, D.rows, L, Xq, ld, W, nq);
      count_launch();
    }
  }
  return (int) cudaGetLastError();
}

}  // namespace tb

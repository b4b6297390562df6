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
#include <mutex>
#include <type_traits>

#include "factor.h"
#include "kernels.h"

namespace tb {

namespace {

constexpr int SB = 32;   // substitution block (one warp)

// Small fronts: G threads per front (256: one CTA; 32: one warp, eight
// fronts per CTA for the many tiny fronts near the leaves).  The threads of
// one front synchronise among themselves only.
template <int G>
__device__ __forceinline__ void group_sync() {
  if (G == 32) __syncwarp();
  else __syncthreads();
}

// forward step of one small front by a group of G threads; xs: the group's
// shared staging of one substitution block
template <typename T, int WS, int G>
__device__ void fwd_small(const FrontDesc& F, const FrontDesc* __restrict__ fronts, const int* __restrict__ children,
                          const int* __restrict__ maps, const int* __restrict__ rows, const T* __restrict__ L,
                          const T* __restrict__ B, int ldb, T* __restrict__ W, int nrhs,
                          T (&xs)[SB][SOLVE_NRHS]) {
  const int f = F.f, s = F.s;
  const int tid = threadIdx.x % G, nt = G, lane = tid & 31, warp = tid >> 5;
  T* Wf = W + F.v_off * WS;
  const int* rw = rows + F.rows_off;
  const T* P = L + F.l_off;

  for (int k = tid; k < f * nrhs; k += nt) {
    const int r = k % f, q = k / f;
    Wf[k] = (r < s) ? B[rw[r] + (size_t) q * ldb] : 0.0;
  }
  group_sync<G>();
  for (int ci = F.child_begin; ci < F.child_end; ci++) {
    const FrontDesc C = fronts[children[ci]];
    const int mc = C.f - C.s;
    const int* mp = maps + C.map_off;
    const T* Wc = W + C.v_off * WS;
    for (int k = tid; k < mc * nrhs; k += nt) {
      const int i = k % mc, q = k / mc;
      Wf[mp[i] + q * f] += Wc[C.s + i + q * C.f];
    }
    group_sync<G>();
  }
  for (int jb = 0; jb < s; jb += SB) {
    const int bw = min(SB, s - jb);
    if (warp == 0) {
      // all right-hand sides advance together through one substitution chain
      const T rd = (lane < bw) ? T(1) / P[(jb + lane) + (size_t) (jb + lane) * f] : T(0);
      T v[SOLVE_NRHS];
#pragma unroll
      for (int q = 0; q < SOLVE_NRHS; q++) v[q] = (q < nrhs && lane < bw) ? Wf[jb + lane + q * f] : T(0);
      for (int j = 0; j < bw; j++) {
        const T rj = __shfl_sync(0xffffffffu, rd, j);
        const T l = (lane > j && lane < bw) ? P[(jb + lane) + (size_t) (jb + j) * f] : T(0);
#pragma unroll
        for (int q = 0; q < SOLVE_NRHS; q++) {
          if (q < nrhs) {
            const T xj = __shfl_sync(0xffffffffu, v[q], j) * rj;
            if (lane == j) v[q] = xj;
            else v[q] -= l * xj;
          }
        }
      }
      if (lane < bw) {
#pragma unroll
        for (int q = 0; q < SOLVE_NRHS; q++)
          if (q < nrhs) {
            Wf[jb + lane + q * f] = v[q];
            xs[lane][q] = v[q];
          }
      }
    }
    group_sync<G>();
    for (int r = jb + bw + tid; r < f; r += nt) {
      T acc[SOLVE_NRHS];
#pragma unroll
      for (int q = 0; q < SOLVE_NRHS; q++) acc[q] = 0.0;
      for (int j = 0; j < bw; j++) {
        const T l = P[r + (size_t) (jb + j) * f];
#pragma unroll
        for (int q = 0; q < SOLVE_NRHS; q++)
          if (q < nrhs) acc[q] += l * xs[j][q];
      }
#pragma unroll
      for (int q = 0; q < SOLVE_NRHS; q++)
        if (q < nrhs) Wf[r + q * f] -= acc[q];
    }
    group_sync<G>();
  }
}

template <typename T, int WS, int G>
__global__ void __launch_bounds__(256)
k_fwd(const int* __restrict__ list, int count, const FrontDesc* __restrict__ fronts, const int* __restrict__ children,
      const int* __restrict__ maps, const int* __restrict__ rows, const T* __restrict__ L,
      const T* __restrict__ B, int ldb, T* __restrict__ W, int nrhs) {
  constexpr int GPC = 256 / G;   // fronts per CTA: one per group of G threads
  __shared__ T xs_all[GPC][SB][SOLVE_NRHS];
  const int grp = threadIdx.x / G, li = blockIdx.x * GPC + grp;
  if (li >= count) return;
  fwd_small<T, WS, G>(fronts[list[li]], fronts, children, maps, rows, L, B, ldb, W, nrhs, xs_all[grp]);
}

// backward step of one small front by a group of G threads
template <typename T, int WS, int G>
__device__ void bwd_small(const FrontDesc& F, const int* __restrict__ rows, const T* __restrict__ L,
                          T* __restrict__ X, int ldx, T* __restrict__ W, int nrhs, T (&xs)[SB][SOLVE_NRHS]) {
  const int f = F.f, s = F.s;
  const int tid = threadIdx.x % G, nt = G, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  T* Wf = W + F.v_off * WS;
  const int* rw = rows + F.rows_off;
  const T* P = L + F.l_off;

  // x at the update rows (final: written by ancestors)
  for (int k = tid; k < (f - s) * nrhs; k += nt) {
    const int i = k % (f - s), q = k / (f - s);
    Wf[s + i + q * f] = X[rw[s + i] + (size_t) q * ldx];
  }
  group_sync<G>();
  // r_j = y_j - sum_{i >= s} L[i,j] x_i
  for (int j = warp; j < s; j += nw) {
    T acc[SOLVE_NRHS];
#pragma unroll
    for (int q = 0; q < SOLVE_NRHS; q++) acc[q] = 0.0;
    const T* pj = P + (size_t) j * f;
    for (int i = s + lane; i < f; i += 32) {
      const T l = pj[i];
#pragma unroll
      for (int q = 0; q < SOLVE_NRHS; q++)
        if (q < nrhs) acc[q] += l * Wf[i + q * f];
    }
#pragma unroll
    for (int q = 0; q < SOLVE_NRHS; q++) {
      T v = acc[q];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      acc[q] = v;
    }
    if (lane == 0) {
#pragma unroll
      for (int q = 0; q < SOLVE_NRHS; q++)
        if (q < nrhs) Wf[j + q * f] -= acc[q];
    }
  }
  group_sync<G>();
  // L11^T substitution, blocks from the end
  const int nblk = (s + SB - 1) / SB;
  for (int b = nblk - 1; b >= 0; b--) {
    const int jb = b * SB, bw = min(SB, s - jb), je = jb + bw;
    // contributions of the already solved x in rows [je, s)
    if (je < s) {
      for (int j = jb + warp; j < je; j += nw) {
        T acc[SOLVE_NRHS];
#pragma unroll
        for (int q = 0; q < SOLVE_NRHS; q++) acc[q] = 0.0;
        const T* pj = P + (size_t) j * f;
        for (int i = je + lane; i < s; i += 32) {
          const T l = pj[i];
#pragma unroll
          for (int q = 0; q < SOLVE_NRHS; q++)
            if (q < nrhs) acc[q] += l * Wf[i + q * f];
        }
#pragma unroll
        for (int q = 0; q < SOLVE_NRHS; q++) {
          T v = acc[q];
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          acc[q] = v;
        }
        if (lane == 0) {
#pragma unroll
          for (int q = 0; q < SOLVE_NRHS; q++)
            if (q < nrhs) Wf[j + q * f] -= acc[q];
        }
      }
      group_sync<G>();
    }
    if (warp == 0) {
      const T rd = (lane < bw) ? T(1) / P[(jb + lane) + (size_t) (jb + lane) * f] : T(0);
      T v[SOLVE_NRHS];
#pragma unroll
      for (int q = 0; q < SOLVE_NRHS; q++) v[q] = (q < nrhs && lane < bw) ? Wf[jb + lane + q * f] : T(0);
      for (int j = bw - 1; j >= 0; j--) {
        const T rj = __shfl_sync(0xffffffffu, rd, j);
        const T l = (lane < j) ? P[(jb + j) + (size_t) (jb + lane) * f] : T(0);
#pragma unroll
        for (int q = 0; q < SOLVE_NRHS; q++) {
          if (q < nrhs) {
            const T xj = __shfl_sync(0xffffffffu, v[q], j) * rj;
            if (lane == j) v[q] = xj;
            else v[q] -= l * xj;
          }
        }
      }
      if (lane < bw) {
#pragma unroll
        for (int q = 0; q < SOLVE_NRHS; q++)
          if (q < nrhs) xs[lane][q] = v[q];
      }
    }
    group_sync<G>();
    for (int k = tid; k < bw * nrhs; k += nt) {
      const int l = k % bw, q = k / bw;
      Wf[jb + l + q * f] = xs[l][q];
    }
    group_sync<G>();
  }
  for (int k = tid; k < s * nrhs; k += nt) {
    const int r = k % s, q = k / s;
    X[rw[r] + (size_t) q * ldx] = Wf[r + q * f];
  }
}

template <typename T, int WS, int G>
__global__ void __launch_bounds__(256)
k_bwd(const int* __restrict__ list, int count, const FrontDesc* __restrict__ fronts, const int* __restrict__ rows,
      const T* __restrict__ L, T* __restrict__ X, int ldx, T* __restrict__ W,
      int nrhs) {
  constexpr int GPC = 256 / G;
  __shared__ T xs_all[GPC][SB][SOLVE_NRHS];
  const int grp = threadIdx.x / G, li = blockIdx.x * GPC + grp;
  if (li >= count) return;
  bwd_small<T, WS, G>(fronts[list[li]], rows, L, X, ldx, W, nrhs, xs_all[grp]);
}

__device__ __forceinline__ int ld_acquire_i(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// One-warp form of the backward small-front step for the persistent launch
// (fronts of order f <= SMALL_F_MAX): the front's vector is kept in the
// warp's shared rows ws[nrhs][f]; each lane holds the L entries it needs for
// the substitution chain in registers, loaded together (in groups of eight,
// as far as the block is wide) before the arithmetic, so that the chain
// waits for memory once per 32-column block instead of once per column.
// (The same form of the forward step measured slower than fwd_small.)
constexpr int PW_SLOTS = (SMALL_F_MAX + 31) / 32;   // rows per lane

// backward step of one small front by one warp: x at the update rows, then
// per diagonal block from the last: r = y - L[below, block]^T x_below (lane
// j takes column jb + j, the rows in batches of eight loads), and the L11^T
// substitution chain from registers
template <typename T, int WS>
__device__ void bwd_warp(const FrontDesc& F, const int* __restrict__ rows, const T* __restrict__ L,
                         T* __restrict__ X, int ldx, const T* __restrict__ W, int nrhs, T (*ws)[SMALL_F_MAX]) {
  constexpr unsigned FULL = 0xffffffffu;
  const int f = F.f, s = F.s, lane = threadIdx.x & 31;
  const T* Wf = W + F.v_off * WS;
  const int* rw = rows + F.rows_off;
  const T* P = L + F.l_off;
  {
    int g[PW_SLOTS];
#pragma unroll
    for (int sl = 0; sl < PW_SLOTS; sl++) {
      const int r = lane + 32 * sl;
      g[sl] = (r >= s && r < f) ? __ldg(rw + r) : -1;
    }
#pragma unroll
    for (int q = 0; q < SOLVE_NRHS; q++) {
      if (q >= nrhs) break;
      T v[PW_SLOTS];
#pragma unroll
      for (int sl = 0; sl < PW_SLOTS; sl++) {
        const int r = lane + 32 * sl;
        v[sl] = g[sl] >= 0 ? X[g[sl] + (size_t) q * ldx] : r < s ? Wf[r + q * f] : T(0);
      }
#pragma unroll
      for (int sl = 0; sl < PW_SLOTS; sl++)
        if (lane + 32 * sl < f) ws[q][lane + 32 * sl] = v[sl];
    }
  }
  __syncwarp();
  const int nblk = (s + SB - 1) / SB;
  for (int b = nblk - 1; b >= 0; b--) {
    const int jb = b * SB, bw = min(SB, s - jb), je = jb + bw;
    const bool own = lane < bw;
    const T* pj = P + (size_t) (jb + lane) * f;
    // the solved rows below the block: x in rows [je, f)
    T acc[SOLVE_NRHS];
#pragma unroll
    for (int q = 0; q < SOLVE_NRHS; q++) acc[q] = T(0);
    for (int i0 = je; i0 < f; i0 += 8) {
      T l[8];
#pragma unroll
      for (int u = 0; u < 8; u++) l[u] = (own && i0 + u < f) ? pj[i0 + u] : T(0);
#pragma unroll
      for (int u = 0; u < 8; u++) {
        if (i0 + u >= f) break;
#pragma unroll
        for (int q = 0; q < SOLVE_NRHS; q++)
          if (q < nrhs) acc[q] += l[u] * ws[q][i0 + u];
      }
    }
    // lane l: column jb + l of the diagonal block
    T lc[SB];
#pragma unroll
    for (int k0 = 0; k0 < SB; k0 += 8) {
      if (k0 >= bw) break;
#pragma unroll
      for (int k = k0; k < k0 + 8; k++) lc[k] = (own && k > lane && k < bw) ? pj[jb + k] : T(0);
    }
    const T rd = own ? T(1) / pj[jb + lane] : T(0);
    T v[SOLVE_NRHS];
#pragma unroll
    for (int q = 0; q < SOLVE_NRHS; q++) v[q] = (q < nrhs && own) ? ws[q][jb + lane] - acc[q] : T(0);
#pragma unroll
    for (int j = SB - 1; j >= 0; j--) {
      if (j >= bw) continue;
      const T rj = __shfl_sync(FULL, rd, j);
#pragma unroll
      for (int q = 0; q < SOLVE_NRHS; q++) {
        if (q >= nrhs) break;
        const T xj = __shfl_sync(FULL, v[q], j) * rj;
        if (lane == j) v[q] = xj;
        else v[q] -= lc[j] * xj;
      }
    }
    if (own)
#pragma unroll
      for (int q = 0; q < SOLVE_NRHS; q++)
        if (q < nrhs) ws[q][jb + lane] = v[q];
    __syncwarp();
  }
#pragma unroll
  for (int sl = 0; sl < PW_SLOTS; sl++) {
    const int r = lane + 32 * sl;
    if (r < s) {
      const int g = __ldg(rw + r);
#pragma unroll
      for (int q = 0; q < SOLVE_NRHS; q++)
        if (q < nrhs) X[g + (size_t) q * ldx] = ws[q][r];
    }
  }
}

// The small fronts with only small fronts below them (Plan::pers_fronts), in
// one launch per direction; each warp takes the next front from a device-
// side queue.  Forward, in level order: a front waits until its children's
// update vectors are in place (pending count), and counts itself off at its
// parent.  Backward, in reverse level order: a front waits until its parent
// has written x at its update rows (done flag = epoch; parents outside the
// set ran in the level launches before this one).  Every wait is bounded
// (SOLVE_TIMEOUT).
template <typename T, int WS>
__global__ void __launch_bounds__(256)
k_fwd_pers(const int* __restrict__ tasks, int ntask, const int* __restrict__ parent_task, int* pending, int* next,
           const FrontDesc* __restrict__ fronts, const int* __restrict__ children, const int* __restrict__ maps,
           const int* __restrict__ rows, const T* __restrict__ L, const T* __restrict__ B, int ldb,
           T* __restrict__ W, int nrhs, int* status) {
  __shared__ T xs_all[8][SB][SOLVE_NRHS];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(next, 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= ntask) break;
    if (lane == 0) {
      int it = 0;
      while (ld_acquire_i(pending + t) != 0) {
        if (++it > (1 << 22)) {
          atomicExch(status, SOLVE_TIMEOUT);
          break;
        }
        __nanosleep(32);
      }
    }
    __syncwarp();
    fwd_small<T, WS, 32>(fronts[tasks[t]], fronts, children, maps, rows, L, B, ldb, W, nrhs, xs_all[wi]);
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      const int pt = parent_task[t];
      if (pt >= 0) atomicSub(pending + pt, 1);
    }
  }
}

template <typename T, int WS>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 2)
k_bwd_pers(const int* __restrict__ tasks, int ntask, const int* __restrict__ parent_task, int* done, int* next,
           int epoch, const FrontDesc* __restrict__ fronts, const int* __restrict__ rows, const T* __restrict__ L,
           T* __restrict__ X, int ldx, T* __restrict__ W, int nrhs, int* status) {
  __shared__ T ws_all[8][SOLVE_NRHS][SMALL_F_MAX];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  for (;;) {
    int q = 0;
    if (lane == 0) q = atomicAdd(next, 1);
    q = __shfl_sync(0xffffffffu, q, 0);
    if (q >= ntask) break;
    const int t = ntask - 1 - q;
    const int pt = parent_task[t];
    if (lane == 0 && pt >= 0) {
      int it = 0;
      while (ld_acquire_i(done + pt) != epoch) {
        if (++it > (1 << 22)) {
          atomicExch(status, SOLVE_TIMEOUT);
          break;
        }
        __nanosleep(32);
      }
    }
    __syncwarp();
    bwd_warp<T, WS>(fronts[tasks[t]], rows, L, X, ldx, W, nrhs, ws_all[wi]);
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      atomicExch(done + t, epoch);
    }
  }
}


// ---------------------------------------------------------------- big fronts
// One CTA per 64-row block.  Forward: block r waits for the solved blocks
// k < r of L11 (flags, release/acquire), accumulates L[r,k] y_k, then solves
// its own diagonal block and publishes y_r.  Backward: blocks run from the
// last one; block k waits for x_j, j > k.  Waits are bounded: on timeout the
// CTA records SOLVE_TIMEOUT in the status word and carries on, so no launch
// can hang.

constexpr int BR = PANEL_NB;   // rows per block
// dynamic shared memory: L_kk^-1, plus one staged 64x64 block of L11 for 8
// columns
template <typename T, int NQ>
constexpr size_t bwd_smem() { return (NQ >= 8 ? 2 : 1) * BR * (BR + 1) * sizeof(T); }

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

}  // namespace

// Controls of the handshake waits on this device: the polling limit, and an
// offset added to the flag value waited for (0; any other value makes every
// wait run out -- a testing aid for the timeout reporting, set through
// taucs_b200_debug_waits).
__device__ int g_solve_wait_limit = 1 << 22;
__device__ int g_solve_wait_skew = 0;

int solve_set_wait_controls(int limit, int skew) {
  cudaError_t e = cudaMemcpyToSymbol(g_solve_wait_limit, &limit, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_solve_wait_skew, &skew, sizeof(int));
  return (int) e;
}

namespace {

// polls flag until it holds epoch (plus the wait offset); on giving up,
// records SOLVE_TIMEOUT
__device__ __forceinline__ void poll_epoch(const int* flag, int epoch, int* status) {
  const int want = epoch + g_solve_wait_skew, limit = g_solve_wait_limit;
  int it = 0;
  while (ld_acquire(flag) != want) {
    // a wait that gave up anywhere ends the others at once, so a broken
    // chain costs one polling limit, not one per wait
    if (++it > limit || ((it & 1023) == 0 && *(volatile int*) status == SOLVE_TIMEOUT)) {
      atomicExch(status, SOLVE_TIMEOUT);
      break;
    }
    __nanosleep(32);
  }
}

// the same wait for one warp: lane 0 polls, the warp follows it
__device__ void wait_epoch_warp(const int* flag, int epoch, int* status) {
  if ((threadIdx.x & 31) == 0) poll_epoch(flag, epoch, status);
  __syncwarp();   // orders the lanes' later loads after lane 0's acquire
}

__device__ void wait_epoch(const int* flag, int epoch, int* status) {
  if (threadIdx.x == 0) poll_epoch(flag, epoch, status);
  __syncthreads();
}


// Forward solve of big fronts.  Diagonal block r of L11 gives
// y_r = L_rr^-1 (w_r - sum_{k<r} L_rk y_k), chained to block r-1 by
// release/acquire flags; update rows i get w_i - sum_k L_ik y_k.
//   FWD_ALL   one launch over all blocks of a level: every block waits for
//             the blocks k it needs, one at a time (short chains);
//   FWD_CHAIN the diagonal blocks of a level with long chains: everything
//             but the last term is done before waiting -- M = L_rr^-1
//             L_{r,r-1} at kernel start, the sum over k < r-1 and
//             c = L_rr^-1 (w_r - ...) -- so after the flag of block r-1
//             only y_r = c - M y_{r-1} remains (one 64x64 product);
//   FWD_UPD   after FWD_CHAIN, the update-row blocks, with every y_k
//             already published.
// In the last diagonal block rows >= s are update rows of the same front.
constexpr int FWD_ALL = 0, FWD_CHAIN = 1, FWD_UPD = 2;
// levels whose largest big front has at least this many columns use
// FWD_CHAIN + FWD_UPD (the split pays off on long chains only)
constexpr int FWD_CHAIN_MIN_S = 2048;

template <typename T, int MODE>
constexpr size_t fwd_smem() {
  return MODE == FWD_CHAIN ? 2 * BR * (BR + 1) * sizeof(T) : MODE == FWD_ALL ? BR * (BR + 1) * sizeof(T) : 0;
}

template <typename T, int NQ, int WS, int MODE>
__global__ void __launch_bounds__(128)
k_fwd_big(const int2_* __restrict__ blocks, const FrontDesc* __restrict__ fronts,
          const int* __restrict__ children, const int* __restrict__ maps, const int* __restrict__ rows,
          const T* __restrict__ L, const T* __restrict__ Dinv, const T* __restrict__ B, int ldb,
          T* __restrict__ W, int nrhs, int* __restrict__ flags, int epoch, int* status) {
  __shared__ T wv[BR][NQ];
  __shared__ T yk[BR][NQ];
  __shared__ T part[BR][NQ];
  __shared__ T ykw[4][BR / 2][NQ];   // per warp: the entries of y_k it needs
  __shared__ int rng[2];
  // CHAIN: dg[col][row] holds L_rr^-1 in rows < bw and the front's own
  // update rows of L (last diagonal block) in rows >= bw; mx[col][row] holds
  // L_{r,r-1}, then M = L_rr^-1 L_{r,r-1} in rows < bw
  extern __shared__ __align__(16) unsigned char fsm[];
  T (*dg)[BR + 1] = reinterpret_cast<T (*)[BR + 1]>(fsm);
  T (*mx)[BR + 1] = reinterpret_cast<T (*)[BR + 1]>(fsm) + BR;
  const int2_ bk = blocks[blockIdx.x];
  const FrontDesc F = fronts[bk.a];
  const int r = bk.b, f = F.f, s = F.s;
  const int nbs = (s + BR - 1) / BR;
  const int r0 = r * BR, nr = min(BR, f - r0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int row = tid % BR, half = tid / BR;
  T* Wf = W + F.v_off * WS;
  const int* rw = rows + F.rows_off;
  const T* P = L + F.l_off;
  constexpr bool CHAIN = MODE == FWD_CHAIN;
  const bool diag = CHAIN || (MODE == FWD_ALL && r < nbs);
  const int bw = diag ? min(BR, s - r0) : 0;

  if (diag) {
    // staged now, off the chain's critical path
    const T* Di = Dinv + F.dinv_off + (size_t) r * BR * BR;
    // 16 entries of each tile per thread in flight before they are stored
#pragma unroll 1
    for (int t0 = 0; t0 < BR * BR / 128; t0 += 16) {
      T dv[16], mv[16];
#pragma unroll
      for (int t = 0; t < 16; t++) {
        const int e = tid + 128 * (t0 + t), i = e % BR, j = e / BR;
        T v = 0.0;
        if (j < bw && i < nr) v = (i < bw) ? (i >= j ? Di[i + j * BR] : T(0)) : P[(r0 + i) + (size_t) (r0 + j) * f];
        dv[t] = v;
        mv[t] = (CHAIN && r > 0 && i < nr) ? P[(r0 + i) + (size_t) (r0 - BR + j) * f] : T(0);
      }
#pragma unroll
      for (int t = 0; t < 16; t++) {
        const int e = tid + 128 * (t0 + t), i = e % BR, j = e / BR;
        dg[j][i] = dv[t];
        if (CHAIN && r > 0) mx[j][i] = mv[t];
      }
    }
  }
  if (CHAIN && r > 0) {
    // M = L_rr^-1 L_{r,r-1} in rows < bw (the inverse is lower triangular),
    // at kernel start, independent of the chain
    __syncthreads();
    T m[BR / 2];
#pragma unroll
    for (int jj = 0; jj < BR / 2; jj++) m[jj] = 0.0;
    if (row < bw)
      for (int t = 0; t <= row; t++) {
        const T d = dg[t][row];
#pragma unroll
        for (int jj = 0; jj < BR / 2; jj++) m[jj] += d * mx[half * (BR / 2) + jj][t];
      }
    __syncthreads();
    if (row < bw)
#pragma unroll
      for (int jj = 0; jj < BR / 2; jj++) mx[half * (BR / 2) + jj][row] = m[jj];
  }
  for (int k = tid; k < BR * NQ; k += 128) {
    const int i = k % BR, q = k / BR;
    wv[i][q] = (i < nr && q < nrhs && r0 + i < s) ? B[rw[r0 + i] + (size_t) q * ldb] : 0.0;
  }
  __syncthreads();
  for (int ci = F.child_begin; ci < F.child_end; ci++) {
    const FrontDesc C = fronts[children[ci]];
    const int mc = C.f - C.s;
    const int* mp = maps + C.map_off;
    if (warp < 2) {
      const int x = warp_lower_bound(mp, mc, warp == 0 ? r0 : r0 + nr);
      if (lane == 0) rng[warp] = x;
    }
    __syncthreads();
    const int ia = rng[0], ib = rng[1];
    __syncthreads();
    if (ia >= ib) continue;
    const T* Wc = W + C.v_off * WS;
    for (int k = tid; k < (ib - ia) * nrhs; k += 128) {
      const int i = ia + k % (ib - ia), q = k / (ib - ia);
      wv[mp[i] - r0][q] += Wc[C.s + i + q * C.f];
    }
    __syncthreads();
  }
  // contributions of the solved blocks k < kend; this thread's 32 entries of
  // L[r, k] are loaded before waiting for y_k
  T acc[NQ];
#pragma unroll
  for (int q = 0; q < NQ; q++) acc[q] = 0.0;
  const int kend = CHAIN ? max(r - 1, 0) : diag ? r : nbs;
  if constexpr (NQ >= 8) {
    // 8 columns: y_k staged once for the whole block (measured faster than
    // the warp-level loop below at 8 columns)
    for (int k = 0; k < kend; k++) {
      const int bwk = min(BR, s - k * BR);
      T lv[BR / 2];
      const T* pc = P + (r0 + row) + (size_t) (k * BR + half * (BR / 2)) * f;
#pragma unroll
      for (int j = 0; j < BR / 2; j++)
        lv[j] = (row < nr && half * (BR / 2) + j < bwk) ? pc[(size_t) j * f] : 0.0;
      wait_epoch(flags + F.blk_off + k, epoch, status);
      for (int e = tid; e < BR * NQ; e += 128) {
        const int j = e % BR, q = e / BR;
        yk[j][q] = (j < bwk && q < nrhs) ? __ldcg(Wf + k * BR + j + (size_t) q * f) : 0.0;
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < BR / 2; j++)
#pragma unroll
        for (int q = 0; q < NQ; q++) acc[q] += lv[j] * yk[half * (BR / 2) + j][q];
      __syncthreads();
    }
  } else {
    // without block-wide barriers: each warp polls the flags itself and
    // stages the 32 entries of y_k its rows need
    T (*yw)[NQ] = ykw[warp];
    for (int k = 0; k < kend; k++) {
      const int bwk = min(BR, s - k * BR);
      T lv[BR / 2];
      const T* pc = P + (r0 + row) + (size_t) (k * BR + half * (BR / 2)) * f;
  #pragma unroll
      for (int j = 0; j < BR / 2; j++)
        lv[j] = (row < nr && half * (BR / 2) + j < bwk) ? pc[(size_t) j * f] : 0.0;
      wait_epoch_warp(flags + F.blk_off + k, epoch, status);
  #pragma unroll
      for (int q = 0; q < NQ; q++) {
        const int j = half * (BR / 2) + lane;
        yw[lane][q] = (j < bwk && q < nrhs) ? __ldcg(Wf + k * BR + j + (size_t) q * f) : T(0);
      }
      __syncwarp();
  #pragma unroll
      for (int j = 0; j < BR / 2; j++)
  #pragma unroll
        for (int q = 0; q < NQ; q++) acc[q] += lv[j] * yw[j][q];
      __syncwarp();
    }
  }
  if (half == 1)
#pragma unroll
    for (int q = 0; q < NQ; q++) part[row][q] = acc[q];
  __syncthreads();
  if (half == 0)
#pragma unroll
    for (int q = 0; q < NQ; q++) wv[row][q] -= acc[q] + part[row][q];
  __syncthreads();
  if (!diag) {
    for (int k = tid; k < nr * nrhs; k += 128) {
      const int i = k % nr, q = k / nr;
      Wf[r0 + i + (size_t) q * f] = wv[i][q];
    }
    return;
  }
  // c = L_rr^-1 w in rows < bw (into yk); update rows keep w
  {
    T y[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) y[q] = 0.0;
#pragma unroll 8
    for (int j = half * (BR / 2); j < half * (BR / 2) + BR / 2; j++) {
      const T d = (row < bw) ? dg[j][row] : T(0);
#pragma unroll
      for (int q = 0; q < NQ; q++) y[q] += d * wv[j][q];
    }
    if (half == 1)
#pragma unroll
      for (int q = 0; q < NQ; q++) part[row][q] = y[q];
    __syncthreads();
    if (half == 0)
#pragma unroll
      for (int q = 0; q < NQ; q++) yk[row][q] = (row < bw) ? y[q] + part[row][q] : wv[row][q];
    __syncthreads();
  }
  // the critical step: y_r = c - M y_{r-1} (update rows: w - L_{i,r-1} y_{r-1})
  if (CHAIN && r > 0) {
    wait_epoch(flags + F.blk_off + r - 1, epoch, status);
    for (int e = tid; e < BR * NQ; e += 128) {
      const int j = e % BR, q = e / BR;
      wv[j][q] = (q < nrhs) ? __ldcg(Wf + (r - 1) * BR + j + (size_t) q * f) : T(0);
    }
    __syncthreads();
    T u[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) u[q] = 0.0;
#pragma unroll 8
    for (int j = half * (BR / 2); j < half * (BR / 2) + BR / 2; j++) {
      const T mv = mx[j][row];
#pragma unroll
      for (int q = 0; q < NQ; q++) u[q] += mv * wv[j][q];
    }
    if (half == 1)
#pragma unroll
      for (int q = 0; q < NQ; q++) part[row][q] = u[q];
    __syncthreads();
    if (half == 0)
#pragma unroll
      for (int q = 0; q < NQ; q++) yk[row][q] -= u[q] + part[row][q];
    __syncthreads();
  }
  if (bw < nr) {
    // update rows inside the last diagonal block: w_i -= L[i, r] y_r
    T u[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) u[q] = 0.0;
    if (row >= bw)
      for (int j = half * (BR / 2); j < min(bw, half * (BR / 2) + BR / 2); j++) {
        const T l = dg[j][row];
#pragma unroll
        for (int q = 0; q < NQ; q++) u[q] += l * yk[j][q];
      }
    if (half == 1)
#pragma unroll
      for (int q = 0; q < NQ; q++) part[row][q] = u[q];
    __syncthreads();
    if (half == 0 && row >= bw)
#pragma unroll
      for (int q = 0; q < NQ; q++) yk[row][q] -= u[q] + part[row][q];
    __syncthreads();
  }
  for (int k = tid; k < nr * nrhs; k += 128) {
    const int i = k % nr, q = k / nr;
    Wf[r0 + i + (size_t) q * f] = yk[i][q];
  }
  __syncthreads();
  // the barrier orders every thread's writes before thread 0's release store
  if (tid == 0) st_release(flags + F.blk_off + r, epoch);
}

// Forward solve of the diagonal blocks of levels with long chains, as a
// walk.  One walker CTA per big front runs the chain y_r = L_rr^-1 (w_r -
// sum_{k<r} L_rk y_k) itself, block after block, keeping the last WALK_D
// y's in shared memory: consecutive steps are linked by barriers inside one
// CTA, not by flags between CTAs.  Helper CTAs, one per diagonal block,
// gather w_r and subtract the far terms k < r - WALK_D as the walker
// publishes y_k, then publish the partial p_r -- WALK_D steps ahead of the
// walker -- and pull the walker's tiles of their block into L2; the walker
// at step r subtracts the WALK_D near terms and applies the block's inverse.
// Every value crossing between CTAs travels as a tagged pair (tag in the
// high word, value in the low word, one 8-byte relaxed store): a reader
// knows a value is current when its tag is, so neither side fences or
// polls a flag.  The tag is (call counter << 12) | epoch, the counter being
// advanced on the device at the start of every solve call (recorded launch
// sequences stay valid), so a slot never holds a current-looking stale pair.
// Inside the walker eight compute warps run the arithmetic while a ninth
// warp loads the partials two steps ahead, handing them over through named
// barriers (one per direction and step parity).  The tiles of step r + 1
// (L_{r+1,k} for the near k and the next inverse) are loaded into registers
// while step r runs.  Walkers have the lowest CTA indices and a helper waits
// only for the walker of its front, which waits only for helpers of lower
// index, so in-order dispatch keeps every wait finite; the waits are bounded
// all the same.  In the last diagonal block rows >= s are update rows of the
// same front; the walker finishes them too.  The update-row blocks follow in
// FWD_UPD (the walker also sets the blocks' flags for it).  Right-hand sides
// are processed eight at a time (the layout of the pairs).
constexpr int WALK_D = 2, WALK_T = WALK_D + 1;
constexpr int WALK_PER = WALK_T * BR * BR / 256;   // staged tile entries per compute thread
constexpr int WALK_THREADS = 288;                   // eight compute warps and a loader warp
constexpr int WALK_PAIRS = BR * SOLVE_NRHS;         // tagged pairs per block: [row][right-hand side]
// levels with more big fronts keep the flag-chained kernels: every walker
// must be resident with room to spare for helpers (two CTAs per SM)
constexpr int WALK_MAX_FRONTS = 64;
constexpr int BWD_WALK_MIN_S = 512;
// named barriers of the walker (0 is __syncthreads): the compute warps
// among themselves; partial of a step ready (+ step parity); partial buffer
// of a step released (+ step parity)
constexpr int WB_COMPUTE = 1, WB_READY = 2, WB_FREE = 4;

// barrier ids are immediates, so that the kernel reserves only the ids it uses
template <int ID, int N>
__device__ __forceinline__ void nbar_sync() {
  asm volatile("bar.sync %0, %1;" ::"n"(ID), "n"(N) : "memory");
}
template <int ID, int N>
__device__ __forceinline__ void nbar_arrive() {
  asm volatile("bar.arrive %0, %1;" ::"n"(ID), "n"(N) : "memory");
}
__device__ __forceinline__ void walk_ready_arrive(int par) {
  if (par) nbar_arrive<WB_READY + 1, WALK_THREADS>();
  else nbar_arrive<WB_READY, WALK_THREADS>();
}
__device__ __forceinline__ void walk_ready_sync(int par) {
  if (par) nbar_sync<WB_READY + 1, WALK_THREADS>();
  else nbar_sync<WB_READY, WALK_THREADS>();
}
__device__ __forceinline__ void walk_free_arrive(int par) {
  if (par) nbar_arrive<WB_FREE + 1, WALK_THREADS>();
  else nbar_arrive<WB_FREE, WALK_THREADS>();
}
__device__ __forceinline__ void walk_free_sync(int par) {
  if (par) nbar_sync<WB_FREE + 1, WALK_THREADS>();
  else nbar_sync<WB_FREE, WALK_THREADS>();
}
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// tagged pairs: one relaxed 8-byte access each (single-copy atomic)
__device__ __forceinline__ void put_pair(unsigned long long* p, unsigned tag, float v) {
  const unsigned long long x = ((unsigned long long) tag << 32) | __float_as_uint(v);
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(x) : "memory");
}
__device__ __forceinline__ unsigned long long get_pair(const unsigned long long* p) {
  unsigned long long x;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(x) : "l"(p) : "memory");
  return x;
}
__device__ __forceinline__ bool pair_ok(unsigned long long x, unsigned tag) { return (unsigned) (x >> 32) == tag; }
__device__ __forceinline__ float pair_value(unsigned long long x) { return __uint_as_float((unsigned) x); }

// a row of eight FP32 values in shared memory (32-byte aligned), read as
// two 128-bit vectors
__device__ __forceinline__ void ld_row8(const float* p, float (&v)[8]) {
  const float4 a = *reinterpret_cast<const float4*>(p), b = *reinterpret_cast<const float4*>(p + 4);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
__device__ __forceinline__ void st_row8(float* p, const float (&v)[8]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  *reinterpret_cast<float4*>(p + 4) = make_float4(v[4], v[5], v[6], v[7]);
}

// the tag of a walk: the solve call's counter and the epoch
__device__ __forceinline__ unsigned walk_tag(const int* counter, int epoch) {
  return ((unsigned) *counter << 12) | (unsigned) epoch;
}

// waits (bounded) until pair x at p carries tag, reloading it
__device__ __forceinline__ unsigned long long wait_pair(const unsigned long long* p, unsigned long long x, unsigned tag,
                                                        int* status) {
  const int limit = g_solve_wait_limit;
  const unsigned want = tag + (unsigned) (g_solve_wait_skew << 12);
  int it = 0;
  while (!pair_ok(x, want)) {
    if (++it > limit || ((it & 1023) == 0 && *(volatile int*) status == SOLVE_TIMEOUT)) {
      atomicExch(status, SOLVE_TIMEOUT);
      break;
    }
    __nanosleep(32);
    x = get_pair(p);
  }
  return x;
}

// dynamic shared memory of the walk: the walker's tiles of one step, its
// ring of y's, two partial buffers, the quarters' products and the reduced
// partial; the helpers use the first part for their partial sums and staged
// y's
template <typename T>
constexpr size_t walk_smem() {
  return (WALK_T * BR * BR + (WALK_T + 2 + 4 + 1) * BR * SOLVE_NRHS) * sizeof(T);
}
// the backward walker's tiles are [row][column], padded against bank
// conflicts of the coalesced staging stores
template <typename T>
constexpr size_t bwalk_smem() {
  return (WALK_T * BR * (BR + 1) + (WALK_T + 2 + 4 + 1) * BR * SOLVE_NRHS) * sizeof(T);
}

// The far terms of a walk's helper: blocks t = 0 .. n-1 of the chain in the
// order the walker publishes them, each adding acc[q] += sum_jj
// load_l(t, jj) ys[qg * 16 + jj][q] with ys[i][q] the value of pair
// [i][q] of block pairs(t).  Every round loads up to WALK_HB blocks, all
// loads in flight at once, and uses the leading blocks whose pairs all carry
// the tag; a round that finds none waits (bounded) for the first.  Threads
// past the first 256 (act false) only keep the barriers.
constexpr int WALK_HB = 4;
template <int NQ, typename LoadL, typename Pairs>
__device__ __forceinline__ void walk_far_terms(unsigned tag, int* status, int n, LoadL load_l, Pairs pairs,
                                               float (*ysb)[BR][NQ], float (&acc)[NQ], int qg, bool act) {
  __shared__ unsigned bad_s;
  constexpr int NY = WALK_HB * BR * NQ / 256;
  for (int t = 0; t < n;) {
    const int nb = min(n - t, WALK_HB);
    if (threadIdx.x == 0) bad_s = 0;
    __syncthreads();
    float lv[WALK_HB][BR / 4];
    unsigned long long yv[NY];
    if (act) {
#pragma unroll
      for (int b = 0; b < WALK_HB; b++)
#pragma unroll
        for (int jj = 0; jj < BR / 4; jj++) lv[b][jj] = (b < nb) ? load_l(t + b, jj) : 0.0f;
#pragma unroll
      for (int u = 0; u < NY; u++) {
        const int e = threadIdx.x + 256 * u, b = e / (BR * NQ);
        yv[u] = (b < nb) ? get_pair(pairs(t + b) + e % (BR * NQ)) : 0ull;
      }
      unsigned bad = 0;
#pragma unroll
      for (int u = 0; u < NY; u++) {
        const int e = threadIdx.x + 256 * u, b = e / (BR * NQ);
        if (b < nb && !pair_ok(yv[u], tag)) bad |= 1u << b;
      }
      if (bad) atomicOr(&bad_s, bad);
    }
    __syncthreads();
    // the leading blocks whose pairs are all current; none: wait for the first
    int ok = __ffs(bad_s | (1u << nb)) - 1;
    if (ok == 0) {
      if (act) {
#pragma unroll
        for (int u = 0; u < NY; u++) {
          const int e = threadIdx.x + 256 * u, b = e / (BR * NQ);
          if (b == 0) yv[u] = wait_pair(pairs(t) + e % (BR * NQ), yv[u], tag, status);
        }
      }
      ok = 1;
    }
    if (act) {
#pragma unroll
      for (int u = 0; u < NY; u++) {
        const int e = threadIdx.x + 256 * u, b = e / (BR * NQ), r = e % (BR * NQ);
        ysb[b][r / NQ][r % NQ] = pair_value(yv[u]);
      }
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int b = 0; b < WALK_HB; b++)
        if (b < ok)
#pragma unroll
          for (int jj = 0; jj < BR / 4; jj++) {
            float yv[NQ];
            ld_row8(ysb[b][qg * (BR / 4) + jj], yv);
#pragma unroll
            for (int q = 0; q < NQ; q++) acc[q] += lv[b][jj] * yv[q];
          }
    }
    __syncthreads();
    t += ok;
  }
}

template <typename T, int WS>
__global__ void __maxnreg__(112)
k_fwd_walk(const int* __restrict__ walk_fronts, int nwalk, const int2_* __restrict__ blocks,
           const FrontDesc* __restrict__ fronts, const int* __restrict__ children, const int* __restrict__ maps,
           const int* __restrict__ rows, const T* __restrict__ L, const T* __restrict__ Dinv,
           const T* __restrict__ B, int ldb, T* __restrict__ W, unsigned long long* __restrict__ ypairs,
           unsigned long long* __restrict__ ppairs, int nrhs, int* __restrict__ flags, const int* counter, int epoch,
           int* status) {
  static_assert(sizeof(T) == 4, "the tagged pairs carry FP32 values");
  constexpr int NQ = SOLVE_NRHS, TPT = BR * BR / 256;
  static_assert(NQ % 4 == 0, "four thread groups share the right-hand sides");
  extern __shared__ __align__(16) unsigned char wsm[];
  __shared__ T hpv[BR][NQ + 1];
  __shared__ int rng[2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int row = tid % BR, qg = tid / BR;
  const unsigned tag = walk_tag(counter, epoch);
  if (blockIdx.x < nwalk) {
    // ---------------------------------------------------------------- walker
    const FrontDesc F = fronts[walk_fronts[blockIdx.x]];
    const int f = F.f, s = F.s, nbs = (s + BR - 1) / BR;
    const T* P = L + F.l_off;
    T* Wf = W + F.v_off * WS;
    unsigned long long* yp = ypairs + (size_t) F.blk_off * WALK_PAIRS;
    const unsigned long long* pp = ppairs + (size_t) F.blk_off * WALK_PAIRS;
    // tl[j] for j < WALK_D: L_{r, r-WALK_D+j} (zero before the first block);
    // tl[WALK_D]: the inverse of block r, and in rows >= bw of the last
    // block the update rows' entries of L_{., r}; all column-major.  yr:
    // the ring of the last y's; pvb: the partials of even and odd steps;
    // red: the four j-quarters' partial products; pf: p_r after the near
    // terms.  Rows of eight right-hand sides, 32 bytes, read as vectors.
    T (*tl)[BR][BR] = reinterpret_cast<T (*)[BR][BR]>(wsm);
    T (*yr)[BR][NQ] = reinterpret_cast<T (*)[BR][NQ]>(wsm + WALK_T * BR * BR * sizeof(T));
    T (*pvb)[BR][NQ] = yr + WALK_T;   // [2]
    T (*red)[BR][NQ] = pvb + 2;        // [4]
    T (*pf)[NQ] = red[4];
    if (warp == 8) {
      // ---- loader warp: the partials two steps ahead
      auto load_p = [&](int r, int buf) {
        constexpr int NV = WALK_PAIRS / 32;
        unsigned long long v[NV];
        const unsigned long long* src = pp + (size_t) r * WALK_PAIRS;
#pragma unroll
        for (int u = 0; u < NV; u++) v[u] = get_pair(src + lane + 32 * u);
#pragma unroll
        for (int u = 0; u < NV; u++) {
          v[u] = wait_pair(src + lane + 32 * u, v[u], tag, status);
          const int e = lane + 32 * u;
          pvb[buf][e / NQ][e % NQ] = pair_value(v[u]);
        }
        walk_ready_arrive(buf);
      };
      load_p(0, 0);
      if (nbs > 1) load_p(1, 1);
      // one wait per step of the compute warps (the last two complete the
      // barriers of the final steps): step r - 2 released its buffer
      for (int r = 2; r < nbs + 2; r++) {
        walk_free_sync(r & 1);
        if (r < nbs) load_p(r, r & 1);
      }
      return;
    }
    // ---- compute warps
    T pre[WALK_PER];
    auto fetch = [&](int r) {
      const int r0 = r * BR, nr = min(BR, f - r0), bw = min(BR, s - r0);
      const T* Di = Dinv + F.dinv_off + (size_t) r * BR * BR;
#pragma unroll
      for (int t = 0; t < WALK_PER; t++) {
        const int jj = t / TPT, e = tid + 256 * (t % TPT);
        const int i = e % BR, j = e / BR;
        T v = 0.0;
        if (jj < WALK_D) {
          const int k = r - WALK_D + jj;   // a full block (k < r <= nbs - 1)
          if (k >= 0 && i < nr) v = P[(r0 + i) + (size_t) (k * BR + j) * f];
        } else if (j < bw && i < nr) {
          v = (i < bw) ? (i >= j ? Di[i + j * BR] : T(0)) : P[(r0 + i) + (size_t) (r0 + j) * f];
        }
        pre[t] = v;
      }
    };
    auto put = [&]() {
#pragma unroll
      for (int t = 0; t < WALK_PER; t++) {
        const int e = tid + 256 * (t % TPT);
        tl[t / TPT][e / BR][e % BR] = pre[t];
      }
    };
    fetch(0);
    put();
    // thread (row, j-quarter jq): the products of its row with 16 of the
    // block's columns for all eight right-hand sides, reduced over the
    // quarters in shared memory
    const int jq = tid / BR, j0 = jq * (BR / 4);
    for (int r = 0; r < nbs; r++) {
      const int r0 = r * BR, nr = min(BR, f - r0), bw = min(BR, s - r0);
      const int slot = r % WALK_T, buf = r & 1;
      // p_r is in place (loader warp) and so are the tiles of step r (every
      // compute thread put its share before arriving here)
      walk_ready_sync(buf);
      if (r + 1 < nbs) fetch(r + 1);   // in flight during the step
      // near terms: p_r -= sum_j L_{r, r-WALK_D+j} y_{r-WALK_D+j}
      {
        T u[NQ];
#pragma unroll
        for (int q = 0; q < NQ; q++) u[q] = 0.0;
#pragma unroll
        for (int jj = 0; jj < WALK_D; jj++) {
          const int k = r - WALK_D + jj;
          if (k < 0) continue;
          const int sl = k % WALK_T;
#pragma unroll 4
          for (int j = j0; j < j0 + BR / 4; j++) {
            const T l = tl[jj][j][row];
            T yv[NQ];
            ld_row8(yr[sl][j], yv);
#pragma unroll
            for (int q = 0; q < NQ; q++) u[q] += l * yv[q];
          }
        }
        st_row8(red[jq][row], u);
      }
      nbar_sync<WB_COMPUTE, 256>();
      // thread (row, jq) finishes right-hand sides 2 jq and 2 jq + 1
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int q = 2 * jq + c;
        pf[row][q] = pvb[buf][row][q] - (red[0][row][q] + red[1][row][q] + red[2][row][q] + red[3][row][q]);
      }
      nbar_sync<WB_COMPUTE, 256>();
      // the partial buffer of this step is free for the loader (step r + 2)
      walk_free_arrive(buf);
      // y_r = L_rr^-1 p_r in rows < bw (the inverse is lower triangular)
      {
        T u[NQ];
#pragma unroll
        for (int q = 0; q < NQ; q++) u[q] = 0.0;
        const int je = min(j0 + BR / 4, min(row + 1, bw));
        for (int j = j0; j < je; j++) {
          const T d = tl[WALK_D][j][row];
          T pv8[NQ];
          ld_row8(pf[j], pv8);
#pragma unroll
          for (int q = 0; q < NQ; q++) u[q] += d * pv8[q];
        }
        st_row8(red[jq][row], u);
      }
      nbar_sync<WB_COMPUTE, 256>();
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int q = 2 * jq + c;
        yr[slot][row][q] = (row < bw) ? red[0][row][q] + red[1][row][q] + red[2][row][q] + red[3][row][q] : pf[row][q];
      }
      nbar_sync<WB_COMPUTE, 256>();
      if (bw < nr) {
        // update rows inside the last diagonal block: w_i -= L[i, r] y_r
        // (reads rows < bw of the ring slot, writes rows >= bw)
        if (row >= bw) {
#pragma unroll
          for (int c = 0; c < 2; c++) {
            const int q = 2 * jq + c;
            T v = 0.0;
            for (int j = 0; j < bw; j++) v += tl[WALK_D][j][row] * yr[slot][j][q];
            yr[slot][row][q] -= v;
          }
        }
        nbar_sync<WB_COMPUTE, 256>();
      }
      // y_r: tagged pairs for the helpers, plain values for later launches
      {
        unsigned long long* dst = yp + (size_t) r * WALK_PAIRS;
#pragma unroll
        for (int u = 0; u < WALK_PAIRS / 256; u++) {
          const int e = tid + 256 * u;
          put_pair(dst + e, tag, yr[slot][e / NQ][e % NQ]);
        }
      }
      for (int e = tid; e < nr * nrhs; e += 256) {
        const int i = e % nr, q = e / nr;
        Wf[r0 + i + (size_t) q * f] = yr[slot][i][q];
      }
      if (tid == 0) flags[F.blk_off + r] = epoch;
      // every read of this step's tiles is done before they are replaced
      nbar_sync<WB_COMPUTE, 256>();
      if (r + 1 < nbs) put();
    }
    return;
  }
  // ------------------------------------------------------------------ helper
  // (the loader warp's threads only keep the barriers here)
  const bool act = tid < 256;
  const int2_ bk = blocks[blockIdx.x - nwalk];
  const FrontDesc F = fronts[bk.a];
  const int r = bk.b, f = F.f, s = F.s;
  const int r0 = r * BR, nr = min(BR, f - r0);
  const T* P = L + F.l_off;
  const int* rw = rows + F.rows_off;
  T (*red)[BR][NQ] = reinterpret_cast<T (*)[BR][NQ]>(wsm);            // [4]
  T (*ysb)[BR][NQ] = reinterpret_cast<T (*)[BR][NQ]>(wsm) + 4;         // [WALK_HB]
  const int kend = max(r - WALK_D, 0);
  const unsigned long long* yp = ypairs + (size_t) F.blk_off * WALK_PAIRS;
  // the walker's tiles of this block into L2: the near blocks' 64 columns
  // (two 128-byte lines each, the second while it holds rows of the front)
  // and the block's inverse
  {
    const int ncol = WALK_D * BR, dlines = (int) (BR * BR * sizeof(T) / 128);
    const T* Di = Dinv + F.dinv_off + (size_t) r * BR * BR;
    for (int e = tid; e < 2 * ncol + dlines; e += WALK_THREADS) {
      if (e < 2 * ncol) {
        const int c = e >> 1, half = e & 1, k = r - WALK_D + c / BR;
        if (k >= 0 && (half == 0 || r0 + 128 / (int) sizeof(T) < f))
          prefetch_l2(P + r0 + half * (128 / (int) sizeof(T)) + (size_t) (k * BR + c % BR) * f);
      } else {
        prefetch_l2(reinterpret_cast<const unsigned char*>(Di) + (size_t) (e - 2 * ncol) * 128);
      }
    }
  }
  for (int k = tid; k < BR * NQ; k += WALK_THREADS) {
    const int i = k % BR, q = k / BR;
    hpv[i][q] = (i < nr && q < nrhs && r0 + i < s) ? B[rw[r0 + i] + (size_t) q * ldb] : T(0);
  }
  __syncthreads();
  for (int ci = F.child_begin; ci < F.child_end; ci++) {
    const FrontDesc C = fronts[children[ci]];
    const int mc = C.f - C.s;
    const int* mp = maps + C.map_off;
    if (warp < 2) {
      const int x = warp_lower_bound(mp, mc, warp == 0 ? r0 : r0 + nr);
      if (lane == 0) rng[warp] = x;
    }
    __syncthreads();
    const int ia = rng[0], ib = rng[1];
    __syncthreads();
    if (ia >= ib) continue;
    const T* Wc = W + C.v_off * WS;
    for (int k = tid; k < (ib - ia) * nrhs; k += WALK_THREADS) {
      const int i = ia + k % (ib - ia), q = k / (ib - ia);
      hpv[mp[i] - r0][q] += Wc[C.s + i + q * C.f];
    }
    __syncthreads();
  }
  // far terms k < r - WALK_D: thread (row, quarter qg) sums 16 columns of
  // each L_rk for every right-hand side
  T acc[NQ];
#pragma unroll
  for (int q = 0; q < NQ; q++) acc[q] = 0.0;
  walk_far_terms<NQ>(
      tag, status, kend,
      [&](int k, int jj) -> T {
        return (row < nr) ? P[(r0 + row) + (size_t) (k * BR + qg * (BR / 4) + jj) * f] : T(0);
      },
      [&](int k) { return yp + (size_t) k * WALK_PAIRS; }, ysb, acc, qg, act);
  if (act) {
#pragma unroll
    for (int q = 0; q < NQ; q++) red[qg][row][q] = acc[q];
  }
  __syncthreads();
  unsigned long long* dst = ppairs + (size_t) (F.blk_off + r) * WALK_PAIRS;
  for (int e = tid; e < WALK_PAIRS; e += WALK_THREADS) {
    const int i = e / NQ, q = e % NQ;
    put_pair(dst + e, tag, hpv[i][q] - (red[0][i][q] + red[1][i][q] + red[2][i][q] + red[3][i][q]));
  }
}

// x at the update rows of every big front of a level, gathered once into the
// front's work vector (rows s..f-1) so the backward blocks read it coalesced
template <typename T, int WS>
__global__ void __launch_bounds__(128)
k_gather_upd(const int2_* __restrict__ blocks, const FrontDesc* __restrict__ fronts,
             const int* __restrict__ rows, const T* __restrict__ X, int ldx, T* __restrict__ W,
             int nrhs) {
  const int2_ bk = blocks[blockIdx.x];
  const FrontDesc F = fronts[bk.a];
  const int r0 = max(bk.b * BR, F.s), r1 = min(bk.b * BR + BR, F.f);
  if (r0 >= r1) return;
  T* Wf = W + F.v_off * WS;
  const int* rw = rows + F.rows_off;
  const int nr = r1 - r0;
  for (int e = threadIdx.x; e < nr * nrhs; e += blockDim.x) {
    const int i = r0 + e % nr, q = e / nr;
    Wf[i + (size_t) q * F.f] = X[rw[i] + (size_t) q * ldx];
  }
}

// Backward solve, L21^T x2 split over (column block, 512-row chunk) CTAs so
// that the whole GPU streams L21; each CTA stores its partial sums, which the
// chain kernel adds in chunk order.  The chunk of x2 is staged in shared
// memory once ([column][row], conflict-free across lanes); each warp takes
// its 16 columns of the block G = 32 / NQ at a time, so that the G x NQ = 32
// sums of a pass finish with one warp reduce-scatter (31 shuffles; lane t
// ends with sum t = column t / NQ, right-hand side t % NQ).
template <typename T, int NQ, int WS>
__global__ void __launch_bounds__(128)
k_bwd_l21(const int2_* __restrict__ tasks, const FrontDesc* __restrict__ fronts, const T* __restrict__ L,
          const T* __restrict__ W, T* __restrict__ part, int nrhs) {
  constexpr int G = 32 / NQ;
  static_assert(G * NQ == 32 && G <= 16, "a pass holds 32 sums of at most 16 columns");
  __shared__ T zs[NQ][SOLVE_RCH];
  const int2_ tk = tasks[blockIdx.x];
  const FrontDesc F = fronts[tk.a];
  const int k = tk.b >> 16, ch = tk.b & 0xffff;
  const int f = F.f, s = F.s, m = f - s;
  const int c0 = k * BR, bw = min(BR, s - c0);
  const int i0 = ch * SOLVE_RCH, nr = min(m - i0, SOLVE_RCH);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const T* z = W + F.v_off * WS + s + i0;
  const T* P = L + F.l_off + s + i0;
  // all of this thread's loads in flight before its first store
  {
    constexpr int NZ = NQ * SOLVE_RCH / 128;
    T zv[NZ];
#pragma unroll
    for (int t = 0; t < NZ; t++) {
      const int e = threadIdx.x + 128 * t, i = e % SOLVE_RCH, q = e / SOLVE_RCH;
      zv[t] = (i < nr && q < nrhs) ? __ldcg(z + i + (size_t) q * f) : T(0);
    }
#pragma unroll
    for (int t = 0; t < NZ; t++) {
      const int e = threadIdx.x + 128 * t;
      zs[e / SOLVE_RCH][e % SOLVE_RCH] = zv[t];
    }
  }
  __syncthreads();
  for (int cg = warp * 16; cg < warp * 16 + 16; cg += G) {
    T v[32];   // v[a * NQ + q]: column cg + a, right-hand side q
#pragma unroll
    for (int j = 0; j < 32; j++) v[j] = T(0);
    // RU rows per lane per round, 16 loads of the panel in flight at once
    // (one round per memory latency)
    constexpr int RU = G >= 16 ? 1 : 16 / G;
    for (int i0 = lane; i0 < nr; i0 += 32 * RU) {
      T lv[RU][G];
#pragma unroll
      for (int u = 0; u < RU; u++)
#pragma unroll
        for (int a = 0; a < G; a++) {
          const int i = i0 + 32 * u;
          lv[u][a] = (i < nr && cg + a < bw) ? P[i + (size_t) (c0 + cg + a) * f] : T(0);
        }
#pragma unroll
      for (int u = 0; u < RU; u++) {
        const int i = i0 + 32 * u;
        if (i < nr) {
          T zi[NQ];
#pragma unroll
          for (int q = 0; q < NQ; q++) zi[q] = zs[q][i];
#pragma unroll
          for (int a = 0; a < G; a++)
#pragma unroll
            for (int q = 0; q < NQ; q++) v[a * NQ + q] += lv[u][a] * zi[q];
        }
      }
    }
    // reduce-scatter: at offset o a lane keeps the half of its remaining
    // sums that matches its bit o and adds the partner's copy of that half
#pragma unroll
    for (int o = 16, h = 16; o >= 1; o >>= 1, h >>= 1) {
      const bool up = (lane & o) != 0;
#pragma unroll
      for (int j = 0; j < h; j++) {
        const T send = up ? v[j] : v[j + h];
        const T keep = up ? v[j + h] : v[j];
        v[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
    }
    const int a = lane / NQ, q = lane % NQ;
    if (cg + a < bw && q < nrhs) part[F.part_off + ((size_t) ch * s + c0 + cg + a) * SOLVE_NRHS + q] = v[0];
  }
}

template <typename T, int NQ, int WS, bool PARTS, bool WARPLOOP = (NQ < 8)>
__global__ void __launch_bounds__(128)
k_bwd_big(const int2_* __restrict__ blocks, const FrontDesc* __restrict__ fronts,
          const int* __restrict__ rows, const T* __restrict__ L, const T* __restrict__ Dinv, T* __restrict__ X, int ldx,
          T* __restrict__ W, const T* __restrict__ part, int nrhs, int* __restrict__ flags, int epoch,
          int* status) {
  constexpr int G = (16 / NQ) > 1 ? 16 / NQ : 1;   // columns per pass of the L21 product
  __shared__ T xv[BR][NQ];
  __shared__ T xj[BR][NQ];
  __shared__ T red[BR][NQ];
  __shared__ T xjw[4][BR / 2][NQ];   // per warp: the rows of x_j it needs
  extern __shared__ __align__(16) unsigned char bsmraw[];
  T (*dgb)[BR + 1] = reinterpret_cast<T (*)[BR + 1]>(bsmraw);                              // L_kk^-1, [row][col]
  T (*tile)[BR + 1] = reinterpret_cast<T (*)[BR + 1]>(bsmraw) + BR;   // NQ >= 8: block of L11, [col][row]
  const int2_ bk = blocks[blockIdx.x];
  const FrontDesc F = fronts[bk.a];
  const int k = bk.b, f = F.f, s = F.s, m = f - s;
  const int nbs = (s + BR - 1) / BR;
  const int c0 = k * BR, bw = min(BR, s - c0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  T* Wf = W + F.v_off * WS;
  const int* rw = rows + F.rows_off;
  const T* P = L + F.l_off;

  // stage the block's inverse now, off the chain's critical path
  const T* Di = Dinv + F.dinv_off + (size_t) k * BR * BR;
#pragma unroll 1
  for (int t0 = 0; t0 < BR * BR / 128; t0 += 16) {
    T dv[16];
#pragma unroll
    for (int t = 0; t < 16; t++) {
      const int e = tid + 128 * (t0 + t), i = e % BR, c = e / BR;
      dv[t] = (i < bw && c < bw && i >= c) ? Di[i + c * BR] : T(0);
    }
#pragma unroll
    for (int t = 0; t < 16; t++) {
      const int e = tid + 128 * (t0 + t);
      dgb[e % BR][e / BR] = dv[t];
    }
  }
  for (int e = tid; e < BR * NQ; e += 128) {
    const int c = e % BR, q = e / BR;
    xv[c][q] = (c < bw && q < nrhs) ? Wf[c0 + c + (size_t) q * f] : 0.0;
  }
  __syncthreads();
  if (PARTS) {
    // y - L21^T x2 from the per-chunk partial sums, added in chunk order
    for (int e = tid; e < bw * NQ; e += 128) {
      const int c = e % bw, q = e / bw;
      if (q < nrhs) {
        T acc = 0.0;
#pragma unroll 4
        for (int ch = 0; ch < F.nchunk; ch++)
          acc += __ldcg(part + F.part_off + ((size_t) ch * s + c0 + c) * SOLVE_NRHS + q);
        xv[c][q] -= acc;
      }
    }
  }
  // y - L21^T x2: warp w owns columns 16w..16w+15, G at a time; lanes run
  // down the update rows with one coalesced load per column per step
  const T* z = Wf + s;
  for (int cg = warp * 16; !PARTS && cg < warp * 16 + 16; cg += G) {
    T acc[G][NQ];
#pragma unroll
    for (int a_ = 0; a_ < G; a_++)
#pragma unroll
      for (int q = 0; q < NQ; q++) acc[a_][q] = 0.0;
    for (int i = lane; i < m; i += 32) {
      T zi[NQ];
#pragma unroll
      for (int q = 0; q < NQ; q++) zi[q] = (q < nrhs) ? __ldcg(z + i + (size_t) q * f) : 0.0;
#pragma unroll
      for (int a_ = 0; a_ < G; a_++) {
        const T l = (cg + a_ < bw) ? P[(s + i) + (size_t) (c0 + cg + a_) * f] : 0.0;
#pragma unroll
        for (int q = 0; q < NQ; q++) acc[a_][q] += l * zi[q];
      }
    }
#pragma unroll
    for (int a_ = 0; a_ < G; a_++)
#pragma unroll
      for (int q = 0; q < NQ; q++) {
        T v = acc[a_][q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0 && cg + a_ < bw) xv[cg + a_][q] -= v;
      }
  }
  __syncthreads();
  const int col = tid % BR, half = tid / BR;
  if constexpr (!WARPLOOP) {
    // 8 columns: the block of L11 is staged in shared memory before the wait
    // for x_j (measured faster than the warp-level loop below at 8 columns)
    for (int j = nbs - 1; j > k; j--) {
      const int bwj = min(BR, s - j * BR);
#pragma unroll 1
      for (int t0 = 0; t0 < BR * BR / 128; t0 += 16) {
        T tv[16];
#pragma unroll
        for (int t = 0; t < 16; t++) {
          const int e = tid + 128 * (t0 + t), i = e % BR, c = e / BR;
          tv[t] = (i < bwj && c < bw) ? P[(j * BR + i) + (size_t) (c0 + c) * f] : T(0);
        }
#pragma unroll
        for (int t = 0; t < 16; t++) {
          const int e = tid + 128 * (t0 + t);
          tile[e / BR][e % BR] = tv[t];
        }
      }
      wait_epoch(flags + F.blk_off + j, epoch, status);
      for (int e = tid; e < BR * NQ; e += 128) {
        const int i = e % BR, q = e / BR;
        xj[i][q] = (i < bwj && q < nrhs) ? __ldcg(Wf + j * BR + i + (size_t) q * f) : 0.0;
      }
      __syncthreads();
      T acc[NQ];
#pragma unroll
      for (int q = 0; q < NQ; q++) acc[q] = 0.0;
#pragma unroll 8
      for (int i = half * (BR / 2); i < half * (BR / 2) + BR / 2; i++) {
        const T l = tile[col][i];
#pragma unroll
        for (int q = 0; q < NQ; q++) acc[q] += l * xj[i][q];
      }
      if (half == 1)
#pragma unroll
        for (int q = 0; q < NQ; q++) red[col][q] = acc[q];
      __syncthreads();
      if (half == 0)
#pragma unroll
        for (int q = 0; q < NQ; q++) xv[col][q] -= acc[q] + red[col][q];
      __syncthreads();
    }
  } else {
  // solved blocks below, last first, without block-wide barriers: thread
  // (col, half) keeps its partial sum over the rows of its half across all
  // tiles (the 32 entries of L it needs are loaded before the wait); each
  // warp polls the flags itself and stages the 32 rows of x_j it needs; the
  // two halves are combined once at the end
  {
    T acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) acc[q] = 0.0;
    const T* pcol = P + (size_t) (c0 + col) * f + half * (BR / 2);
    T (*xw)[NQ] = xjw[warp];
    for (int j = nbs - 1; j > k; j--) {
      const int bwj = min(BR, s - j * BR);
      T lv[BR / 2];
#pragma unroll
      for (int t = 0; t < BR / 2; t++)
        lv[t] = (col < bw && half * (BR / 2) + t < bwj) ? __ldg(pcol + (size_t) j * BR + t) : T(0);
      wait_epoch_warp(flags + F.blk_off + j, epoch, status);
#pragma unroll
      for (int q = 0; q < NQ; q++) {
        const int i = half * (BR / 2) + lane;
        xw[lane][q] = (i < bwj && q < nrhs) ? __ldcg(Wf + (size_t) j * BR + i + (size_t) q * f) : T(0);
      }
      __syncwarp();
#pragma unroll
      for (int t = 0; t < BR / 2; t++)
#pragma unroll
        for (int q = 0; q < NQ; q++) acc[q] += lv[t] * xw[t][q];
      __syncwarp();
    }
    if (half == 1)
#pragma unroll
      for (int q = 0; q < NQ; q++) red[col][q] = acc[q];
    __syncthreads();
    if (half == 0)
#pragma unroll
      for (int q = 0; q < NQ; q++) xv[col][q] -= acc[q] + red[col][q];
    __syncthreads();
  }
  }
  // x_k = L_kk^-T v_k from the staged inverse, split over the two halves
  {
    T x[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) x[q] = 0.0;
#pragma unroll 8
    for (int i = half * (BR / 2); i < half * (BR / 2) + BR / 2; i++) {
      const T d = dgb[i][col];
#pragma unroll
      for (int q = 0; q < NQ; q++) x[q] += d * xv[i][q];
    }
    if (half == 1)
#pragma unroll
      for (int q = 0; q < NQ; q++) red[col][q] = x[q];
    __syncthreads();
    if (half == 0)
#pragma unroll
      for (int q = 0; q < NQ; q++) xj[col][q] = x[q] + red[col][q];
    __syncthreads();
  }
  for (int e = tid; e < bw * nrhs; e += 128) {
    const int c = e % bw, q = e / bw;
    Wf[c0 + c + (size_t) q * f] = xj[c][q];
    X[rw[c0 + c] + (size_t) q * ldx] = xj[c][q];
  }
  __syncthreads();
  // the barrier orders every thread's writes before thread 0's release store
  if (tid == 0) st_release(flags + F.blk_off + k, epoch);
}

// Backward solve of the diagonal blocks of levels with long chains, as a
// walk: the mirror of k_fwd_walk.  The walker of a front runs
// x_k = L_kk^-T (v_k - sum_{j>k} L_jk^T x_j) from the last block to the
// first, subtracting the WALK_D near terms j = k+1, k+2 itself, with the
// same split into compute warps and a loader warp; helper CTAs, one per
// diagonal block (listed last block first), form v_k = y_k - L21^T x2 from
// the chunk partial sums, subtract the far terms j > k + WALK_D as the
// walker publishes x_j, publish the partial and pull the walker's tiles of
// their block into L2.  Values cross between CTAs as tagged pairs, as in
// the forward walk, and the same in-order dispatch argument keeps every
// wait finite.
template <typename T, int WS>
__global__ void __maxnreg__(112)
k_bwd_walk(const int* __restrict__ walk_fronts, int nwalk, const int2_* __restrict__ blocks,
           const FrontDesc* __restrict__ fronts, const int* __restrict__ rows, const T* __restrict__ L,
           const T* __restrict__ Dinv, T* __restrict__ X, int ldx, T* __restrict__ W,
           const T* __restrict__ part, unsigned long long* __restrict__ ypairs,
           unsigned long long* __restrict__ ppairs, int nrhs, int* __restrict__ flags, const int* counter, int epoch,
           int* status) {
  static_assert(sizeof(T) == 4, "the tagged pairs carry FP32 values");
  constexpr int NQ = SOLVE_NRHS, TPT = BR * BR / 256;
  extern __shared__ __align__(16) unsigned char wsm[];
  __shared__ T hpv[BR][NQ + 1];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int col = tid % BR, qg = tid / BR;
  const unsigned tag = walk_tag(counter, epoch);
  if (blockIdx.x < nwalk) {
    // ---------------------------------------------------------------- walker
    const FrontDesc F = fronts[walk_fronts[blockIdx.x]];
    const int f = F.f, s = F.s, nbs = (s + BR - 1) / BR;
    const T* P = L + F.l_off;
    T* Wf = W + F.v_off * WS;
    const int* rw = rows + F.rows_off;
    unsigned long long* yp = ypairs + (size_t) F.blk_off * WALK_PAIRS;
    const unsigned long long* pp = ppairs + (size_t) F.blk_off * WALK_PAIRS;
    // tl[j] for j < WALK_D: L_{k+1+j, k} (zero past the last block);
    // tl[WALK_D]: the inverse of block k; all [row][column]
    T (*tl)[BR][BR + 1] = reinterpret_cast<T (*)[BR][BR + 1]>(wsm);
    T (*xr)[BR][NQ] = reinterpret_cast<T (*)[BR][NQ]>(wsm + WALK_T * BR * (BR + 1) * sizeof(T));
    T (*pvb)[BR][NQ] = xr + WALK_T;   // [2]: the partials by step parity
    T (*red)[BR][NQ] = pvb + 2;        // [4]: the i-quarters' products
    T (*pf)[NQ] = red[4];              // p_k after the near terms
    if (warp == 8) {
      // ---- loader warp; step t of the walk is block nbs - 1 - t
      auto load_p = [&](int t, int buf) {
        constexpr int NV = WALK_PAIRS / 32;
        unsigned long long v[NV];
        const unsigned long long* src = pp + (size_t) (nbs - 1 - t) * WALK_PAIRS;
#pragma unroll
        for (int u = 0; u < NV; u++) v[u] = get_pair(src + lane + 32 * u);
#pragma unroll
        for (int u = 0; u < NV; u++) {
          v[u] = wait_pair(src + lane + 32 * u, v[u], tag, status);
          const int e = lane + 32 * u;
          pvb[buf][e / NQ][e % NQ] = pair_value(v[u]);
        }
        walk_ready_arrive(buf);
      };
      load_p(0, 0);
      if (nbs > 1) load_p(1, 1);
      for (int t = 2; t < nbs + 2; t++) {
        walk_free_sync(t & 1);
        if (t < nbs) load_p(t, t & 1);
      }
      return;
    }
    // ---- compute warps
    T pre[WALK_PER];
    auto fetch = [&](int k) {
      const int c0 = k * BR, bw = min(BR, s - c0);
      const T* Di = Dinv + F.dinv_off + (size_t) k * BR * BR;
#pragma unroll
      for (int t = 0; t < WALK_PER; t++) {
        const int jj = t / TPT, e = tid + 256 * (t % TPT);
        const int i = e % BR, c = e / BR;
        T v = 0.0;
        if (jj < WALK_D) {
          const int j = k + 1 + jj;
          if (j < nbs && c < bw && i < min(BR, s - j * BR)) v = P[(j * BR + i) + (size_t) (c0 + c) * f];
        } else if (c < bw && i < bw && i >= c) {
          v = Di[i + c * BR];
        }
        pre[t] = v;
      }
    };
    auto put = [&]() {
#pragma unroll
      for (int t = 0; t < WALK_PER; t++) {
        const int e = tid + 256 * (t % TPT);
        tl[t / TPT][e % BR][e / BR] = pre[t];
      }
    };
    fetch(nbs - 1);
    put();
    // thread (col, i-quarter iq): the products of its column with 16 of the
    // block's rows for all eight right-hand sides, reduced over the quarters
    // in shared memory
    const int iq = tid / BR, i0 = iq * (BR / 4);
    for (int t = 0; t < nbs; t++) {
      const int k = nbs - 1 - t;
      const int c0 = k * BR, bw = min(BR, s - c0);
      const int slot = k % WALK_T, buf = t & 1;
      walk_ready_sync(buf);   // p_k and the tiles of step k are in place
      if (k > 0) fetch(k - 1);   // in flight during the step
      // the global row of this thread's x entry (full blocks), loaded now so
      // that the scatter at the end of the step does not wait for it
      const int gx = (bw == BR) ? __ldg(rw + c0 + tid % BR) : 0;
      // near terms: p_k -= sum_j L_{k+1+j, k}^T x_{k+1+j}
      {
        T u[NQ];
#pragma unroll
        for (int q = 0; q < NQ; q++) u[q] = 0.0;
#pragma unroll
        for (int jj = 0; jj < WALK_D; jj++) {
          const int j = k + 1 + jj;
          if (j >= nbs) continue;
          const int sl = j % WALK_T;
#pragma unroll 4
          for (int i = i0; i < i0 + BR / 4; i++) {
            const T l = tl[jj][i][col];
            T xv[NQ];
            ld_row8(xr[sl][i], xv);
#pragma unroll
            for (int q = 0; q < NQ; q++) u[q] += l * xv[q];
          }
        }
        st_row8(red[iq][col], u);
      }
      nbar_sync<WB_COMPUTE, 256>();
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int q = 2 * iq + c;
        pf[col][q] = pvb[buf][col][q] - (red[0][col][q] + red[1][col][q] + red[2][col][q] + red[3][col][q]);
      }
      nbar_sync<WB_COMPUTE, 256>();
      walk_free_arrive(buf);   // the partial buffer of this step is free
      // x_k = L_kk^-T p_k (the inverse is lower triangular)
      {
        T u[NQ];
#pragma unroll
        for (int q = 0; q < NQ; q++) u[q] = 0.0;
#pragma unroll
        for (int ii = 0; ii < BR / 4; ii++) {
          const int i = i0 + ii;
          const bool ok = i >= col && i < bw;
          const T d = tl[WALK_D][i][col];
          T pv8[NQ];
          ld_row8(pf[i], pv8);
#pragma unroll
          for (int q = 0; q < NQ; q++) u[q] += ok ? d * pv8[q] : T(0);
        }
        st_row8(red[iq][col], u);
      }
      nbar_sync<WB_COMPUTE, 256>();
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int q = 2 * iq + c;
        xr[slot][col][q] = (col < bw) ? red[0][col][q] + red[1][col][q] + red[2][col][q] + red[3][col][q] : T(0);
      }
      nbar_sync<WB_COMPUTE, 256>();
      {
        unsigned long long* dst = yp + (size_t) k * WALK_PAIRS;
#pragma unroll
        for (int u = 0; u < WALK_PAIRS / 256; u++) {
          const int e = tid + 256 * u;
          put_pair(dst + e, tag, xr[slot][e / NQ][e % NQ]);
        }
      }
      for (int e = tid; e < bw * nrhs; e += 256) {
        const int c = e % bw, q = e / bw;
        const T v = xr[slot][c][q];
        Wf[c0 + c + (size_t) q * f] = v;
        X[(bw == BR ? gx : rw[c0 + c]) + (size_t) q * ldx] = v;
      }
      if (tid == 0) flags[F.blk_off + k] = epoch;
      // every read of this step's tiles is done before they are replaced
      nbar_sync<WB_COMPUTE, 256>();
      if (k > 0) put();
    }
    return;
  }
  // ------------------------------------------------------------------ helper
  // (the loader warp's threads only keep the barriers here)
  const bool act = tid < 256;
  const int2_ bk = blocks[blockIdx.x - nwalk];
  const FrontDesc F = fronts[bk.a];
  const int k = bk.b, f = F.f, s = F.s;
  const int nbs = (s + BR - 1) / BR;
  const int c0 = k * BR, bw = min(BR, s - c0);
  const T* P = L + F.l_off;
  const T* Wf = W + F.v_off * WS;
  T (*red)[BR][NQ] = reinterpret_cast<T (*)[BR][NQ]>(wsm);            // [4]
  T (*ysb)[BR][NQ] = reinterpret_cast<T (*)[BR][NQ]>(wsm) + 4;         // [WALK_HB]
  const int jlo = k + WALK_D + 1;   // far blocks j = nbs-1 .. jlo
  const unsigned long long* yp = ypairs + (size_t) F.blk_off * WALK_PAIRS;
  // the walker's tiles of this block into L2: the near blocks' 64-row
  // column pieces of block column k (two 128-byte lines each, the second
  // while it holds rows of the near block) and the block's inverse
  {
    const int ncol = WALK_D * BR, dlines = (int) (BR * BR * sizeof(T) / 128);
    const T* Di = Dinv + F.dinv_off + (size_t) k * BR * BR;
    for (int e = tid; e < 2 * ncol + dlines; e += WALK_THREADS) {
      if (e < 2 * ncol) {
        const int c = e >> 1, half = e & 1, j = k + 1 + c / BR;
        const int rows_j = j < nbs ? min(BR, s - j * BR) : 0;
        if (c % BR < bw && (half == 0 ? rows_j > 0 : rows_j > 128 / (int) sizeof(T)))
          prefetch_l2(P + (size_t) j * BR + half * (128 / (int) sizeof(T)) + (size_t) (c0 + c % BR) * f);
      } else {
        prefetch_l2(reinterpret_cast<const unsigned char*>(Di) + (size_t) (e - 2 * ncol) * 128);
      }
    }
  }
  // v_k = y_k - L21^T x2, the chunk partial sums added in chunk order
  for (int e = tid; e < BR * NQ; e += WALK_THREADS) {
    const int c = e % BR, q = e / BR;
    T v = 0.0;
    if (c < bw && q < nrhs) {
      v = Wf[c0 + c + (size_t) q * f];
      T acc = 0.0;
#pragma unroll 4
      for (int ch = 0; ch < F.nchunk; ch++)
        acc += __ldcg(part + F.part_off + ((size_t) ch * s + c0 + c) * SOLVE_NRHS + q);
      v -= acc;
    }
    hpv[c][q] = v;
  }
  // far terms: blocks j = nbs-1 down to jlo (block t of the helper's order
  // is j = nbs-1-t); rows past the block's last column are zero in the pairs
  T acc[NQ];
#pragma unroll
  for (int q = 0; q < NQ; q++) acc[q] = 0.0;
  walk_far_terms<NQ>(
      tag, status, max(nbs - jlo, 0),
      [&](int t, int tt) -> T {
        const int j = nbs - 1 - t, i = qg * (BR / 4) + tt;
        return (col < bw && i < min(BR, s - j * BR)) ? __ldg(P + (size_t) (c0 + col) * f + j * BR + i) : T(0);
      },
      [&](int t) { return yp + (size_t) (nbs - 1 - t) * WALK_PAIRS; }, ysb, acc, qg, act);
  if (act) {
#pragma unroll
    for (int q = 0; q < NQ; q++) red[qg][col][q] = acc[q];
  }
  __syncthreads();
  unsigned long long* dst = ppairs + (size_t) (F.blk_off + k) * WALK_PAIRS;
  for (int e = tid; e < WALK_PAIRS; e += WALK_THREADS) {
    const int c = e / NQ, q = e % NQ;
    put_pair(dst + e, tag, hpv[c][q] - (red[0][c][q] + red[1][c][q] + red[2][c][q] + red[3][c][q]));
  }
}

// advances the walks' call counter (one thread)
__global__ void k_walk_counter(int* counter) { *counter += 1; }

}  // namespace

// algorithmic bytes of one solve pass over a front, values of esz bytes: the
// lower panel read once, its row list, the work vector read and written
static double solve_pass_bytes(const FrontDesc& F, int nrhs, double esz) {
  const double s = F.s, m = F.f - F.s;
  return esz * (s * (s + 1.0) / 2.0 + m * s) + 4.0 * F.f + 2.0 * esz * nrhs * F.f;
}

// the forward and backward walks on levels with long chains of FP32
// factors (TAUCS_B200_NO_SOLVE_WALK=1 selects the flag-chained kernels
// instead; FP64 keeps them: the walker's staged FP64 tiles take 164
// registers, one CTA per SM, too few resident helpers)
static bool walk_enabled() {
  static const bool on = [] {
    const char* e = getenv("TAUCS_B200_NO_SOLVE_WALK");
    return !(e && *e && strcmp(e, "0") != 0);
  }();
  return on;
}

template <typename T>
static void solve_attrs() {
  // once per device and type (request-server workers reach this concurrently)
  static PerDeviceOnce pd;
  per_device_once(pd, [] {
    // static + dynamic shared memory of these kernels can exceed the default
    // 48 KB (8 columns in FP64)
    cudaFuncSetAttribute(k_fwd_big<T, 2, SOLVE_NRHS, FWD_ALL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) fwd_smem<T, FWD_ALL>());
    cudaFuncSetAttribute(k_fwd_big<T, 4, SOLVE_NRHS, FWD_ALL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) fwd_smem<T, FWD_ALL>());
    cudaFuncSetAttribute(k_fwd_big<T, 8, SOLVE_NRHS, FWD_ALL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) fwd_smem<T, FWD_ALL>());
    cudaFuncSetAttribute(k_fwd_big<T, 1, 1, FWD_ALL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) fwd_smem<T, FWD_ALL>());
    cudaFuncSetAttribute(k_fwd_big<T, 2, SOLVE_NRHS, FWD_CHAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) fwd_smem<T, FWD_CHAIN>());
    cudaFuncSetAttribute(k_fwd_big<T, 4, SOLVE_NRHS, FWD_CHAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) fwd_smem<T, FWD_CHAIN>());
    cudaFuncSetAttribute(k_fwd_big<T, 8, SOLVE_NRHS, FWD_CHAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) fwd_smem<T, FWD_CHAIN>());
    cudaFuncSetAttribute(k_bwd_big<T, 2, SOLVE_NRHS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bwd_smem<T, 2>());
    cudaFuncSetAttribute(k_bwd_big<T, 4, SOLVE_NRHS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bwd_smem<T, 4>());
    cudaFuncSetAttribute(k_bwd_big<T, 8, SOLVE_NRHS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bwd_smem<T, 8>());
    cudaFuncSetAttribute(k_bwd_big<T, 1, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bwd_smem<T, 1>());
    cudaFuncSetAttribute(k_bwd_big<T, 8, SOLVE_NRHS, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bwd_smem<T, 8>());
    if constexpr (std::is_same<T, float>::value) {
      cudaFuncSetAttribute(k_fwd_walk<T, SOLVE_NRHS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int) walk_smem<T>());
      cudaFuncSetAttribute(k_bwd_walk<T, SOLVE_NRHS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int) bwalk_smem<T>());
    }
    return true;
  });
}

// CTAs (eight warps each) of the persistent small-front solve launches: up
// to four per SM, no more than the fronts need
static int pers_solve_grid(int ntask) {
  static PerDeviceOnce pd;
  static int sms[MAX_DEVICES];
  per_device_once(pd, [] {
    int d = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&sms[d], cudaDevAttrMultiProcessorCount, d);
    return true;
  });
  int d = 0;
  cudaGetDevice(&d);
  return std::max(1, std::min((ntask + 7) / 8, 4 * std::max(sms[d], 1)));
}

template <typename T>
static int launch_solve(const Plan& P, const DevPlan& D, const T* L, const T* Dinv, int nrhs, T* X, const T* B, int ld, T* W,
                        T* part, int* flags, int* epoch, int* status, cudaStream_t st) {
  solve_attrs<T>();
  // the handshake flags restart from zero on every call, so the epochs of a
  // call are always 1, 2, ... and a recorded launch sequence stays valid
  cudaMemsetAsync(flags, 0, sizeof(int) * solve_flag_words(P), st);
  // the walks: their tagged pairs, and the call counter in the word after
  // the cleared ones, advanced on the device once per call
  int* counter = flags + solve_flag_words(P);
  unsigned long long* ypairs = reinterpret_cast<unsigned long long*>(part + P.fpart_off);
  unsigned long long* ppairs = ypairs + (size_t) P.n_blk * WALK_PAIRS;
  // the forward walk pays off on chains of 32 blocks or more, the backward
  // one from 8 (both measured on the 80^3 lognormal system)
  auto walk_level = [&](const LevelPlan& LP, bool fwd) {
    return std::is_same<T, float>::value && walk_enabled() && LP.max_s_big >= (fwd ? FWD_CHAIN_MIN_S : BWD_WALK_MIN_S) &&
           (int) LP.big_fronts.size() <= WALK_MAX_FRONTS && LP.max_s_big < 4095 * BR;
  };
  bool walks = false;
  for (const LevelPlan& LP : P.levels) walks = walks || walk_level(LP, true) || walk_level(LP, false);
  if (walks) {
    k_walk_counter<<<1, 1, 0, st>>>(counter);
    count_launch();
  }
  const int np = D.n_pers;
  if (np > 0) cudaMemsetAsync(D.pers_solve, 0, sizeof(int) * (size_t) (2 * np + 2), st);
  int ep = 0;
  for (int q0 = 0; q0 < nrhs; q0 += SOLVE_NRHS) {
    const int nq = std::min(SOLVE_NRHS, nrhs - q0);
    const T* Bq = B + (size_t) q0 * ld;
    T* Xq = X + (size_t) q0 * ld;
    const int ef = ++ep;
    if (np > 0) {
      // every small front with only small fronts below it, one launch
      cudaMemcpyAsync(D.pers_solve, D.pers_pending0, sizeof(int) * np, cudaMemcpyDeviceToDevice, st);
      cudaMemsetAsync(D.pers_solve + 2 * np, 0, 2 * sizeof(int), st);
      double by = 0.0;
      if (prof_enabled())
        for (int i : P.pers_fronts) by += solve_pass_bytes(P.fronts[i], nq, sizeof(T));
      prof_begin(KC_SOLVE_FWD, st);
      k_fwd_pers<T, SOLVE_NRHS><<<pers_solve_grid(np), 256, 0, st>>>(
          D.pers_list, np, D.pers_parent, D.pers_solve, D.pers_solve + 2 * np, D.fronts, D.children, D.maps, D.rows,
          L, Bq, ld, W, nq, status);
      prof_end(KC_SOLVE_FWD, st, 0.0, by);
      count_launch();
    }
    for (int h = 0; h < P.n_levels; h++) {
      const LevelPlan& LP = P.levels[h];
      double by = 0.0;
      if (prof_enabled())
        for (int i = LP.front_begin; i < LP.front_end; i++) by += solve_pass_bytes(P.fronts[i], nq, sizeof(T));
      prof_begin(KC_SOLVE_FWD, st);
      const int ns = (int) LP.small_numeric.size();
      if (ns > 0) {
        const int* sl = D.small_num + D.small_num_off[h];
        const int nw = LP.small_numeric_warp;
        if (nw > 0) {
          k_fwd<T, SOLVE_NRHS, 32><<<(nw + 7) / 8, 256, 0, st>>>(sl, nw, D.fronts, D.children, D.maps, D.rows, L,
                                                                 Bq, ld, W, nq);
          count_launch();
        }
        if (ns > nw) {
          k_fwd<T, SOLVE_NRHS, 256><<<ns - nw, 256, 0, st>>>(sl + nw, ns - nw, D.fronts, D.children, D.maps, D.rows,
                                                             L, Bq, ld, W, nq);
          count_launch();
        }
      }
      const int nb = (int) LP.solve_fwd_blocks.size();
      if (nb > 0) {
        const int2_* bl = D.sfwd + D.sfwd_off[h];
        const int nd = LP.n_fwd_diag, nu = nb - nd;
        // one right-hand side runs the two-column variant, measured faster
        // than a one-column instantiation (columns >= nrhs are skipped)
        auto run = [&](auto nqc) {
          constexpr int Q = decltype(nqc)::value;
          if (walk_level(LP, true)) {
            const int nbig = (int) LP.big_fronts.size();
            if constexpr (std::is_same<T, float>::value)
              k_fwd_walk<T, SOLVE_NRHS><<<nbig + nd, WALK_THREADS, walk_smem<T>(), st>>>(
                  D.big_list + D.big_off[h], nbig, bl, D.fronts, D.children, D.maps, D.rows, L, Dinv, Bq, ld, W, ypairs,
                  ppairs, nq, flags, counter, ef, status);
            if (nu)
              k_fwd_big<T, Q, SOLVE_NRHS, FWD_UPD><<<nu, 128, 0, st>>>(bl + nd, D.fronts, D.children, D.maps, D.rows,
                                                                      L, Dinv, Bq, ld, W, nq, flags, ef, status);
            count_launch(nu ? 2 : 1);
          } else if (LP.max_s_big >= FWD_CHAIN_MIN_S) {
            k_fwd_big<T, Q, SOLVE_NRHS, FWD_CHAIN><<<nd, 128, fwd_smem<T, FWD_CHAIN>(), st>>>(
                bl, D.fronts, D.children, D.maps, D.rows, L, Dinv, Bq, ld, W, nq, flags, ef, status);
            if (nu)
              k_fwd_big<T, Q, SOLVE_NRHS, FWD_UPD><<<nu, 128, 0, st>>>(bl + nd, D.fronts, D.children, D.maps, D.rows,
                                                                      L, Dinv, Bq, ld, W, nq, flags, ef, status);
            count_launch(nu ? 2 : 1);
          } else {
            k_fwd_big<T, Q, SOLVE_NRHS, FWD_ALL><<<nb, 128, fwd_smem<T, FWD_ALL>(), st>>>(
                bl, D.fronts, D.children, D.maps, D.rows, L, Dinv, Bq, ld, W, nq, flags, ef, status);
            count_launch();
          }
        };
        if (nq <= 2) run(std::integral_constant<int, 2>());
        else if (nq <= 4) run(std::integral_constant<int, 4>());
        else run(std::integral_constant<int, 8>());
      }
      prof_end(KC_SOLVE_FWD, st, 0.0, by);
    }
    const int eb = ++ep;
    for (int h = P.n_levels - 1; h >= 0; h--) {
      const LevelPlan& LP = P.levels[h];
      double by = 0.0;
      if (prof_enabled())
        for (int i = LP.front_begin; i < LP.front_end; i++) by += solve_pass_bytes(P.fronts[i], nq, sizeof(T));
      prof_begin(KC_SOLVE_BWD, st);
      const int nb = (int) LP.solve_bwd_blocks.size();
      if (nb > 0) {
        k_gather_upd<T, SOLVE_NRHS><<<(int) LP.solve_fwd_blocks.size(), 128, 0, st>>>(D.sfwd + D.sfwd_off[h], D.fronts, D.rows,
                                                                        Xq, ld, W, nq);
        count_launch();
        const int nt = (int) LP.solve_l21_tasks.size();
        const int2_* tl = D.sl21 + D.sl21_off[h];
        if (nt > 0) {
          if (nq <= 2) k_bwd_l21<T, 2, SOLVE_NRHS><<<nt, 128, 0, st>>>(tl, D.fronts, L, W, part, nq);
          else if (nq <= 4) k_bwd_l21<T, 4, SOLVE_NRHS><<<nt, 128, 0, st>>>(tl, D.fronts, L, W, part, nq);
          else k_bwd_l21<T, 8, SOLVE_NRHS><<<nt, 128, 0, st>>>(tl, D.fronts, L, W, part, nq);
          count_launch();
        }
        const int2_* bl = D.sbwd + D.sbwd_off[h];
        if (walk_level(LP, false)) {
          const int nbig = (int) LP.big_fronts.size();
          if constexpr (std::is_same<T, float>::value)
            k_bwd_walk<T, SOLVE_NRHS><<<nbig + nb, WALK_THREADS, bwalk_smem<T>(), st>>>(
                D.big_list + D.big_off[h], nbig, bl, D.fronts, D.rows, L, Dinv, Xq, ld, W, part, ypairs, ppairs, nq,
                flags, counter, eb, status);
        } else if (nq <= 2)
          k_bwd_big<T, 2, SOLVE_NRHS, true><<<nb, 128, bwd_smem<T, 2>(), st>>>(bl, D.fronts, D.rows, L, Dinv, Xq, ld, W, part, nq, flags, eb, status);
        else if (nq <= 4)
          k_bwd_big<T, 4, SOLVE_NRHS, true><<<nb, 128, bwd_smem<T, 4>(), st>>>(bl, D.fronts, D.rows, L, Dinv, Xq, ld, W, part, nq, flags, eb, status);
        else if (LP.max_s_big >= FWD_CHAIN_MIN_S)
          // long chains: the barrier-free warp loop (every block's iterations are on the chain)
          k_bwd_big<T, 8, SOLVE_NRHS, true, true><<<nb, 128, bwd_smem<T, 8>(), st>>>(bl, D.fronts, D.rows, L, Dinv, Xq, ld, W, part, nq, flags, eb, status);
        else
          k_bwd_big<T, 8, SOLVE_NRHS, true><<<nb, 128, bwd_smem<T, 8>(), st>>>(bl, D.fronts, D.rows, L, Dinv, Xq, ld, W, part, nq, flags, eb, status);
        count_launch();
      }
      const int ns = (int) LP.small_numeric.size();
      if (ns > 0) {
        const int* sl = D.small_num + D.small_num_off[h];
        const int nw = LP.small_numeric_warp;
        if (nw > 0) {
          k_bwd<T, SOLVE_NRHS, 32><<<(nw + 7) / 8, 256, 0, st>>>(sl, nw, D.fronts, D.rows, L, Xq, ld, W, nq);
          count_launch();
        }
        if (ns > nw) {
          k_bwd<T, SOLVE_NRHS, 256><<<ns - nw, 256, 0, st>>>(sl + nw, ns - nw, D.fronts, D.rows, L, Xq, ld, W, nq);
          count_launch();
        }
      }
      prof_end(KC_SOLVE_BWD, st, 0.0, by);
    }
    if (np > 0) {
      double by = 0.0;
      if (prof_enabled())
        for (int i : P.pers_fronts) by += solve_pass_bytes(P.fronts[i], nq, sizeof(T));
      prof_begin(KC_SOLVE_BWD, st);
      k_bwd_pers<T, SOLVE_NRHS><<<pers_solve_grid(np), 256, 0, st>>>(
          D.pers_list, np, D.pers_parent, D.pers_solve + np, D.pers_solve + 2 * np + 1, eb, D.fronts, D.rows, L, Xq, ld,
          W, nq, status);
      prof_end(KC_SOLVE_BWD, st, 0.0, by);
      count_launch();
    }
  }
  (void) epoch;
  return (int) cudaGetLastError();
}

int launch_solve_fp64(const Plan& P, const DevPlan& D, const double* L, const double* Dinv, int nrhs, double* X,
                      const double* B, int ld, double* W, double* part, int* flags, int* epoch, int* status,
                      cudaStream_t st) {
  return launch_solve<double>(P, D, L, Dinv, nrhs, X, B, ld, W, part, flags, epoch, status, st);
}

int launch_solve_fp32(const Plan& P, const DevPlan& D, const float* L, const float* Dinv, int nrhs, float* X,
                      const float* B, int ld, float* W, float* part, int* flags, int* epoch, int* status,
                      cudaStream_t st) {
  return launch_solve<float>(P, D, L, Dinv, nrhs, X, B, ld, W, part, flags, epoch, status, st);
}

}  // namespace tb

// ------------------------------------------------------------------------
// Solve without any allocation.
//
// Some callers must not allocate device memory: a serving thread that works
// inside a fixed, pre-reserved memory budget it may not grow; a latency-
// critical thread that may not call cudaMalloc/cudaFree because they can
// synchronise the device and stall every other stream; a host framework whose
// caching allocator already holds the rest of the GPU's memory.  They can
// still solve with an existing factor: taucs_b200_solve_device_noalloc keeps
// the solve's work vectors, handshake flags and status word in the one static
// device array below instead of the factor's own buffers.  It is the same
// level-scheduled solve as taucs_b200_solve_device, run one right-hand side
// per pass.  taucs_b200_solve_device_noalloc_status reads the status word.
// ------------------------------------------------------------------------

namespace tb {

constexpr size_t NOALLOC_W_DOUBLES = size_t(4) << 20;   // work vectors: 4 Mi doubles (32 MiB)
constexpr size_t NOALLOC_FLAGS = 16384;                 // handshake flags of the big fronts
constexpr size_t NOALLOC_DOUBLES = NOALLOC_W_DOUBLES + NOALLOC_FLAGS / 2 + 32;

// Every GPU that loads this library holds this array (about 32 MiB) until
// the process exits; all calls on a device share it.
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[256];

// Device address of the static array on the current device, looked up once
// per device (the name is only a host-side stand-in for it).
static int noalloc_scratch(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 256) {
    set_error(std::string("taucs_b200_solve_device_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    return -1;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error(std::string("taucs_b200_solve_device_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return -1;
    }
    g_noalloc_ptr[dev] = (double*) p;
  }
  *out = g_noalloc_ptr[dev];
  return 0;
}

// one right-hand side, work vectors at stride 1 (f doubles per front)
static int launch_solve_noalloc(const Plan& P, const DevPlan& D, const double* L, const double* Dinv, double* X,
                                const double* B,
                                int ld, double* W, int* flags, int* epoch, int* status, cudaStream_t st) {
  solve_attrs<double>();
  const int ef = ++*epoch;
  for (int h = 0; h < P.n_levels; h++) {
    const LevelPlan& LP = P.levels[h];
    const int ns = (int) LP.small_fronts.size();
    if (ns > 0) {
      k_fwd<double, 1, 256><<<ns, 256, 0, st>>>(D.small_list + D.small_off[h], ns, D.fronts, D.children, D.maps, D.rows, L, B, ld,
                                   W, 1);
      count_launch();
    }
    const int nb = (int) LP.solve_fwd_blocks.size();
    if (nb > 0) {
      k_fwd_big<double, 1, 1, FWD_ALL><<<nb, 128, fwd_smem<double, FWD_ALL>(), st>>>(
          D.sfwd + D.sfwd_off[h], D.fronts, D.children, D.maps, D.rows, L, Dinv, B, ld, W, 1, flags, ef, status);
      count_launch();
    }
  }
  const int eb = ++*epoch;
  for (int h = P.n_levels - 1; h >= 0; h--) {
    const LevelPlan& LP = P.levels[h];
    const int nb = (int) LP.solve_bwd_blocks.size();
    if (nb > 0) {
      k_gather_upd<double, 1><<<(int) LP.solve_fwd_blocks.size(), 128, 0, st>>>(D.sfwd + D.sfwd_off[h], D.fronts, D.rows,
                                                                         X, ld, W, 1);
      count_launch();
      k_bwd_big<double, 1, 1, false><<<nb, 128, bwd_smem<double, 1>(), st>>>(D.sbwd + D.sbwd_off[h], D.fronts, D.rows, L, Dinv, X, ld, W, nullptr, 1,
                                                 flags, eb, status);
      count_launch();
    }
    const int ns = (int) LP.small_fronts.size();
    if (ns > 0) {
      k_bwd<double, 1, 256><<<ns, 256, 0, st>>>(D.small_list + D.small_off[h], ns, D.fronts, D.rows, L, X, ld, W, 1);
      count_launch();
    }
  }
  return (int) cudaGetLastError();
}

}  // namespace tb

extern "C" int taucs_b200_solve_device_noalloc(void* vL, int nrhs, double* d_X, const double* d_B, int ld) {
  using namespace tb;
  Factor* F = (Factor*) vL;
  if (!F || nrhs < 0 || ld < F->n || (nrhs > 0 && (!d_X || !d_B))) {
    set_error("taucs_b200_solve_device_noalloc: bad arguments");
    return -1;
  }
  const Plan& P = F->plan;
  if ((size_t) P.v_len > NOALLOC_W_DOUBLES || (size_t) P.n_blk > NOALLOC_FLAGS) {
    char msg[320];
    snprintf(msg, sizeof msg,
             "taucs_b200_solve_device_noalloc: this factor needs %lld doubles of work vectors and %d flags; "
             "the static scratch holds %zu doubles and %zu flags (use taucs_b200_solve_device)",
             (long long) P.v_len, P.n_blk, NOALLOC_W_DOUBLES, NOALLOC_FLAGS);
    set_error(msg);
    return -1;
  }
  if (!F->has_numeric || !F->dev_ready) {
    set_error("taucs_b200_solve_device_noalloc: the factor has no numeric part");
    return -1;
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev != F->device) {
    set_error("taucs_b200_solve_device_noalloc: the current device is not the one the factor lives on");
    return -1;
  }
  if (nrhs == 0) return 0;
  double* base = nullptr;
  if (noalloc_scratch(&base)) return -1;
  double* W = base;
  int* flags = (int*) (base + NOALLOC_W_DOUBLES);
  int* status = flags + NOALLOC_FLAGS;
  cudaStream_t st = current_stream();
  // the array keeps whatever the previous call left: the flags and the status
  // word must start at zero, the work vectors are written before being read
  cudaError_t e = cudaMemsetAsync(flags, 0, sizeof(int) * (size_t) P.n_blk, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, sizeof(int), st);
  if (e != cudaSuccess) {
    set_error(std::string("taucs_b200_solve_device_noalloc: ") + cudaGetErrorString(e));
    return -1;
  }
  int epoch = 0;
  for (int q = 0; q < nrhs; q++) {
    e = (cudaError_t) launch_solve_noalloc(P, F->dp, F->dL, F->dDinv, d_X + (size_t) q * ld, d_B + (size_t) q * ld, ld, W,
                                           flags, &epoch, status, st);
    if (e != cudaSuccess) {
      set_error(std::string("taucs_b200_solve_device_noalloc: ") + cudaGetErrorString(e));
      return -1;
    }
  }
  return 0;
}

// Status of the no-alloc solves issued on the current device: waits for the
// current stream, then reads the status word that those solves share.
extern "C" int taucs_b200_solve_device_noalloc_status(void) {
  using namespace tb;
  double* base = nullptr;
  if (noalloc_scratch(&base)) return -1;
  const int* status = (const int*) (base + NOALLOC_W_DOUBLES) + NOALLOC_FLAGS;
  cudaError_t e = cudaStreamSynchronize(current_stream());
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, status, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    set_error(std::string("taucs_b200_solve_device_noalloc_status: ") + cudaGetErrorString(e));
    return -1;
  }
  if (h != 0) {
    set_error("taucs_b200_solve_device_noalloc: a bounded wait between thread blocks timed out; "
              "the solution is not valid");
    return -1;
  }
  return 0;
}

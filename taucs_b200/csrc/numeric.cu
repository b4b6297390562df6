// FP64 multifrontal numeric factorization on sm_100a.
//
// The reference factors one front at a time in a depth-first recursion
// (src/taucs_sn_llt.c:1829-1977): calloc F1/F2/U, extend-add each child
// (:1200-1240), assemble A's columns (:1099-1119), then LAPACK/BLAS POTRF
// (:1131), TRSM (:1150) and SYRK (:1180).  Here every front of one level of
// the supernodal tree is processed by the same launches:
//
//   k_small_persistent  the small fronts with only small fronts below them,
//                   all levels in one launch from a device-side queue;
//   k_small_front   the other fronts of order <= SMALL_F_MAX: one CTA builds the whole
//                   front in shared memory (zero + assemble + extend-add),
//                   factors it (right-looking partial Cholesky of the first s
//                   columns, i.e. POTRF+TRSM+SYRK fused) and writes the panel
//                   and the update matrix once;
//   k_build         larger fronts: one CTA per 128x32 tile of the front's lower
//                   part gathers A's entries (shared-memory atomic adds:
//                   duplicate entries are summed) and the children's update
//                   matrices in a fixed child order into shared memory and
//                   writes the tile once;
//   k_leaf          blocked partial Cholesky, step kb: one launch factors
//                   the 64x64 diagonal block and applies it to every row
//                   below it (one CTA per 64-row slab, each factoring the
//                   diagonal block itself);
//   k_gemm          C -= A B^T on DMMA (mma.sync m16n8k8 f64) tiles: the
//                   panel updates of a recursive (left half, GEMM, right
//                   half) panel factorization, and the update matrix
//                   U -= L21 L21^T with k = s at the end;
//   k_dinv          after all levels, the inverses of every big front's
//                   64x64 diagonal blocks (used by the solve).
//
// Every kernel first reads the status word and returns when an earlier front
// hit a nonpositive pivot; the smallest failing global column is recorded
// with atomicMin (the reference reports the failing column, :1139-1145).
#include <climits>
#include <cstdio>
#include <cuda_fp16.h>

#include "kernels.h"

namespace tb {

namespace {

__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }

__device__ __forceinline__ bool failed(const int* status) {
  return *(volatile const int*) status != INT_MAX;
}

__global__ void k_init_status(int* status) { *status = INT_MAX; }

// ------------------------------------------------------------ small fronts

// One small front by one CTA (128 threads) in shared memory W (f x f): zero,
// assemble A's columns, extend-add the children's update matrices in child
// order, partial Cholesky of the first s columns, then write the panel and
// the update matrix.  Every thread returns together; on a nonpositive pivot
// the front's global column is recorded and it returns early.
template <typename T>
__device__ void small_front(const FrontDesc& F, const FrontDesc* __restrict__ fronts, T* W,
                            const int* __restrict__ children,
                            const int* __restrict__ maps, const int* __restrict__ rows,
                            const int* __restrict__ acol_ptr, const int* __restrict__ a_rows,
                            const int* __restrict__ a_idx, const T* __restrict__ vals, T* __restrict__ L,
                            T* __restrict__ U, int* status) {
  const int f = F.f, s = F.s, m = f - s;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;

  for (int k = tid; k < f * f; k += nt) W[k] = 0.0;
  __syncthreads();
  // A's columns, one thread per column (duplicate rows add in order), the
  // entries four at a time with their loads issued together
  for (int c = tid; c < s; c += nt) {
    int e = __ldg(acol_ptr + F.acol_off + c);
    const int e1 = __ldg(acol_ptr + F.acol_off + c + 1);
    for (; e < e1; e += 4) {
      int r[4];
      T v[4];
#pragma unroll
      for (int q = 0; q < 4; q++) r[q] = e + q < e1 ? __ldg(a_rows + e + q) : -1;
#pragma unroll
      for (int q = 0; q < 4; q++) v[q] = e + q < e1 ? __ldg(vals + __ldg(a_idx + e + q)) : T(0);
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (r[q] >= 0) W[r[q] + c * f] += v[q];
    }
  }
  __syncthreads();
  // the children's update matrices in child order: warp w takes the child's
  // columns w + nw u (eight per pass), lane l its rows l + 32 v; a pass
  // issues all its loads before its adds
  constexpr int SJ = 8, SV = (SMALL_F_MAX + 31) / 32;
  for (int ci = F.child_begin; ci < F.child_end; ci++) {
    const FrontDesc C = fronts[children[ci]];
    const int mc = C.f - C.s;
    const int* mp = maps + C.map_off;
    const T* Uc = U + C.u_off;
    int pi[SV];
#pragma unroll
    for (int v = 0; v < SV; v++) pi[v] = lane + 32 * v < mc ? __ldg(mp + lane + 32 * v) : -1;
    for (int j0 = warp; j0 < mc; j0 += nw * SJ) {
      int pj[SJ];
      T val[SJ][SV];
#pragma unroll
      for (int u = 0; u < SJ; u++) {
        const int j = j0 + nw * u;
        pj[u] = j < mc ? __ldg(mp + j) * f : -1;
#pragma unroll
        for (int v = 0; v < SV; v++) {
          const int i = lane + 32 * v;
          val[u][v] = (j < mc && i >= j && i < mc) ? __ldg(Uc + i + (size_t) j * mc) : T(0);
        }
      }
#pragma unroll
      for (int u = 0; u < SJ; u++) {
        const int j = j0 + nw * u;
#pragma unroll
        for (int v = 0; v < SV; v++) {
          const int i = lane + 32 * v;
          if (pj[u] >= 0 && i >= j && i < mc) W[pi[v] + pj[u]] += val[u][v];
        }
      }
    }
    __syncthreads();
  }
  // column j stays unscaled in W: its multipliers W[i][j] rj are formed
  // where they are used (the same products as scaling it in place), and the
  // panel is scaled by rjs[] on its way out -- one barrier per column
  __shared__ T rjs[SMALL_F_MAX];
  constexpr int KU = 4;
  for (int j = 0; j < s; j++) {
    const T d = W[j + j * f];
    if (!(d > 0.0)) {
      if (tid == 0) atomicMin(status, rows[F.rows_off + j]);
      return;
    }
    const T rj = rsqrt_t(d);
    if (tid == 0) rjs[j] = rj;
    // warp w takes columns k0 + nw u (u < KU) of the trailing part, lane l
    // the rows from k0 + l; each pass loads before it stores
    const T* wj = W + j * f;
    for (int k0 = j + 1 + warp; k0 < f; k0 += nw * KU) {
      T lk[KU];
#pragma unroll
      for (int u = 0; u < KU; u++) {
        const int k = k0 + nw * u;
        lk[u] = k < f ? wj[k] * rj : T(0);
      }
      for (int i = k0 + lane; i < f; i += 32) {
        const T li = wj[i] * rj;
        T w[KU];
#pragma unroll
        for (int u = 0; u < KU; u++) {
          const int k = k0 + nw * u;
          w[u] = (k < f && i >= k) ? W[i + k * f] : T(0);
        }
#pragma unroll
        for (int u = 0; u < KU; u++) {
          const int k = k0 + nw * u;
          if (k < f && i >= k) W[i + k * f] = w[u] - li * lk[u];
        }
      }
    }
    __syncthreads();
  }
  T* Lp = L + F.l_off;
  for (int k = tid; k < f * s; k += nt) Lp[k] = W[k] * rjs[k / f];
  if (m > 0) {
    T* Up = U + F.u_off;
    for (int k = tid; k < m * m; k += nt) {
      const int i = k % m, c = k / m;
      Up[k] = W[(s + i) + (s + c) * f];
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(128)
k_small_front(const int* __restrict__ list, const FrontDesc* __restrict__ fronts,
              const int* __restrict__ children, const int* __restrict__ maps,
              const int* __restrict__ rows, const int* __restrict__ acol_ptr,
              const int* __restrict__ a_rows, const int* __restrict__ a_idx,
              const T* __restrict__ vals, T* __restrict__ L, T* __restrict__ U,
              int* status) {
  extern __shared__ __align__(16) unsigned char smraw[];
  if (failed(status)) return;
  small_front<T>(fronts[list[blockIdx.x]], fronts, reinterpret_cast<T*>(smraw), children, maps, rows, acol_ptr, a_rows,
                 a_idx, vals, L, U, status);
}

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// One front of order f <= SMALL_WARP_F by one warp: the front is assembled
// in the warp's shared rows Ws (row-major, one padded row per front row),
// then lane i holds row i in registers for the partial Cholesky of the first
// s columns (column j's multipliers passed by shuffles; the same operations
// as small_front), and writes the panel and the update matrix with zeros
// above the diagonal.  On a nonpositive pivot the front's global column is
// recorded and the warp returns early.
template <typename T>
__device__ void warp_front(const FrontDesc& F, const FrontDesc* __restrict__ fronts, T (*Ws)[SMALL_WARP_F + 1],
                           const int* __restrict__ children, const int* __restrict__ maps,
                           const int* __restrict__ rows, const int* __restrict__ acol_ptr,
                           const int* __restrict__ a_rows, const int* __restrict__ a_idx,
                           const T* __restrict__ vals, T* __restrict__ L, T* __restrict__ U, int* status) {
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int WF = SMALL_WARP_F;
  const int f = F.f, s = F.s, m = f - s;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int c = 0; c < WF; c++) Ws[lane][c] = T(0);
  __syncwarp();
  // A's column `lane` (one lane per column: duplicate rows add in order)
  if (lane < s) {
    int e = __ldg(acol_ptr + F.acol_off + lane);
    const int e1 = __ldg(acol_ptr + F.acol_off + lane + 1);
    for (; e + 4 <= e1; e += 4) {
      int r[4];
      T v[4];
#pragma unroll
      for (int q = 0; q < 4; q++) r[q] = __ldg(a_rows + e + q);
#pragma unroll
      for (int q = 0; q < 4; q++) v[q] = __ldg(vals + __ldg(a_idx + e + q));
#pragma unroll
      for (int q = 0; q < 4; q++) Ws[r[q]][lane] += v[q];
    }
    for (; e < e1; e++) Ws[__ldg(a_rows + e)][lane] += __ldg(vals + __ldg(a_idx + e));
  }
  // the children's update matrices in child order: lane i takes the child's
  // row i, all its loads before its adds (distinct rows: no conflicts)
  for (int ci = F.child_begin; ci < F.child_end; ci++) {
    const FrontDesc C = fronts[children[ci]];
    const int mc = C.f - C.s;
    const T* Uc = U + C.u_off;
    const int pi = lane < mc ? __ldg(maps + C.map_off + lane) : 0;
    T v[WF];
#pragma unroll
    for (int j = 0; j < WF; j++) v[j] = (j <= lane && lane < mc) ? __ldg(Uc + lane + (size_t) j * mc) : T(0);
    __syncwarp();
#pragma unroll
    for (int j = 0; j < WF; j++) {
      if (j >= mc) break;
      const int pj = __shfl_sync(FULL, pi, j);
      if (j <= lane && lane < mc) Ws[pi][pj] += v[j];
    }
  }
  __syncwarp();
  T w[WF];
#pragma unroll
  for (int c = 0; c < WF; c++) w[c] = Ws[lane][c];
  __syncwarp();
  // pivot j in a rolled loop: the row is rotated left by one entry per
  // pivot, so column j is always w[0] and column j + k is w[k] (one body of
  // row code instead of one per pivot keeps the kernel cache-resident); the
  // finished column goes straight to the panel
  T* Lp = L + F.l_off;
#pragma unroll 1
  for (int j = 0; j < s; j++) {
    const T d = __shfl_sync(FULL, w[0], j);
    if (!(d > T(0))) {
      if (lane == 0) atomicMin(status, rows[F.rows_off + j]);
      return;
    }
    const T rj = rsqrt_t(d);
    const T lij = lane > j ? w[0] * rj : (lane == j ? d * rj : T(0));
    if (lane < f) Lp[lane + (size_t) j * f] = lij;
#pragma unroll
    for (int k = 1; k < WF; k++) {
      const T lkj = __shfl_sync(FULL, lij, (j + k) & (WF - 1));
      if (lane >= j + k && j + k < f) w[k] -= lij * lkj;
    }
#pragma unroll
    for (int k = 0; k < WF - 1; k++) w[k] = w[k + 1];
    w[WF - 1] = T(0);
  }
  // after s rotations w[k] is the row's column s + k
  if (lane < f && lane >= s) {
    T* Up = U + F.u_off;
#pragma unroll
    for (int k = 0; k < WF; k++)
      if (k < m) Up[(lane - s) + (size_t) k * m] = k <= lane - s ? w[k] : T(0);
  }
}

// The first part of the persistent set (fronts whose subtree has only
// fronts of order <= SMALL_WARP_F), in one launch of resident CTAs of four
// warps: each warp takes the next front from a device-side queue (tasks
// t0 .. t1-1 in level order), waits until the front's children are done
// (pending count), factors it (warp_front) and counts itself off at its
// parent -- also when the parent is in the second part, whose launch runs
// after this one.  Waits are bounded (NUMERIC_TIMEOUT); after a nonpositive
// pivot anywhere the remaining fronts are only counted off.
template <typename T>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 6 : 4)
k_small_warp(const int* __restrict__ tasks, int t0, int t1, const int* __restrict__ parent_task, int* pending,
             int* next, const FrontDesc* __restrict__ fronts, const int* __restrict__ children,
             const int* __restrict__ maps, const int* __restrict__ rows, const int* __restrict__ acol_ptr,
             const int* __restrict__ a_rows, const int* __restrict__ a_idx, const T* __restrict__ vals,
             T* __restrict__ L, T* __restrict__ U, int* status) {
  __shared__ T Ws_all[4][SMALL_WARP_F][SMALL_WARP_F + 1];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  for (;;) {
    int t = 0;
    if (lane == 0) t = t0 + atomicAdd(next, 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= t1) break;
    int skip = 0;
    if (lane == 0) {
      int it = 0;
      while (ld_acquire_gpu(pending + t) != 0) {
        if (++it > (1 << 22)) {
          atomicMin(status, NUMERIC_TIMEOUT);
          break;
        }
        __nanosleep(32);
      }
      skip = failed(status);
    }
    skip = __shfl_sync(0xffffffffu, skip, 0);
    if (!skip)
      warp_front<T>(fronts[tasks[t]], fronts, Ws_all[wi], children, maps, rows, acol_ptr, a_rows, a_idx, vals, L,
                    U, status);
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      const int pt = parent_task[t];
      if (pt >= 0) atomicSub(pending + pt, 1);
    }
  }
}

// The small fronts whose whole subtree is small (Plan::pers_fronts), in one
// launch of resident CTAs: each CTA takes the next front from a device-side
// queue (an atomic counter over the fronts in level order), waits until the
// front's children are done (its pending count, decremented by each child's
// CTA after its update matrix is written), factors it, and marks it done
// for its parent.  A front is only taken after all fronts before it in level
// order were taken by running CTAs, so every wait ends; the waits are bounded
// all the same (NUMERIC_TIMEOUT).  After a nonpositive pivot anywhere the
// remaining fronts are only marked done.
template <typename T>
__global__ void __launch_bounds__(128)
k_small_persistent(const int* __restrict__ tasks, int t0, int t1, const int* __restrict__ parent_task, int* pending,
                   int* next, const FrontDesc* __restrict__ fronts, const int* __restrict__ children,
                   const int* __restrict__ maps, const int* __restrict__ rows, const int* __restrict__ acol_ptr,
                   const int* __restrict__ a_rows, const int* __restrict__ a_idx, const T* __restrict__ vals,
                   T* __restrict__ L, T* __restrict__ U, int* status) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ int t_s, skip_s;
  T* W = reinterpret_cast<T*>(smraw);
  for (;;) {
    if (threadIdx.x == 0) t_s = t0 + atomicAdd(next, 1);
    __syncthreads();
    const int t = t_s;
    if (t >= t1) break;
    if (threadIdx.x == 0) {
      int it = 0;
      while (ld_acquire_gpu(pending + t) != 0) {
        if (++it > (1 << 22)) {
          atomicMin(status, NUMERIC_TIMEOUT);
          break;
        }
        __nanosleep(64);
      }
      skip_s = failed(status);
    }
    __syncthreads();
    if (!skip_s)
      small_front<T>(fronts[tasks[t]], fronts, W, children, maps, rows, acol_ptr, a_rows, a_idx, vals, L, U, status);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const int pt = parent_task[t];
      if (pt >= 0) atomicSub(pending + pt, 1);
    }
  }
}

// --------------------------------------------------------------- front build

// threads of a build CTA: four warps, sixteen CTAs resident per SM
constexpr int BUILD_THREADS = 128;

// The child records of the build tiles, once per plan: CTA t (four warps)
// finds for each child of tile t's front the child's columns and rows that
// land in the tile, the four bounds searched at once (32-ary warp searches
// of the child's increasing map).
__global__ void __launch_bounds__(128)
k_tile_ranges(const Tile* __restrict__ tiles, const FrontDesc* __restrict__ fronts, const int* __restrict__ children,
              const int* __restrict__ maps, TileChild* __restrict__ rec) {
  const Tile tl = tiles[blockIdx.x];
  const FrontDesc F = fronts[tl.front];
  const int f = F.f, s = F.s, m = f - s;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int R0, C0, nr, nc;
  if (tl.c0 >= 0) {
    R0 = tl.r0; C0 = tl.c0;
    nr = min(BUILD_TR, f - R0); nc = min(BUILD_TC, s - C0);
  } else {
    const int uc0 = -1 - tl.c0;
    R0 = s + tl.r0; C0 = s + uc0;
    nr = min(BUILD_TR, m - tl.r0); nc = min(BUILD_TC, m - uc0);
  }
  for (int ci = F.child_begin; ci < F.child_end; ci++) {
    const FrontDesc C = fronts[children[ci]];
    const int mc = C.f - C.s;
    const int key = warp == 0 ? C0 : warp == 1 ? C0 + nc : warp == 2 ? R0 : R0 + nr;
    const int r = warp_lower_bound(maps + C.map_off, mc, key);
    TileChild* out = rec + tl.ch_off + (ci - F.child_begin);
    if (lane == 0) {
      int* o = &out->ja;
      o[warp] = r;   // ja, jb, ia, ib in warp order
      if (warp == 0) {
        out->map_off = C.map_off;
        out->mc = mc;
        out->u_off = C.u_off;
      }
    }
  }
}


template <typename T>
__global__ void __launch_bounds__(BUILD_THREADS)
k_build(const Tile* __restrict__ tiles, const TileChild* __restrict__ tile_ch, const FrontDesc* __restrict__ fronts,
        const int* __restrict__ maps,
        const int* __restrict__ acol_ptr, const int* __restrict__ a_rows,
        const int* __restrict__ a_idx, const T* __restrict__ vals,
        T* __restrict__ L, T* __restrict__ U, const int* status) {
  __shared__ T W[BUILD_TR * BUILD_TC];
  if (failed(status)) return;
  const Tile tl = tiles[blockIdx.x];
  const FrontDesc F = fronts[tl.front];
  const int f = F.f, s = F.s, m = f - s;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const bool panel = tl.c0 >= 0;
  int R0, C0, nr, nc;
  if (panel) {
    R0 = tl.r0; C0 = tl.c0;
    nr = min(BUILD_TR, f - R0); nc = min(BUILD_TC, s - C0);
  } else {
    const int uc0 = -1 - tl.c0;
    R0 = s + tl.r0; C0 = s + uc0;
    nr = min(BUILD_TR, m - tl.r0); nc = min(BUILD_TC, m - uc0);
  }
  for (int k = tid; k < BUILD_TR * BUILD_TC; k += nt) W[k] = 0.0;
  __syncthreads();
  if (panel) {
    // A's entries of the tile's columns: thread (column c, slot q) takes the
    // column's entries q, q + 8, ... -- the loads of all slots in flight at
    // once; the adds are atomic, as a column may list a row more than once
    // (duplicates are summed)
    const int c = tid % BUILD_TC, q = tid / BUILD_TC;
    constexpr int NQS = BUILD_THREADS / BUILD_TC;
    int e = 0, e1 = 0;
    if (c < nc) {
      e = __ldg(acol_ptr + F.acol_off + C0 + c) + q;
      e1 = __ldg(acol_ptr + F.acol_off + C0 + c + 1);
    }
    for (; e < e1; e += NQS) {
      const int r = __ldg(a_rows + e) - R0;
      if (r >= 0 && r < nr) atomicAdd(&W[r + c * BUILD_TR], __ldg(vals + __ldg(a_idx + e)));
    }
    __syncthreads();
  }
  // the children's shares, in child order, from the tile's records (found
  // once per plan); every load of a child's share is issued before the
  // first add (the children's update matrices were written by earlier
  // launches)
  const int nch = F.child_end - F.child_begin;
  for (int c = 0; c < nch; c++) {
    const TileChild R = tile_ch[tl.ch_off + c];
    const int ja = R.ja, jb = R.jb, ia = R.ia, ib = R.ib;
    if (ja >= jb || ia >= ib) continue;
    const int mc = R.mc;
    const int* mp = maps + R.map_off;
    const T* Uc = U + R.u_off;
    // warp w takes the child's columns ja + w + NW u, lane l its rows
    // ia + l + 32v
    constexpr int NW = BUILD_THREADS / 32, JU = (BUILD_TC + NW - 1) / NW, IU = BUILD_TR / 32;
    int pi[IU], pj[JU];
    T val[JU][IU];
#pragma unroll
    for (int v = 0; v < IU; v++) {
      const int i = ia + lane + 32 * v;
      pi[v] = (i < ib) ? __ldg(mp + i) - R0 : -1;
    }
#pragma unroll
    for (int u = 0; u < JU; u++) {
      const int j = ja + warp + NW * u;
      const bool jv = j < jb;
      pj[u] = jv ? (__ldg(mp + j) - C0) * BUILD_TR : -1;
#pragma unroll
      for (int v = 0; v < IU; v++) {
        const int i = ia + lane + 32 * v;
        val[u][v] = (jv && i < ib && i >= j) ? __ldg(Uc + (size_t) j * mc + i) : T(0);
      }
    }
#pragma unroll
    for (int u = 0; u < JU; u++)
#pragma unroll
      for (int v = 0; v < IU; v++) {
        const int i = ia + lane + 32 * v, j = ja + warp + NW * u;
        if (pj[u] >= 0 && pi[v] >= 0 && i >= j) W[pi[v] + pj[u]] += val[u][v];
      }
    __syncthreads();
  }
  if (panel) {
    T* dst = L + F.l_off;
    for (int k = tid; k < BUILD_TR * BUILD_TC; k += nt) {
      const int r = k % BUILD_TR, c = k / BUILD_TR;
      if (r < nr && c < nc) dst[(R0 + r) + (size_t) (C0 + c) * f] = W[k];
    }
  } else {
    T* dst = U + F.u_off;
    for (int k = tid; k < BUILD_TR * BUILD_TC; k += nt) {
      const int r = k % BUILD_TR, c = k / BUILD_TR;
      if (r < nr && c < nc) dst[(R0 - s + r) + (size_t) (C0 - s + c) * m] = W[k];
    }
  }
}

// ---------------------------------------------------------- panel leaves

// Panel leaf, step kb: the columns [kb, kb + w) of the level's big fronts, w =
// min(64, s - kb), factored and applied to every row below them in ONE
// launch (the reference's POTRF :1131 and TRSM :1150 on a 64-column piece).
// CTA x of front y owns the 64 rows [kb + w + 64 x, ...) below the diagonal
// block.  Every CTA of the launch reads the diagonal block as it was before
// the step, so CTA 0 parks the factored block in the block's slot of the
// inverse array rather than in the panel; k_dinv moves it into the panel
// after the factorization and replaces it there by its inverse.  Every CTA
// factors the 64x64 diagonal block itself -- a redundant Cholesky instead of
// waiting for the CTA that owns it.  Each thread holds one row in registers
// (threads 0-63 the slab's rows, 64-127 the diagonal block's), and the block
// goes in four 16-column steps: the warp whose lanes hold the piece's rows
// factors the 16x16 piece by shuffles, every row below it solves against
// the piece by substitution, and every row updates its columns to the right
// from the diagonal block's new rows (published row-major in shared memory).
// The inverses of the 64x64 diagonal blocks, which the solve applies, are
// formed afterwards for all fronts at once (k_dinv).  Nothing reads a
// diagonal block of the panel between its leaf and k_dinv: the later
// products read rows below it only.
constexpr int LLD = PANEL_NB + 4;   // padded column stride of k_dinv's blocks in shared memory
constexpr int LQ = 16;              // column step inside a leaf
constexpr int LYD = LQ + 1;         // column stride of a 16x16 inverse

template <typename T>
constexpr size_t dinv_smem() { return (2 * PANEL_NB * LLD + (PANEL_NB / LQ) * LQ * LYD) * sizeof(T); }

// Inverse of the lower-triangular 16x16 factor held one row per lane (a[k] =
// L[i][k], i = lane & 15, k <= i) into Y (column-major, ld LYD): lane t forms
// column t by forward substitution, reading L[r][k] by broadcast shuffles.
template <typename T>
__device__ __forceinline__ void warp_inv16_rows(const T (&a)[LQ], T* Y) {
  const int i = threadIdx.x & 15;
  T y[LQ];
#pragma unroll
  for (int r = 0; r < LQ; r++) {
    T acc = (r == i) ? T(1) : T(0);
#pragma unroll
    for (int k = 0; k < r; k++) acc -= __shfl_sync(0xffffffffu, a[k], r) * y[k];
    const T lrr = __shfl_sync(0xffffffffu, a[r], r);
    y[r] = (r >= i) ? acc * (T(1) / lrr) : T(0);
  }
  if ((threadIdx.x & 31) < LQ) {
#pragma unroll
    for (int r = 0; r < LQ; r++) Y[r + i * LYD] = y[r];
  }
}

// One pivot J of the 16x16 warp Cholesky of the leaf, unrolled through the
// recursion so that every index into the row held in registers is a
// constant: lane base + i holds row i of the piece (a[k] = L[i][k], k <= i);
// the pivot comes by shuffle, the column is scaled by rsqrt(pivot), and the
// columns right of J take the right-looking update.  Lanes outside the piece
// run along on values that are never written back.
template <typename T, int J>
struct CholStep {
  __device__ __forceinline__ static void run(T (&a)[LQ], int i, int base, int& bad) {
    const T d = __shfl_sync(0xffffffffu, a[J], base + J);
    if (!(d > T(0)) && bad < 0) bad = J;
    const T r = rsqrt_t(d);
    a[J] = (i == J) ? d * r : a[J] * r;
#pragma unroll
    for (int k = J + 1; k < LQ; k++) {
      const T lkj = __shfl_sync(0xffffffffu, a[J], base + k);
      if (i >= k) a[k] -= a[J] * lkj;
    }
    CholStep<T, J + 1>::run(a, i, base, bad);
  }
};
template <typename T>
struct CholStep<T, LQ> {
  __device__ __forceinline__ static void run(T (&)[LQ], int, int, int&) {}
};

// The split copy of one slab row for the tensor-core products: chunks of CW
// columns, hi and lo parts, written for chunk indices [0, nch) of the leaf
// (columns past w are zero: the front's last leaf pads K to the products'
// stage width).
template <int CW>
__device__ __forceinline__ void leaf_split_row(const float (&rw)[PANEL_NB], int w, int nch, unsigned char* base,
                                               int64_t part, int64_t kc0, int64_t rg, int r) {
  constexpr int CMAX = PANEL_NB / CW + 4;
#pragma unroll
  for (int c = 0; c < CMAX; c++) {
    if (c >= nch) break;
    const int64_t o = ((kc0 + c) * rg + (r >> 3)) * 128 + (r & 7) * 16;
    if (CW == 4) {
      unsigned h[4], l[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int k = c * 4 + q;
        const float x = (k < PANEL_NB && k < w) ? rw[k < PANEL_NB ? k : 0] : 0.0f;
        h[q] = __float_as_uint(x) & 0xffffe000u;
        l[q] = __float_as_uint(x - __uint_as_float(h[q]));
      }
      *reinterpret_cast<uint4*>(base + o) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(base + part + o) = make_uint4(l[0], l[1], l[2], l[3]);
    } else {
      unsigned short h[8], l[8];
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const int k = c * 8 + q;
        const float x = (k < PANEL_NB && k < w) ? rw[k < PANEL_NB ? k : 0] : 0.0f;
        const __half hh = __float2half_rn(x);
        h[q] = __half_as_ushort(hh);
        l[q] = __half_as_ushort(__float2half_rn((x - __half2float(hh)) * 2048.0f));
      }
      uint4 vh, vl;
      vh.x = h[0] | (unsigned) h[1] << 16; vh.y = h[2] | (unsigned) h[3] << 16;
      vh.z = h[4] | (unsigned) h[5] << 16; vh.w = h[6] | (unsigned) h[7] << 16;
      vl.x = l[0] | (unsigned) l[1] << 16; vl.y = l[2] | (unsigned) l[3] << 16;
      vl.z = l[4] | (unsigned) l[5] << 16; vl.w = l[6] | (unsigned) l[7] << 16;
      *reinterpret_cast<uint4*>(base + o) = vh;
      *reinterpret_cast<uint4*>(base + part + o) = vl;
    }
  }
}
template <int CW>
__device__ __forceinline__ void leaf_split_row(const double (&)[PANEL_NB], int, int, unsigned char*, int64_t, int64_t,
                                               int64_t, int) {}

template <typename T, int SPF>
__global__ void __launch_bounds__(128)
k_leaf(const int* __restrict__ list, const FrontDesc* __restrict__ fronts, const int* __restrict__ rows,
       T* __restrict__ L, T* __restrict__ Dinv, float* __restrict__ sp, int kb, int* status) {
  // SPF: the split format of the copy for the tensor-core products (one
  // instantiation each: the fully unrolled row code is large)
  constexpr int sp_fmt = SPF;
  // Xt[buf][c][k]: the new L[c][c0 + k] of the diagonal block's rows c below
  // the current piece (row-major, 16-byte aligned rows, two buffers by piece
  // parity); Lp, rinv: the factored piece and its reciprocal diagonal
  constexpr int XLD = sizeof(T) == 4 ? LQ + 4 : LQ + 2;
  __shared__ __align__(16) T Xt[2][PANEL_NB][XLD];
  __shared__ T Lp[LQ][LQ + 1];
  __shared__ T rinv[LQ];
  __shared__ int bad_s;
  if (failed(status)) return;
  const FrontDesc F = fronts[list[blockIdx.y]];
  const int f = F.f, s = F.s;
  if (kb >= s) return;
  const int w = min(PANEL_NB, s - kb);
  const int r0 = kb + w + blockIdx.x * PANEL_NB;
  const int nr = max(0, min(PANEL_NB, f - r0));
  if (blockIdx.x > 0 && nr == 0) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // threads 0-63: the slab's rows; threads 64-127: the diagonal block's rows
  // (identity past w); each thread holds its row's 64 entries in registers
  const bool is_d = tid >= PANEL_NB;
  const int i = is_d ? tid - PANEL_NB : tid;
  T* P = L + F.l_off;
  T rw[PANEL_NB];
  {
    const size_t g = is_d ? (size_t) (kb + i) : (size_t) (r0 + i);
    const bool rv = is_d ? (i < w) : (i < nr);
#pragma unroll
    for (int c = 0; c < PANEL_NB; c++) {
      const bool in = rv && c < w && (!is_d || c <= i);
      rw[c] = in ? P[g + (size_t) (kb + c) * f] : ((is_d && c == i) ? T(1) : T(0));
    }
  }
  // the four 16-column pieces in a rolled loop over one body: the row is
  // rotated left by 16 entries after each piece, so the current piece is
  // always rw[0..15] and its trailing columns rw[16..63 - c0] (after the
  // fourth rotation the row is back in column order); one copy of the row
  // code instead of four keeps the kernel's instructions cache-resident
#pragma unroll 1
  for (int b = 0; b < PANEL_NB / LQ; b++) {
    const int c0 = b * LQ;
    // the piece's 16 rows are lanes base .. base + 15 of warp 2 + c0 / 32
    const int base = c0 % 32;
    if (warp == 2 + c0 / 32) {
      const int ii = lane - base;
      T a[LQ];
#pragma unroll
      for (int k = 0; k < LQ; k++) a[k] = (k <= ii) ? rw[k] : T(0);
      int bad = -1;
      CholStep<T, 0>::run(a, ii, base, bad);
      if (ii >= 0 && ii < LQ) {
        T dg = T(1);
#pragma unroll
        for (int k = 0; k < LQ; k++) {
          if (k <= ii) rw[k] = a[k];
          Lp[ii][k] = (k <= ii) ? a[k] : T(0);
          if (k == ii) dg = a[k];
        }
        rinv[ii] = T(1) / dg;
      }
      if (lane == 0) bad_s = bad;
    }
    __syncthreads();
    if (bad_s >= 0) {
      if (tid == 0 && blockIdx.x == 0 && c0 + bad_s < w) atomicMin(status, rows[F.rows_off + kb + c0 + bad_s]);
      return;
    }
    // rows below the piece: X L_p^T = M by substitution (in registers), the
    // diagonal block's rows also published for the update below
    const bool below = !is_d || i >= c0 + LQ;
    T x[LQ];
#pragma unroll
    for (int c = 0; c < LQ; c++) x[c] = rw[c];
    if (below) {
#pragma unroll
      for (int c = 0; c < LQ; c++) {
        x[c] *= rinv[c];
#pragma unroll
        for (int c2 = c + 1; c2 < LQ; c2++) x[c2] -= x[c] * Lp[c2][c];
      }
#pragma unroll
      for (int c = 0; c < LQ; c++) rw[c] = x[c];
      if (is_d) {
#pragma unroll
        for (int c = 0; c < LQ; c++) Xt[b & 1][i][c] = x[c];
      }
    }
    __syncthreads();
    // the columns right of the piece: rw[c] -= sum_k x[k] L[c0 + c][c0 + k].
    // A warp of the diagonal block stops at the last row it holds (the
    // columns past it are upper-triangle entries of all its rows, never
    // read): the warp that factors the next piece is on the chain and does
    // the least
    const int cmax = (is_d ? (warp - 2) * 32 + 31 : PANEL_NB - 1) - c0;
    if (below) {
#pragma unroll
      for (int c = LQ; c < PANEL_NB; c++) {
        if (c > cmax) break;
        const T* xr = Xt[b & 1][c0 + c];
        T acc = rw[c];
#pragma unroll
        for (int k = 0; k < LQ; k++) acc -= x[k] * xr[k];
        rw[c] = acc;
      }
    }
    // rotate left by one piece
#pragma unroll
    for (int k = 0; k < LQ; k++) x[k] = rw[k];
#pragma unroll
    for (int k = 0; k < PANEL_NB - LQ; k++) rw[k] = rw[k + LQ];
#pragma unroll
    for (int k = 0; k < LQ; k++) rw[PANEL_NB - LQ + k] = x[k];
  }
  if (is_d) {
    if (blockIdx.x == 0) {
      T* Dk = Dinv + F.dinv_off + (size_t) (kb / PANEL_NB) * PANEL_NB * PANEL_NB;
#pragma unroll
      for (int c = 0; c < PANEL_NB; c++) Dk[i + c * PANEL_NB] = (c <= i && i < w) ? rw[c] : T(0);
    }
    return;
  }
  if (i < nr) {
    const size_t g = (size_t) (r0 + i);
#pragma unroll
    for (int c = 0; c < PANEL_NB; c++)
      if (c < w) P[g + (size_t) (kb + c) * f] = rw[c];
    if (sizeof(T) == 4 && sp != nullptr && F.sp_off >= 0) {
      // the row's final values, split, into the split arena for the tensor-
      // core products; the front's last leaf also writes the zero columns
      // that pad K to the products' stage width
      const int64_t rg = sp_rgroups(f), part = sp_part_bytes(F, sp_fmt);
      unsigned char* base = reinterpret_cast<unsigned char*>(sp + F.sp_off);
      const int cw = sp_chunk_cols(sp_fmt);
      const int kc_end = (kb + w == s) ? (int) sp_kchunks(s, sp_fmt) : (kb + w) / cw;
      const int nch = kc_end - kb / cw;
      leaf_split_row<SPF ? 8 : 4>(rw, w, nch, base, part, kb / (SPF ? 8 : 4), rg, r0 + i);
    }
  }
}

// After the factorization, one CTA per 64x64 diagonal block of every big
// front: the factored block L_kk that its leaf parked in the block's slot of
// Dinv goes into the panel, and the slot receives L_kk^-1 (lower, zero
// beyond the block's width), which the solve applies.  Warp q inverts the
// 16x16 diagonal piece q; then warp b forms block column b below the
// diagonal, X_cb = -X_cc sum_{b<=k<c} L_ck X_kb.
template <typename T>
__global__ void __launch_bounds__(128)
k_dinv(const int2_* __restrict__ blocks, const FrontDesc* __restrict__ fronts, T* __restrict__ L,
       T* __restrict__ Dinv, const int* status) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* S = reinterpret_cast<T*>(smraw);   // L_kk, 64 x 64, ld LLD (identity beyond w)
  T* X = S + PANEL_NB * LLD;            // its inverse, ld LLD
  T* Tm = X + PANEL_NB * LLD;           // per warp: a 16x16 partial sum, ld LYD
  if (failed(status)) return;
  const int2_ bl = blocks[blockIdx.x];
  const FrontDesc F = fronts[bl.a];
  const int f = F.f, kb = bl.b * PANEL_NB;
  const int w = min(PANEL_NB, F.s - kb);
  T* P = L + F.l_off;
  T* Di = Dinv + F.dinv_off + (size_t) bl.b * PANEL_NB * PANEL_NB;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
#pragma unroll 8
  for (int t = 0; t < PANEL_NB * PANEL_NB / 128; t++) {
    const int e = tid + 128 * t, i = e % PANEL_NB, j = e / PANEL_NB;
    const T v = (i < w && j < w && i >= j) ? Di[e] : (i == j ? T(1) : T(0));
    S[i + j * LLD] = v;
    X[i + j * LLD] = T(0);
    if (i < w && j < w && i >= j) P[(kb + i) + (size_t) (kb + j) * f] = v;
  }
  __syncthreads();
  {
    const int q0 = warp * LQ, i = lane & 15;
    T a[LQ];
#pragma unroll
    for (int k = 0; k < LQ; k++) a[k] = (k <= i) ? S[(q0 + i) + (q0 + k) * LLD] : T(0);
    T* Yq = Tm + warp * LQ * LYD;
    warp_inv16_rows(a, Yq);
    __syncwarp();
    if (lane < LQ)
      for (int r = 0; r < LQ; r++) X[(q0 + r) + (q0 + lane) * LLD] = Yq[r + lane * LYD];
  }
  __syncthreads();
  if (warp < PANEL_NB / LQ - 1) {
    const int b0 = warp * LQ, t = lane & 15;
    T* Tw = Tm + warp * LQ * LYD;
    for (int c = warp + 1; c < PANEL_NB / LQ; c++) {
      const int c0 = c * LQ;
      // Tw[:, t] = sum_{k=b}^{c-1} L_ck X_kb[:, t]
      T acc[LQ];
#pragma unroll
      for (int r = 0; r < LQ; r++) acc[r] = T(0);
      for (int j = b0; j < c0; j++) {
        const T xj = X[j + (b0 + t) * LLD];
#pragma unroll
        for (int r = 0; r < LQ; r++) acc[r] += S[(c0 + r) + j * LLD] * xj;
      }
      __syncwarp();
      if (lane < LQ)
#pragma unroll
        for (int r = 0; r < LQ; r++) Tw[r + t * LYD] = acc[r];
      __syncwarp();
      // X_cb[:, t] = -X_cc Tw[:, t]
#pragma unroll
      for (int r = 0; r < LQ; r++) acc[r] = T(0);
      for (int j = 0; j < LQ; j++) {
        const T tj = Tw[j + t * LYD];
#pragma unroll
        for (int r = 0; r < LQ; r++) acc[r] += X[(c0 + r) + (c0 + j) * LLD] * tj;
      }
      if (lane < LQ)
#pragma unroll
        for (int r = 0; r < LQ; r++) X[(c0 + r) + (b0 + t) * LLD] = -acc[r];
      __syncwarp();
    }
  }
  __syncthreads();
  for (int e = tid; e < PANEL_NB * PANEL_NB; e += 128) {
    const int i = e % PANEL_NB, j = e / PANEL_NB;
    Di[e] = (i < w && j < w) ? X[i + j * LLD] : T(0);
  }
}

// ------------------------------------------------------------- DMMA GEMM

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool pred) {
  const unsigned saddr = (unsigned) __cvta_generic_to_shared(smem);
  const int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma16888(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

__device__ __forceinline__ void cp_async_t(double* smem, const double* gmem, bool pred) { cp_async8(smem, gmem, pred); }
__device__ __forceinline__ void cp_async_t(float* smem, const float* gmem, bool pred) {
  const unsigned saddr = (unsigned) __cvta_generic_to_shared(smem);
  const int sz = pred ? 4 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(saddr), "l"(gmem), "r"(sz));
}

// FP64 fronts: one DMMA per fragment pair
// FP32 fronts: three TF32 products per fragment pair (hi*hi + hi*lo + lo*hi,
// the operands split as x = tf32(x) + tf32(x - tf32(x))), which keeps close
// to FP32 accuracy on the TF32 tensor path (same m16n8k8 fragment layout as
// the FP64 DMMA)
__device__ __forceinline__ void split_tf32(float x, unsigned& hi, unsigned& lo) {
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
  const float r = x - __uint_as_float(hi);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

__device__ __forceinline__ void mma_tf32(float (&c)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// MI x NI fragment products of one k8 step.  FP32: every A and B fragment is
// split into TF32 hi/lo parts once, then three products per pair.
template <int MI, int NI>
__device__ __forceinline__ void mma_block(double (&acc)[MI][NI][4], const double (&a)[MI][4], const double (&b)[NI][2]) {
#pragma unroll
  for (int mi = 0; mi < MI; mi++)
#pragma unroll
    for (int ni = 0; ni < NI; ni++) dmma16888(acc[mi][ni], a[mi], b[ni]);
}

template <int MI, int NI>
__device__ __forceinline__ void mma_block(float (&acc)[MI][NI][4], const float (&a)[MI][4], const float (&b)[NI][2]) {
  unsigned ah[MI][4], al[MI][4], bh[NI][2], bl[NI][2];
#pragma unroll
  for (int mi = 0; mi < MI; mi++)
#pragma unroll
    for (int i = 0; i < 4; i++) split_tf32(a[mi][i], ah[mi][i], al[mi][i]);
#pragma unroll
  for (int ni = 0; ni < NI; ni++)
#pragma unroll
    for (int i = 0; i < 2; i++) split_tf32(b[ni][i], bh[ni][i], bl[ni][i]);
#pragma unroll
  for (int mi = 0; mi < MI; mi++)
#pragma unroll
    for (int ni = 0; ni < NI; ni++) {
      mma_tf32(acc[mi][ni], al[mi], bh[ni]);
      mma_tf32(acc[mi][ni], ah[mi], bl[ni]);
      mma_tf32(acc[mi][ni], ah[mi], bh[ni]);
    }
}

constexpr int GEMM_STAGES = 3;

// number of lower-trapezoid tiles of a region with `rows` rows and `cols`
// columns whose column tile c covers rows [c*BN, rows)
__host__ __device__ inline int trap_tiles(int rows, int cols, int bm, int bn) {
  int t = 0;
  for (int c0 = 0; c0 < cols; c0 += bn) t += (rows - c0 + bm - 1) / bm;
  return t;
}

template <int BM, int BN>
struct GemmCfg {
  static constexpr int WM = 2;                     // warps along M
  static constexpr int WN = BN / 32;               // warps along N (32 columns each)
  static constexpr int THREADS = 32 * WM * WN;
  static constexpr int MI = BM / WM / 16;          // m16 tiles per warp
  static constexpr int NI = 4;                     // n8 tiles per warp
  static constexpr int LD = BM + 8;                // padded k-row stride (BM >= BN)
  template <typename T>
  static constexpr size_t smem() { return (size_t) GEMM_STAGES * 2 * GEMM_BK * LD * sizeof(T); }
};

// C -= A B^T on DMMA m16n8k8 tiles of BM x BN (64x64: 4 warps, 128x128: 8
// warps), GEMM_STAGES-deep cp.async pipeline, accumulators preloaded with -C.
// mode 0: panel update of columns [c_lo, min(c_hi, s)) and all rows below
//         c_lo by the panel columns [k_lo, k_hi) (one node of the recursive
//         panel factorization);
// mode 1: U -= L21 L21^T (K = [0, s))
template <typename T, int BM, int BN>
__global__ void __launch_bounds__(GemmCfg<BM, BN>::THREADS)
k_gemm(const int* __restrict__ list, const FrontDesc* __restrict__ fronts, T* __restrict__ L,
       T* __restrict__ U, int c_lo, int c_hi, int k_lo, int k_hi, int mode, const int* status) {
  using Cfg = GemmCfg<BM, BN>;
  constexpr int MI = Cfg::MI, NI = Cfg::NI, LD = Cfg::LD, NT = Cfg::THREADS;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* gsm = reinterpret_cast<T*>(smraw);   // GEMM_STAGES x {A, B} x GEMM_BK x LD
  if (failed(status)) return;
  const FrontDesc F = fronts[list[blockIdx.y]];
  const int f = F.f, s = F.s, m = f - s;
  int rows, cols, roff, kbeg, kend, ldc;
  const T* P = L + F.l_off;
  T* Cbase;
  if (mode == 0) {
    const int cb = c_lo, ce = min(c_hi, s);
    if (cb >= ce) return;
    rows = f - cb; cols = ce - cb; roff = cb;
    kbeg = k_lo; kend = k_hi;
    Cbase = L + F.l_off + cb + (size_t) cb * f;
    ldc = f;
  } else {
    if (m <= 0 || s <= 0) return;
    rows = m; cols = m; roff = s;
    kbeg = 0; kend = s;
    Cbase = U + F.u_off;
    ldc = m;
  }
  // decode the lower-trapezoid tile
  int idx = blockIdx.x, c0 = 0;
  for (;;) {
    if (c0 >= cols) return;
    const int nt_c = (rows - c0 + BM - 1) / BM;
    if (idx < nt_c) break;
    idx -= nt_c;
    c0 += BN;
  }
  const int r0 = c0 + idx * BM;
  const int nr = min(BM, rows - r0), nc = min(BN, cols - c0);
  const T* Ag = P + (roff + r0);
  const T* Bg = P + (roff + c0);
  T* C = Cbase + r0 + (size_t) c0 * ldc;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % Cfg::WM, wn = warp / Cfg::WM, g = lane >> 2, t = lane & 3;
  const int wrow = wm * (BM / Cfg::WM), wcol = wn * 32;
  // accumulators start at -C, so acc = A B^T - C and the result is -acc
  T acc[MI][NI][4];
#pragma unroll
  for (int mi = 0; mi < MI; mi++)
#pragma unroll
    for (int ni = 0; ni < NI; ni++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int r = wrow + mi * 16 + g + ((q & 2) ? 8 : 0);
        const int c = wcol + ni * 8 + 2 * t + (q & 1);
        acc[mi][ni][q] = (r < nr && c < nc && r0 + r >= c0 + c) ? -C[r + (size_t) c * ldc] : 0.0;
      }

  auto load = [&](int st, int k0) {
    T* As = gsm + (size_t) (st * 2) * GEMM_BK * LD;
    T* Bs = As + GEMM_BK * LD;
#pragma unroll
    for (int q = 0; q < (BM * GEMM_BK) / NT; q++) {
      const int e = tid + q * NT;
      const int r = e % BM, k = e / BM;
      const bool kv = (k0 + k) < kend;
      const bool pa = kv && r < nr;
      const size_t col = (size_t) (kv ? k0 + k : kbeg) * f;
      cp_async_t(As + k * LD + r, Ag + (pa ? r : 0) + col, pa);
    }
#pragma unroll
    for (int q = 0; q < (BN * GEMM_BK) / NT; q++) {
      const int e = tid + q * NT;
      const int r = e % BN, k = e / BN;
      const bool kv = (k0 + k) < kend;
      const bool pb = kv && r < nc;
      const size_t col = (size_t) (kv ? k0 + k : kbeg) * f;
      cp_async_t(Bs + k * LD + r, Bg + (pb ? r : 0) + col, pb);
    }
  };

  const int nk = (kend - kbeg + GEMM_BK - 1) / GEMM_BK;
#pragma unroll
  for (int st = 0; st < GEMM_STAGES - 1; st++) {
    if (st < nk) load(st, kbeg + st * GEMM_BK);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; kt++) {
    cp_async_wait<GEMM_STAGES - 2>();
    __syncthreads();
    const int kn = kt + GEMM_STAGES - 1;
    if (kn < nk) load(kn % GEMM_STAGES, kbeg + kn * GEMM_BK);
    cp_async_commit();
    const T* As = gsm + (size_t) ((kt % GEMM_STAGES) * 2) * GEMM_BK * LD;
    const T* Bs = As + GEMM_BK * LD;
#pragma unroll
    for (int kk = 0; kk < GEMM_BK; kk += 8) {
      T a[MI][4], b[NI][2];
#pragma unroll
      for (int mi = 0; mi < MI; mi++) {
        const int r = wrow + mi * 16 + g;
        a[mi][0] = As[(kk + t) * LD + r];
        a[mi][1] = As[(kk + t) * LD + r + 8];
        a[mi][2] = As[(kk + t + 4) * LD + r];
        a[mi][3] = As[(kk + t + 4) * LD + r + 8];
      }
#pragma unroll
      for (int ni = 0; ni < NI; ni++) {
        const int c = wcol + ni * 8 + g;
        b[ni][0] = Bs[(kk + t) * LD + c];
        b[ni][1] = Bs[(kk + t + 4) * LD + c];
      }
      mma_block<MI, NI>(acc, a, b);
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int mi = 0; mi < MI; mi++)
#pragma unroll
    for (int ni = 0; ni < NI; ni++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int r = wrow + mi * 16 + g + ((q & 2) ? 8 : 0);
        const int c = wcol + ni * 8 + 2 * t + (q & 1);
        if (r < nr && c < nc && r0 + r >= c0 + c) C[r + (size_t) c * ldc] = -acc[mi][ni][q];
      }
}

}  // namespace

// algorithmic work of a whole front (the reference's flop count,
// src/taucs_sn_llt.c:3957-3965) and of its assembly / extend-add traffic
static double front_flops(const FrontDesc& F) {
  double fl = 0.0;
  for (int k = 0, c = F.f; k < F.s; k++, c--) fl += 1.0 + (double) c * (double) c;
  return fl;
}

// algorithmic bytes of building one front, values of esz bytes: children's U
// read once (plus their maps), panel and U written once, A entries (value +
// row index)
static double build_bytes(const Plan& P, const FrontDesc& F, double esz) {
  double by = 0.0;
  for (int ci = F.child_begin; ci < F.child_end; ci++) {
    const FrontDesc& C = P.fronts[P.children[ci]];
    const double mc = C.f - C.s;
    by += esz * mc * (mc + 1.0) / 2.0 + 4.0 * mc;
  }
  const double m = F.f - F.s;
  by += esz * ((double) F.f * F.s - (double) F.s * (F.s - 1) / 2.0) + esz * m * (m + 1.0) / 2.0;
  by += (esz + 4.0) * (P.acol_ptr[F.acol_off + F.s] - P.acol_ptr[F.acol_off]);
  return by;
}

// small fronts: read children's U and A once, write panel and U once
static double front_bytes(const Plan& P, const FrontDesc& F, double esz) {
  return build_bytes(P, F, esz);
}

// GEMM variant of level h for the panel updates (kind 0) or the update
// matrix (kind 1): FP64 fronts choose between 64x64 tiles (4 warps, 3 CTAs
// per SM; the default, 24 TF/s on the 64^3 update matrices) and 128x128
// tiles (8 warps, one CTA per SM; 19 TF/s there), FP32 fronts between the
// two tcgen05 variants.  The choice comes from the autotuner's measurements
// (Plan::gemm_choice), the default variant otherwise.
template <typename T>
static bool gemm_alt(const Plan& P, int h, int kind) {
  const std::vector<uint8_t>& c = P.gemm_choice[sizeof(T) == 4 ? 1 : 0];
  return (size_t) (2 * h + kind) < c.size() && c[2 * h + kind] != 0;
}

template <typename T>
static void launch_gemm(bool big, int gx128, int gx64, int nb, const int* blst, const DevPlan& D, T* L, T* U,
                        int c_lo, int c_hi, int k_lo, int k_hi, int mode, int* status, cudaStream_t st,
                        const float* = nullptr, int = 0, int = 0) {
  if (big)
    k_gemm<T, 128, 128><<<dim3(gx128, nb), GemmCfg<128, 128>::THREADS, GemmCfg<128, 128>::smem<T>(), st>>>(
        blst, D.fronts, L, U, c_lo, c_hi, k_lo, k_hi, mode, status);
  else
    k_gemm<T, 64, 64><<<dim3(gx64, nb), GemmCfg<64, 64>::THREADS, GemmCfg<64, 64>::smem<T>(), st>>>(
        blst, D.fronts, L, U, c_lo, c_hi, k_lo, k_hi, mode, status);
}

// FP32 fronts take the tcgen05 kernels (gemm_tc.cu): by default the one fed
// from the split arena (gx_sp tiles per front), with `alt` the one whose
// producer warps split the operands as they load them
static void launch_gemm(bool alt, int gx128, int gx64, int nb, const int* blst, const DevPlan& D, float* L, float* U,
                        int c_lo, int c_hi, int k_lo, int k_hi, int mode, int* status, cudaStream_t st,
                        const float* sp = nullptr, int gx_sp = 0, int sp_fmt = 0) {
  if (!alt && sp && gemm_sp_init()) {
    launch_gemm_sp(sp_fmt, gx_sp, nb, blst, D.fronts, sp, L, U, c_lo, c_hi, k_lo, k_hi, mode, status, st);
    return;
  }
  if (gemm_tc_init()) {
    launch_gemm_tc(0, gx128, nb, blst, D.fronts, L, U, c_lo, c_hi, k_lo, k_hi, mode, status, st);
    return;
  }
  launch_gemm<float>(false, gx128, gx64, nb, blst, D, L, U, c_lo, c_hi, k_lo, k_hi, mode, status, st);
}

// CTAs of the persistent small-front launch: all that fit on the device at
// once with `smem` bytes each (the shared memory of the largest front in the
// persistent set: a set of small fronts fits many more CTAs per SM)
template <typename T>
static int pers_grid(size_t smem) {
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
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_small_persistent<T>, 128, smem) != cudaSuccess) b = 1;
  return std::max(1, std::max(b, 1) * sms[d]);
}

// CTAs (four warps) of the one-warp-per-front persistent launch: all that
// fit on the device at once
template <typename T>
static int warp_grid() {
  static PerDeviceOnce pd;
  static int grid[MAX_DEVICES];
  per_device_once(pd, [] {
    int d = 0, sms = 0, b = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_small_warp<T>, 128, 0) != cudaSuccess) b = 1;
    grid[d] = std::max(1, std::max(b, 1) * sms);
    return true;
  });
  int d = 0;
  cudaGetDevice(&d);
  return grid[d];
}

template <typename T>
static void set_smem_attrs() {
  // once per device and type (request-server workers reach this concurrently)
  static PerDeviceOnce pd;
  per_device_once(pd, [] {
    cudaFuncSetAttribute(k_small_front<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         SMALL_F_MAX * SMALL_F_MAX * (int) sizeof(T));
    cudaFuncSetAttribute(k_small_persistent<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         SMALL_F_MAX * SMALL_F_MAX * (int) sizeof(T));
    cudaFuncSetAttribute(k_dinv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) dinv_smem<T>());
    cudaFuncSetAttribute(k_gemm<T, 64, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int) GemmCfg<64, 64>::smem<T>());
    cudaFuncSetAttribute(k_gemm<T, 128, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int) GemmCfg<128, 128>::smem<T>());
    return true;
  });
}

template <typename T>
static int launch_numeric(const Plan& P, const DevPlan& D, const T* vals, T* L, T* U, T* Dinv, float* sp,
                          int sp_fmt, int* status, cudaStream_t st) {
  set_smem_attrs<T>();
  k_init_status<<<1, 1, 0, st>>>(status);
  count_launch();
  if (D.n_pers > 0) {
    // every small front with only small fronts below it, in two launches:
    // one warp per front for the subtrees of fronts of order <= SMALL_WARP_F
    // (tasks 0 .. nw-1), then one CTA per front for the rest (their children
    // in the first part counted themselves off in the first launch)
    const int nw = P.pers_nwarp, np = D.n_pers;
    cudaMemcpyAsync(D.pers_work, D.pers_pending0, sizeof(int) * np, cudaMemcpyDeviceToDevice, st);
    cudaMemsetAsync(D.pers_work + np, 0, 2 * sizeof(int), st);
    auto prof_range = [&](int t0, int t1, double& fl, double& by) {
      fl = by = 0.0;
      if (prof_enabled())
        for (int t = t0; t < t1; t++) {
          fl += front_flops(P.fronts[P.pers_fronts[t]]);
          by += front_bytes(P, P.fronts[P.pers_fronts[t]], sizeof(T));
        }
    };
    double fl, by;
    if (nw > 0) {
      const int grid = std::min((nw + 3) / 4, warp_grid<T>());
      prof_range(0, nw, fl, by);
      prof_begin(KC_SMALL, st);
      k_small_warp<T><<<grid, 128, 0, st>>>(D.pers_list, 0, nw, D.pers_parent, D.pers_work, D.pers_work + np,
                                            D.fronts, D.children, D.maps, D.rows, D.acol_ptr, D.a_rows, D.a_idx,
                                            vals, L, U, status);
      prof_end(KC_SMALL, st, fl, by);
      count_launch();
    }
    if (np > nw) {
      const size_t smem = (size_t) P.pers_fmax * P.pers_fmax * sizeof(T);
      const int grid = std::min(np - nw, pers_grid<T>(smem));
      prof_range(nw, np, fl, by);
      prof_begin(KC_SMALL, st);
      k_small_persistent<T><<<grid, 128, smem, st>>>(D.pers_list, nw, np, D.pers_parent, D.pers_work,
                                                     D.pers_work + np + 1, D.fronts, D.children, D.maps, D.rows,
                                                     D.acol_ptr, D.a_rows, D.a_idx, vals, L, U, status);
      prof_end(KC_SMALL, st, fl, by);
      count_launch();
    }
  }
  for (int h = 0; h < P.n_levels; h++) {
    const LevelPlan& LP = P.levels[h];
    prof_tag(h);
    // small fronts above a big one (the rest went through the persistent
    // launch), in size classes so that the shared-memory request fits the class
    const int ns = (int) LP.small_numeric.size();
    if (ns > 0) {
      const int* lst = D.small_num + D.small_num_off[h];
      int b = 0;
      const int classes[3] = {32, 64, SMALL_F_MAX};
      for (int cl = 0; cl < 3 && b < ns; cl++) {
        int e = b;
        while (e < ns && P.fronts[LP.small_numeric[e]].f <= classes[cl]) e++;
        if (e > b) {
          const size_t smem = (size_t) classes[cl] * classes[cl] * sizeof(T);
          double fl = 0.0, by = 0.0;
          if (prof_enabled())
            for (int q = b; q < e; q++) {
              const FrontDesc& F = P.fronts[LP.small_numeric[q]];
              fl += front_flops(F);
              by += front_bytes(P, F, sizeof(T));
            }
          prof_begin(KC_SMALL, st);
          k_small_front<T><<<e - b, 128, smem, st>>>(lst + b, D.fronts, D.children, D.maps, D.rows,
                                                   D.acol_ptr, D.a_rows, D.a_idx, vals, L, U, status);
          prof_end(KC_SMALL, st, fl, by);
          count_launch();
        }
        b = e;
      }
    }
    const int nb = (int) LP.big_fronts.size();
    if (nb == 0) continue;
    const int* blst = D.big_list + D.big_off[h];
    const int ntiles = (int) LP.build_tiles.size();
    {
      double by = 0.0;
      if (prof_enabled())
        for (int fi : LP.big_fronts) by += build_bytes(P, P.fronts[fi], sizeof(T));
      prof_begin(KC_BUILD, st);
      k_build<T><<<ntiles, BUILD_THREADS, 0, st>>>(D.tiles + D.tile_off[h], D.tile_ch, D.fronts, D.maps, D.acol_ptr,
                                      D.a_rows, D.a_idx, vals, L, U, status);
      prof_end(KC_BUILD, st, 0.0, by);
      count_launch();
    }
    // recursive panel factorization over aligned column intervals: factor
    // the left half, update the right half with one GEMM (K = half width),
    // factor the right half; leaves are 64-column steps (k_leaf: POTRF of
    // the diagonal block and TRSM of the rows below in one launch)
    const int S = LP.max_s_big;
    int span = PANEL_NB;
    while (span < S) span *= 2;
    auto leaf = [&](int kb) {
      int gx = 1;
      double fl = 0.0, by = 0.0;
      for (int fi : LP.big_fronts) {
        const FrontDesc& F = P.fronts[fi];
        if (kb >= F.s) continue;
        const int w = std::min(PANEL_NB, F.s - kb);
        gx = std::max(gx, (F.f - kb - w + PANEL_NB - 1) / PANEL_NB);
        if (prof_enabled()) {
          const double ww = w, below = F.f - kb - w;
          fl += ww * ww * ww / 3.0 + below * ww * ww;
          by += 2.0 * sizeof(T) * (ww * (ww + 1.0) / 2.0 + below * ww);
        }
      }
      prof_begin(KC_LEAF, st);
      if (sp_fmt)
        k_leaf<T, 1><<<dim3(gx, nb), 128, 0, st>>>(blst, D.fronts, D.rows, L, Dinv, sp, kb, status);
      else
        k_leaf<T, 0><<<dim3(gx, nb), 128, 0, st>>>(blst, D.fronts, D.rows, L, Dinv, sp, kb, status);
      prof_end(KC_LEAF, st, fl, by);
      count_launch();
    };
    auto update = [&](int c_lo, int c_hi, int k_lo, int k_hi) {
      int gx = 0, gx64 = 0, maxc = 0, maxr = 0;
      double fg = 0.0, bg = 0.0;
      for (int fi : LP.big_fronts) {
        const FrontDesc& F = P.fronts[fi];
        const int ce = std::min(c_hi, F.s);
        if (c_lo >= ce) continue;
        gx = std::max(gx, trap_tiles(F.f - c_lo, ce - c_lo, 128, 128));
        gx64 = std::max(gx64, trap_tiles(F.f - c_lo, ce - c_lo, 64, 64));
        maxc = std::max(maxc, ce - c_lo);
        maxr = std::max(maxr, F.f - c_lo);
        if (prof_enabled()) {
          const double c = ce - c_lo, below = F.f - ce, k = k_hi - k_lo;
          const double entries = c * (c + 1.0) / 2.0 + below * c;
          fg += 2.0 * k * entries;
          bg += 2.0 * sizeof(T) * entries + sizeof(T) * k * (F.f - c_lo);
        }
      }
      if (gx64 == 0) return;
      prof_begin(KC_GEMM_PANEL, st);
      (void) maxr; (void) maxc;
      launch_gemm(gemm_alt<T>(P, h, 0), gx, gx64, nb, blst, D, L, U, c_lo, c_hi, k_lo, k_hi, 0, status, st, sp, gx, sp_fmt);
      prof_end(KC_GEMM_PANEL, st, fg, bg);
      count_launch();
    };
    struct Rec {
      static void run(int a, int b, int S_, const decltype(leaf)& lf, const decltype(update)& up) {
        if (a >= S_) return;
        if (b - a <= PANEL_NB) { lf(a); return; }
        const int mid = (a + b) / 2;
        run(a, mid, S_, lf, up);
        if (mid < S_) up(mid, b, a, mid);
        run(mid, b, S_, lf, up);
      }
    };
    Rec::run(0, span, S, leaf, update);
    int gx_u = 0, gx_u64 = 0, gx_usp = 0, maxm = 0;
    for (int fi : LP.big_fronts) {
      const FrontDesc& F = P.fronts[fi];
      const int m = F.f - F.s;
      if (m > 0) {
        gx_u = std::max(gx_u, trap_tiles(m, m, 128, 128));
        gx_usp = std::max(gx_usp, gemm_sp_tiles_u(F.s, F.f));
        gx_u64 = std::max(gx_u64, trap_tiles(m, m, 64, 64));
        maxm = std::max(maxm, m);
      }
    }
    if (gx_u64 > 0) {
      double fu = 0.0, bu = 0.0;
      if (prof_enabled())
        for (int fi : LP.big_fronts) {
          const FrontDesc& F = P.fronts[fi];
          const double m = F.f - F.s;
          fu += 2.0 * F.s * m * (m + 1.0) / 2.0;
          bu += 2.0 * sizeof(T) * m * (m + 1.0) / 2.0 + sizeof(T) * m * F.s;
        }
      prof_begin(KC_GEMM_U, st);
      (void) maxm;
      launch_gemm(gemm_alt<T>(P, h, 1), gx_u, gx_u64, nb, blst, D, L, U, 0, 0, 0, 0, 1, status, st, sp, gx_usp, sp_fmt);
      prof_end(KC_GEMM_U, st, fu, bu);
      count_launch();
    }
  }
  prof_tag(-1);
  if (D.n_dblk > 0) {
    prof_begin(KC_DINV, st);
    k_dinv<T><<<D.n_dblk, 128, dinv_smem<T>(), st>>>(D.dblk, D.fronts, L, Dinv, status);
    prof_end(KC_DINV, st, (double) D.n_dblk * PANEL_NB * PANEL_NB * PANEL_NB / 3.0,
             2.0 * sizeof(T) * D.n_dblk * PANEL_NB * PANEL_NB);
    count_launch();
  }
  return (int) cudaGetLastError();
}

int launch_tile_ranges(const DevPlan& D, int ntiles, cudaStream_t st) {
  k_tile_ranges<<<ntiles, 128, 0, st>>>(D.tiles, D.fronts, D.children, D.maps, D.tile_ch);
  return (int) cudaGetLastError();
}

int launch_numeric_fp64(const Plan& P, const DevPlan& D, const double* vals, double* L, double* U, double* Dinv,
                        int* status, cudaStream_t st) {
  return launch_numeric<double>(P, D, vals, L, U, Dinv, nullptr, 0, status, st);
}

int launch_numeric_fp32(const Plan& P, const DevPlan& D, const float* vals, float* L, float* U, float* Dinv,
                        float* sp, int sp_fmt, int* status, cudaStream_t st) {
  return launch_numeric<float>(P, D, vals, L, U, Dinv, sp, sp_fmt, status, st);
}

}  // namespace tb

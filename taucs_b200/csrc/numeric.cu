// FP64 multifrontal numeric factorization on sm_100a.
//
// The reference factors one front at a time in a depth-first recursion
// (src/taucs_sn_llt.c:1829-1977): calloc F1/F2/U, extend-add each child
// (:1200-1240), assemble A's columns (:1099-1119), then LAPACK/BLAS POTRF
// (:1131), TRSM (:1150) and SYRK (:1180).  Here every front of one level of
// the supernodal tree is processed by the same launches:
//
//   k_small_front   fronts of order <= SMALL_F_MAX: one CTA builds the whole
//                   front in shared memory (zero + assemble + extend-add),
//                   factors it (right-looking partial Cholesky of the first s
//                   columns, i.e. POTRF+TRSM+SYRK fused) and writes the panel
//                   and the update matrix once;
//   k_build         larger fronts: one CTA per 64x32 tile of the front's lower
//                   part gathers A's entries and the children's update
//                   matrices into shared memory in a fixed child order
//                   (deterministic, no atomics) and writes the tile once;
//   k_potrf_diag    blocked partial Cholesky, step kb: one CTA per front
//                   factors the 64x64 diagonal block in place and forms its
//                   inverse;
//   k_trsm          then one CTA per 64-row slab below it computes
//                   X L_kk^-T = X Dinv^T on DMMA;
//   k_gemm          C -= A B^T on DMMA (mma.sync m16n8k8 f64) tiles: the
//                   trailing update of the panel after each step, and the
//                   update matrix U -= L21 L21^T with k = s at the end.
//
// Every kernel first reads the status word and returns when an earlier front
// hit a nonpositive pivot; the smallest failing global column is recorded
// with atomicMin (the reference reports the failing column, :1139-1145).
#include <climits>
#include <cstdio>

#include "kernels.h"

namespace tb {

namespace {

__device__ __forceinline__ int lower_bound_dev(const int* a, int n, int key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool failed(const int* status) {
  return *(volatile const int*) status != INT_MAX;
}

__global__ void k_init_status(int* status) { *status = INT_MAX; }

// ------------------------------------------------------------ small fronts

__global__ void __launch_bounds__(128)
k_small_front(const int* __restrict__ list, const FrontDesc* __restrict__ fronts,
              const int* __restrict__ children, const int* __restrict__ maps,
              const int* __restrict__ rows, const int* __restrict__ acol_ptr,
              const int* __restrict__ a_rows, const int* __restrict__ a_idx,
              const double* __restrict__ vals, double* __restrict__ L, double* __restrict__ U,
              int* status) {
  extern __shared__ double W[];
  if (failed(status)) return;
  const FrontDesc F = fronts[list[blockIdx.x]];
  const int f = F.f, s = F.s, m = f - s;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;

  for (int k = tid; k < f * f; k += nt) W[k] = 0.0;
  __syncthreads();
  for (int c = tid; c < s; c += nt) {
    const int e1 = acol_ptr[F.acol_off + c + 1];
    for (int e = acol_ptr[F.acol_off + c]; e < e1; e++) W[a_rows[e] + c * f] += vals[a_idx[e]];
  }
  __syncthreads();
  for (int ci = F.child_begin; ci < F.child_end; ci++) {
    const FrontDesc C = fronts[children[ci]];
    const int mc = C.f - C.s;
    const int* mp = maps + C.map_off;
    const double* Uc = U + C.u_off;
    for (int j = warp; j < mc; j += nw) {
      const int pj = mp[j] * f;
      for (int i = j + lane; i < mc; i += 32) W[mp[i] + pj] += Uc[i + (size_t) j * mc];
    }
    __syncthreads();
  }
  for (int j = 0; j < s; j++) {
    const double d = W[j + j * f];
    if (!(d > 0.0)) {
      if (tid == 0) atomicMin(status, rows[F.rows_off + j]);
      return;
    }
    __syncthreads();
    const double ljj = sqrt(d);
    for (int i = j + 1 + tid; i < f; i += nt) W[i + j * f] /= ljj;
    if (tid == 0) W[j + j * f] = ljj;
    __syncthreads();
    for (int k = j + 1 + warp; k < f; k += nw) {
      const double lkj = W[k + j * f];
      double* wk = W + k * f;
      const double* wj = W + j * f;
      for (int i = k + lane; i < f; i += 32) wk[i] -= wj[i] * lkj;
    }
    __syncthreads();
  }
  double* Lp = L + F.l_off;
  for (int k = tid; k < f * s; k += nt) Lp[k] = W[k];
  if (m > 0) {
    double* Up = U + F.u_off;
    for (int k = tid; k < m * m; k += nt) {
      const int i = k % m, c = k / m;
      Up[k] = W[(s + i) + (s + c) * f];
    }
  }
}

// --------------------------------------------------------------- front build

__global__ void __launch_bounds__(256)
k_build(const Tile* __restrict__ tiles, const FrontDesc* __restrict__ fronts,
        const int* __restrict__ children, const int* __restrict__ maps,
        const int* __restrict__ acol_ptr, const int* __restrict__ a_rows,
        const int* __restrict__ a_idx, const double* __restrict__ vals,
        double* __restrict__ L, double* __restrict__ U, const int* status) {
  __shared__ double W[BUILD_TR * BUILD_TC];
  if (failed(status)) return;
  const Tile T = tiles[blockIdx.x];
  const FrontDesc F = fronts[T.front];
  const int f = F.f, s = F.s, m = f - s;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const bool panel = T.c0 >= 0;
  int R0, C0, nr, nc;
  if (panel) {
    R0 = T.r0; C0 = T.c0;
    nr = min(BUILD_TR, f - R0); nc = min(BUILD_TC, s - C0);
  } else {
    const int uc0 = -1 - T.c0;
    R0 = s + T.r0; C0 = s + uc0;
    nr = min(BUILD_TR, m - T.r0); nc = min(BUILD_TC, m - uc0);
  }
  for (int k = tid; k < BUILD_TR * BUILD_TC; k += nt) W[k] = 0.0;
  __syncthreads();
  if (panel) {
    for (int c = tid; c < nc; c += nt) {
      const int e1 = acol_ptr[F.acol_off + C0 + c + 1];
      for (int e = acol_ptr[F.acol_off + C0 + c]; e < e1; e++) {
        const int r = a_rows[e] - R0;
        if (r >= 0 && r < nr) W[r + c * BUILD_TR] += vals[a_idx[e]];
      }
    }
    __syncthreads();
  }
  for (int ci = F.child_begin; ci < F.child_end; ci++) {
    const FrontDesc C = fronts[children[ci]];
    const int mc = C.f - C.s;
    const int* mp = maps + C.map_off;
    const int ja = lower_bound_dev(mp, mc, C0), jb = lower_bound_dev(mp, mc, C0 + nc);
    if (ja >= jb) continue;
    const int ia = lower_bound_dev(mp, mc, R0), ib = lower_bound_dev(mp, mc, R0 + nr);
    if (ia >= ib) continue;
    const double* Uc = U + C.u_off;
    for (int j = ja + warp; j < jb; j += nw) {
      const int pj = (mp[j] - C0) * BUILD_TR;
      const double* uj = Uc + (size_t) j * mc;
      for (int i = max(ia, j) + lane; i < ib; i += 32) W[(mp[i] - R0) + pj] += uj[i];
    }
    __syncthreads();
  }
  if (panel) {
    double* dst = L + F.l_off;
    for (int k = tid; k < BUILD_TR * BUILD_TC; k += nt) {
      const int r = k % BUILD_TR, c = k / BUILD_TR;
      if (r < nr && c < nc) dst[(R0 + r) + (size_t) (C0 + c) * f] = W[k];
    }
  } else {
    double* dst = U + F.u_off;
    for (int k = tid; k < BUILD_TR * BUILD_TC; k += nt) {
      const int r = k % BUILD_TR, c = k / BUILD_TR;
      if (r < nr && c < nc) dst[(R0 - s + r) + (size_t) (C0 - s + c) * m] = W[k];
    }
  }
}

// ------------------------------------------------------- blocked POTRF+TRSM

constexpr int DLD = PANEL_NB + 1;  // padded column stride of the diagonal block
constexpr size_t POTRF_SMEM = (2 * PANEL_NB * DLD + 32 * 33) * sizeof(double);

// Lower Cholesky of an n x n (n <= 32) block held in shared memory (ld `ld`),
// by one warp: lane i keeps row i in registers and the right-looking updates
// exchange L[k][j] with shuffles.  Returns the first nonpositive pivot (or -1)
// in every lane.
__device__ int warp_potrf32(double* S, int ld, int n) {
  const int lane = threadIdx.x & 31;
  double a[32];
#pragma unroll
  for (int k = 0; k < 32; k++) a[k] = (lane < n && k <= lane) ? S[lane + k * ld] : 0.0;
  int bad = -1;
#pragma unroll
  for (int j = 0; j < 32; j++) {
    if (j < n) {
      const double d = __shfl_sync(0xffffffffu, a[j], j);
      if (!(d > 0.0) && bad < 0) bad = j;
      const double ljj = sqrt(d);
      if (lane == j) a[j] = ljj;
      else if (lane > j) a[j] /= ljj;
#pragma unroll
      for (int k = j + 1; k < 32; k++) {
        const double lkj = __shfl_sync(0xffffffffu, a[j], k);
        if (lane >= k) a[k] -= a[j] * lkj;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 32; k++)
    if (lane < n && k <= lane) S[lane + k * ld] = a[k];
  return bad;
}

// Inverse of an n x n (n <= 32) lower-triangular block by one warp: lane t
// computes column t by forward substitution (L read as broadcasts).
__device__ void warp_trinv32(const double* S, int ld, double* X, int ldx, int n) {
  const int t = threadIdx.x & 31;
  double x[32];
#pragma unroll
  for (int i = 0; i < 32; i++) {
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < i; k++) acc += S[i + k * ld] * x[k];
    x[i] = (i < n) ? (((i == t) ? 1.0 : 0.0) - acc) / S[i + i * ld] : 0.0;
  }
#pragma unroll
  for (int i = 0; i < 32; i++) X[i + t * ldx] = (t < n) ? x[i] : 0.0;
}

// Step kb, one CTA per front: factor the w x w diagonal block in place as a
// 2 x 2 recursion over 32-blocks (warp-level POTRF of the diagonal blocks,
// inverse-based TRSM and the SYRK update in between) and store the inverse of
// the factored block (lower, ld PANEL_NB) for the TRSM of the rows below.
__global__ void __launch_bounds__(128)
k_potrf_diag(const int* __restrict__ list, const FrontDesc* __restrict__ fronts,
             const int* __restrict__ rows, double* __restrict__ L, double* __restrict__ Dinv, int kb,
             int* status) {
  extern __shared__ double sm[];
  double* D = sm;                        // the block, col-major, ld DLD
  double* X = sm + PANEL_NB * DLD;       // its inverse
  double* T = X + PANEL_NB * DLD;        // 32 x 33 scratch
  __shared__ int bad;
  if (failed(status)) return;
  const FrontDesc F = fronts[list[blockIdx.x]];
  const int f = F.f, s = F.s;
  if (kb >= s) return;
  const int w = min(PANEL_NB, s - kb);
  const int w1 = min(32, w), w2 = w - w1;
  const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5;
  double* P = L + F.l_off;
  for (int k = tid; k < PANEL_NB * PANEL_NB; k += nt) {
    const int i = k % PANEL_NB, j = k / PANEL_NB;
    D[i + j * DLD] = (i < w && j < w && i >= j) ? P[(kb + i) + (size_t) (kb + j) * f] : 0.0;
    X[i + j * DLD] = 0.0;
  }
  if (tid == 0) bad = -1;
  __syncthreads();
  if (warp == 0) {
    const int b = warp_potrf32(D, DLD, w1);
    if (b < 0) warp_trinv32(D, DLD, X, DLD, w1);
    if ((tid & 31) == 0) bad = b;
  }
  __syncthreads();
  if (bad >= 0) {
    if (tid == 0) atomicMin(status, rows[F.rows_off + kb + bad]);
    return;
  }
  if (w2 > 0) {
    double* D21 = D + 32;
    double* D22 = D + 32 + 32 * DLD;
    const double* X11 = X;
    // L21 = D21 X11^T
    for (int e = tid; e < 32 * 32; e += nt) {
      const int i = e % 32, j = e / 32;
      double acc = 0.0;
      for (int k = 0; k <= j; k++) acc += D21[i + k * DLD] * X11[j + k * DLD];
      T[i + j * 33] = (i < w2) ? acc : 0.0;
    }
    __syncthreads();
    for (int e = tid; e < 32 * 32; e += nt) {
      const int i = e % 32, j = e / 32;
      D21[i + j * DLD] = T[i + j * 33];
    }
    __syncthreads();
    // D22 -= L21 L21^T (lower)
    for (int e = tid; e < 32 * 32; e += nt) {
      const int i = e % 32, j = e / 32;
      if (i >= j && i < w2) {
        double acc = 0.0;
        for (int k = 0; k < 32; k++) acc += D21[i + k * DLD] * D21[j + k * DLD];
        D22[i + j * DLD] -= acc;
      }
    }
    __syncthreads();
    if (warp == 0) {
      const int b = warp_potrf32(D22, DLD, w2);
      if (b < 0) warp_trinv32(D22, DLD, X + 32 + 32 * DLD, DLD, w2);
      if ((tid & 31) == 0) bad = b < 0 ? -1 : 32 + b;
    }
    __syncthreads();
    if (bad >= 0) {
      if (tid == 0) atomicMin(status, rows[F.rows_off + kb + bad]);
      return;
    }
    // X21 = -X22 (L21 X11)
    const double* X22 = X + 32 + 32 * DLD;
    for (int e = tid; e < 32 * 32; e += nt) {
      const int i = e % 32, j = e / 32;
      double acc = 0.0;
      for (int k = j; k < 32; k++) acc += D21[i + k * DLD] * X11[k + j * DLD];
      T[i + j * 33] = acc;
    }
    __syncthreads();
    for (int e = tid; e < 32 * 32; e += nt) {
      const int i = e % 32, j = e / 32;
      double acc = 0.0;
      for (int k = 0; k <= i; k++) acc += X22[i + k * DLD] * T[k + j * 33];
      X[32 + i + j * DLD] = -acc;
    }
    __syncthreads();
  }
  for (int k = tid; k < w * w; k += nt) {
    const int i = k % w, j = k / w;
    if (i >= j) P[(kb + i) + (size_t) (kb + j) * f] = D[i + j * DLD];
  }
  double* Di = Dinv + F.dinv_off + (size_t) (kb / PANEL_NB) * PANEL_NB * PANEL_NB;
  for (int k = tid; k < PANEL_NB * PANEL_NB; k += nt) {
    const int i = k % PANEL_NB, j = k / PANEL_NB;
    Di[k] = X[i + j * DLD];
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

constexpr int TLD = PANEL_NB + 8;  // padded k-row stride of the TRSM operands

// Step kb: rows below the diagonal block, X := X L_kk^-T = X * Dinv^T, one
// CTA per 64-row slab, DMMA m16n8k8; in place (the slab is staged first).
__global__ void __launch_bounds__(128)
k_trsm(const int* __restrict__ list, const FrontDesc* __restrict__ fronts,
       double* __restrict__ L, const double* __restrict__ Dinv, int kb, const int* status) {
  extern __shared__ double sm[];
  double* As = sm;                        // [k][r]: slab, k-major
  double* Bs = sm + PANEL_NB * TLD;       // [k][c]: Dinv[c][k]
  if (failed(status)) return;
  const FrontDesc F = fronts[list[blockIdx.y]];
  const int f = F.f, s = F.s;
  if (kb >= s) return;
  const int w = min(PANEL_NB, s - kb);
  const int r0 = kb + w + blockIdx.x * TRSM_ROWS;
  if (r0 >= f) return;
  const int nr = min(TRSM_ROWS, f - r0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double* P = L + F.l_off;
  const double* Di = Dinv + F.dinv_off + (size_t) (kb / PANEL_NB) * PANEL_NB * PANEL_NB;
  for (int e = tid; e < PANEL_NB * PANEL_NB; e += 128) {
    const int r = e % PANEL_NB, k = e / PANEL_NB;
    As[k * TLD + r] = (r < nr && k < w) ? P[(r0 + r) + (size_t) (kb + k) * f] : 0.0;
    Bs[k * TLD + r] = Di[r + k * PANEL_NB];
  }
  __syncthreads();
  const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t = lane & 3;
  double acc[2][4][4];
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[a][b][c] = 0.0;
  for (int kk = 0; kk < PANEL_NB; kk += 8) {
    double a[2][4], b[4][2];
#pragma unroll
    for (int mi = 0; mi < 2; mi++) {
      const int r = wm * 32 + mi * 16 + g;
      a[mi][0] = As[(kk + t) * TLD + r];
      a[mi][1] = As[(kk + t) * TLD + r + 8];
      a[mi][2] = As[(kk + t + 4) * TLD + r];
      a[mi][3] = As[(kk + t + 4) * TLD + r + 8];
    }
#pragma unroll
    for (int ni = 0; ni < 4; ni++) {
      const int c = wn * 32 + ni * 8 + g;
      b[ni][0] = Bs[(kk + t) * TLD + c];
      b[ni][1] = Bs[(kk + t + 4) * TLD + c];
    }
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
      for (int ni = 0; ni < 4; ni++) dmma16888(acc[mi][ni], a[mi], b[ni]);
  }
#pragma unroll
  for (int mi = 0; mi < 2; mi++)
#pragma unroll
    for (int ni = 0; ni < 4; ni++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int r = wm * 32 + mi * 16 + g + ((q & 2) ? 8 : 0);
        const int c = wn * 32 + ni * 8 + 2 * t + (q & 1);
        if (r < nr && c < w) P[(r0 + r) + (size_t) (kb + c) * f] = acc[mi][ni][q];
      }
}

constexpr int GLD = GEMM_BM + 8;  // padded k-row stride of the staged tiles

// number of lower-trapezoid tiles of a region with `rows` rows and `cols`
// columns whose column tile c covers rows [c*BN, rows)
__host__ __device__ inline int trap_tiles(int rows, int cols) {
  int t = 0;
  for (int c0 = 0; c0 < cols; c0 += GEMM_BN) t += (rows - c0 + GEMM_BM - 1) / GEMM_BM;
  return t;
}

// mode 0: trailing update of the panel after step kb (K = [kb, kb+w));
// mode 1: U -= L21 L21^T (K = [0, s))
__global__ void __launch_bounds__(128)
k_gemm(const int* __restrict__ list, const FrontDesc* __restrict__ fronts, double* __restrict__ L,
       double* __restrict__ U, int kb, int mode, const int* status) {
  __shared__ __align__(16) double As[2][GEMM_BK][GLD];
  __shared__ __align__(16) double Bs[2][GEMM_BK][GLD];
  if (failed(status)) return;
  const FrontDesc F = fronts[list[blockIdx.y]];
  const int f = F.f, s = F.s, m = f - s;
  int rows, cols, roff, kbeg, kend, ldc;
  const double* P = L + F.l_off;
  double* Cbase;
  if (mode == 0) {
    if (kb >= s) return;
    const int w = min(PANEL_NB, s - kb);
    const int cb = kb + w;
    if (cb >= s) return;
    rows = f - cb; cols = s - cb; roff = cb;
    kbeg = kb; kend = kb + w;
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
    const int nt_c = (rows - c0 + GEMM_BM - 1) / GEMM_BM;
    if (idx < nt_c) break;
    idx -= nt_c;
    c0 += GEMM_BN;
  }
  const int r0 = c0 + idx * GEMM_BM;
  const int nr = min(GEMM_BM, rows - r0), nc = min(GEMM_BN, cols - c0);
  const double* Ag = P + (roff + r0);
  const double* Bg = P + (roff + c0);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t = lane & 3;
  double acc[2][4][4];
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[a][b][c] = 0.0;

  auto load = [&](int stage, int k0) {
#pragma unroll
    for (int q = 0; q < (GEMM_BM * GEMM_BK) / 128; q++) {
      const int e = tid + q * 128;
      const int r = e % GEMM_BM, k = e / GEMM_BM;
      const bool kv = (k0 + k) < kend;
      const bool pa = kv && r < nr, pb = kv && r < nc;
      const size_t col = (size_t) (kv ? k0 + k : kbeg) * f;
      cp_async8(&As[stage][k][r], Ag + (pa ? r : 0) + col, pa);
      cp_async8(&Bs[stage][k][r], Bg + (pb ? r : 0) + col, pb);
    }
    cp_async_commit();
  };

  int stage = 0;
  load(0, kbeg);
  for (int k0 = kbeg; k0 < kend; k0 += GEMM_BK) {
    const bool more = k0 + GEMM_BK < kend;
    if (more) load(stage ^ 1, k0 + GEMM_BK);
    if (more) cp_async_wait<1>();
    else cp_async_wait<0>();
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GEMM_BK; kk += 8) {
      double a[2][4], b[4][2];
#pragma unroll
      for (int mi = 0; mi < 2; mi++) {
        const int r = wm * 32 + mi * 16 + g;
        a[mi][0] = As[stage][kk + t][r];
        a[mi][1] = As[stage][kk + t][r + 8];
        a[mi][2] = As[stage][kk + t + 4][r];
        a[mi][3] = As[stage][kk + t + 4][r + 8];
      }
#pragma unroll
      for (int ni = 0; ni < 4; ni++) {
        const int c = wn * 32 + ni * 8 + g;
        b[ni][0] = Bs[stage][kk + t][c];
        b[ni][1] = Bs[stage][kk + t + 4][c];
      }
#pragma unroll
      for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++) dmma16888(acc[mi][ni], a[mi], b[ni]);
    }
    __syncthreads();
    stage ^= 1;
  }
  double* C = Cbase + r0 + (size_t) c0 * ldc;
#pragma unroll
  for (int mi = 0; mi < 2; mi++)
#pragma unroll
    for (int ni = 0; ni < 4; ni++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int r = wm * 32 + mi * 16 + g + ((q & 2) ? 8 : 0);
        const int c = wn * 32 + ni * 8 + 2 * t + (q & 1);
        if (r < nr && c < nc && r0 + r >= c0 + c) C[r + (size_t) c * ldc] -= acc[mi][ni][q];
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

static double build_bytes(const Plan& P, const FrontDesc& F) {
  double by = 0.0;
  for (int ci = F.child_begin; ci < F.child_end; ci++) {
    const FrontDesc& C = P.fronts[P.children[ci]];
    const double mc = C.f - C.s;
    by += 8.0 * mc * (mc + 1.0) / 2.0 + 4.0 * mc;
  }
  const double m = F.f - F.s;
  by += 8.0 * ((double) F.f * F.s - (double) F.s * (F.s - 1) / 2.0) + 8.0 * m * (m + 1.0) / 2.0;
  by += 12.0 * (P.acol_ptr[F.acol_off + F.s] - P.acol_ptr[F.acol_off]);
  return by;
}

// small fronts: read children's U and A once, write panel and U once
static double front_bytes(const Plan& P, const FrontDesc& F) {
  return build_bytes(P, F);
}

static void set_smem_attrs() {
  static bool done = false;
  if (done) return;
  cudaFuncSetAttribute(k_small_front, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       SMALL_F_MAX * SMALL_F_MAX * (int) sizeof(double));
  cudaFuncSetAttribute(k_potrf_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) POTRF_SMEM);
  cudaFuncSetAttribute(k_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       2 * PANEL_NB * TLD * (int) sizeof(double));
  done = true;
}

int launch_numeric_fp64(const Plan& P, const DevPlan& D, const double* vals, double* L, double* U,
                        double* Dinv, int* status, cudaStream_t st) {
  set_smem_attrs();
  k_init_status<<<1, 1, 0, st>>>(status);
  count_launch();
  for (int h = 0; h < P.n_levels; h++) {
    const LevelPlan& LP = P.levels[h];
    // small fronts, in size classes so that the shared-memory request fits the class
    const int ns = (int) LP.small_fronts.size();
    if (ns > 0) {
      const int* lst = D.small_list + D.small_off[h];
      int b = 0;
      const int classes[3] = {32, 64, SMALL_F_MAX};
      for (int cl = 0; cl < 3 && b < ns; cl++) {
        int e = b;
        while (e < ns && P.fronts[LP.small_fronts[e]].f <= classes[cl]) e++;
        if (e > b) {
          const size_t smem = (size_t) classes[cl] * classes[cl] * sizeof(double);
          double fl = 0.0, by = 0.0;
          if (prof_enabled())
            for (int q = b; q < e; q++) {
              const FrontDesc& F = P.fronts[LP.small_fronts[q]];
              fl += front_flops(F);
              by += front_bytes(P, F);
            }
          prof_begin(KC_SMALL, st);
          k_small_front<<<e - b, 128, smem, st>>>(lst + b, D.fronts, D.children, D.maps, D.rows,
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
        for (int fi : LP.big_fronts) by += build_bytes(P, P.fronts[fi]);
      prof_begin(KC_BUILD, st);
      k_build<<<ntiles, 256, 0, st>>>(D.tiles + D.tile_off[h], D.fronts, D.children, D.maps, D.acol_ptr,
                                      D.a_rows, D.a_idx, vals, L, U, status);
      prof_end(KC_BUILD, st, 0.0, by);
      count_launch();
    }
    const size_t trsm_smem = 2 * PANEL_NB * TLD * sizeof(double);
    for (int kb = 0; kb < LP.max_s_big; kb += PANEL_NB) {
      int gx_t = 0, gx_g = 0;
      for (int fi : LP.big_fronts) {
        const FrontDesc& F = P.fronts[fi];
        if (kb >= F.s) continue;
        const int w = std::min(PANEL_NB, F.s - kb);
        gx_t = std::max(gx_t, (F.f - kb - w + TRSM_ROWS - 1) / TRSM_ROWS);
        const int cb = kb + w;
        if (cb < F.s) gx_g = std::max(gx_g, trap_tiles(F.f - cb, F.s - cb));
      }
      double fp = 0.0, ft = 0.0, fg = 0.0, bp = 0.0, bt = 0.0, bg = 0.0;
      if (prof_enabled())
        for (int fi : LP.big_fronts) {
          const FrontDesc& F = P.fronts[fi];
          if (kb >= F.s) continue;
          const double w = std::min(PANEL_NB, F.s - kb);
          const double below = F.f - kb - w;              // rows under the diagonal block
          const double sq = F.s - kb - w;                 // trailing columns of the panel
          fp += w * w * w / 3.0;
          bp += 8.0 * w * w;
          ft += below * w * w;
          bt += 16.0 * below * w + 8.0 * w * w / 2.0;
          fg += 2.0 * w * (sq * (sq + 1.0) / 2.0 + (F.f - F.s) * sq);
          bg += 16.0 * (sq * (sq + 1.0) / 2.0 + (F.f - F.s) * sq) + 8.0 * below * w;
        }
      prof_begin(KC_POTRF, st);
      k_potrf_diag<<<nb, 128, POTRF_SMEM, st>>>(blst, D.fronts, D.rows, L, Dinv, kb, status);
      prof_end(KC_POTRF, st, fp, bp);
      count_launch();
      if (gx_t > 0) {
        prof_begin(KC_TRSM, st);
        k_trsm<<<dim3(gx_t, nb), 128, trsm_smem, st>>>(blst, D.fronts, L, Dinv, kb, status);
        prof_end(KC_TRSM, st, ft, bt);
        count_launch();
      }
      if (gx_g > 0) {
        prof_begin(KC_GEMM_PANEL, st);
        k_gemm<<<dim3(gx_g, nb), 128, 0, st>>>(blst, D.fronts, L, U, kb, 0, status);
        prof_end(KC_GEMM_PANEL, st, fg, bg);
        count_launch();
      }
    }
    int gx_u = 0;
    for (int fi : LP.big_fronts) {
      const FrontDesc& F = P.fronts[fi];
      const int m = F.f - F.s;
      if (m > 0) gx_u = std::max(gx_u, trap_tiles(m, m));
    }
    if (gx_u > 0) {
      double fu = 0.0, bu = 0.0;
      if (prof_enabled())
        for (int fi : LP.big_fronts) {
          const FrontDesc& F = P.fronts[fi];
          const double m = F.f - F.s;
          fu += 2.0 * F.s * m * (m + 1.0) / 2.0;
          bu += 16.0 * m * (m + 1.0) / 2.0 + 8.0 * m * F.s;
        }
      prof_begin(KC_GEMM_U, st);
      k_gemm<<<dim3(gx_u, nb), 128, 0, st>>>(blst, D.fronts, L, U, 0, 1, status);
      prof_end(KC_GEMM_U, st, fu, bu);
      count_launch();
    }
  }
  return (int) cudaGetLastError();
}

}  // namespace tb

// Tunables and host-side launchers of the device kernels.
#pragma once

#include <cstdint>
#include <mutex>
#include <vector>
#include <cuda_runtime.h>

#include "internal.h"

namespace tb {

// fronts of order <= SMALL_F_MAX are built and factored entirely in shared
// memory by one CTA (k_small_front); larger ones go through the tiled path
constexpr int SMALL_F_MAX = 96;
// persistent fronts whose subtree has only fronts of order <= SMALL_WARP_F
// are factored by one warp each, the front's rows in the lanes' registers
constexpr int SMALL_WARP_F = 32;
// front-build tile (rows x columns of one front held in shared memory)
constexpr int BUILD_TR = 128;
constexpr int BUILD_TC = 32;
// block column width of the blocked partial Cholesky of large fronts
constexpr int PANEL_NB = 64;
// rows per CTA of the panel POTRF+TRSM kernel
constexpr int TRSM_ROWS = 64;
// GEMM tile of the trailing / update-matrix kernels
constexpr int GEMM_BM = 64;
constexpr int GEMM_BN = 64;
constexpr int GEMM_BK = 16;
// right-hand sides handled per solve pass
constexpr int SOLVE_NRHS = 8;
// small fronts up to this order are solved by one warp each (eight per CTA)
constexpr int SOLVE_WARP_F = 48;
// rows of L21 per CTA in the backward solve's partial products
constexpr int SOLVE_RCH = 512;

#ifdef __CUDACC__
// First index of the sorted a[0, n) whose value is >= key, found by one
// warp: 32 probes per round narrow the range 32-fold, so a search costs
// ceil(log32 n) dependent loads instead of log2 n.  Every lane returns the
// result; all 32 lanes must call it.
__device__ __forceinline__ int warp_lower_bound(const int* a, int n, int key) {
  const int lane = threadIdx.x & 31;
  int lo = 0, hi = n;
  while (hi - lo > 32) {
    const int step = (hi - lo + 31) / 32;
    const int p = lo + lane * step;
    const unsigned less = __ballot_sync(0xffffffffu, p < hi && a[p] < key);
    const int cnt = __popc(less);   // the probes below key form a prefix
    if (cnt == 0) return lo;
    const int nlo = lo + (cnt - 1) * step + 1;
    hi = min(hi, lo + cnt * step);
    lo = nlo;
  }
  const int p = lo + lane;
  return lo + __popc(__ballot_sync(0xffffffffu, p < hi && a[p] < key));
}
#endif

// Device copies of the plan arrays.
struct DevPlan {
  FrontDesc* fronts = nullptr;
  int* children = nullptr;
  int* rows = nullptr;
  int* maps = nullptr;
  int* acol_ptr = nullptr;
  int* a_rows = nullptr;
  int* a_idx = nullptr;
  int* small_list = nullptr;   // all levels, concatenated
  int* big_list = nullptr;
  TileChild* tile_ch = nullptr;   // per build tile, one record per child of its front
  Tile* tiles = nullptr;
  int2_* sfwd = nullptr;       // solve blocks, all levels concatenated
  int2_* sbwd = nullptr;
  int2_* sl21 = nullptr;
  int2_* dblk = nullptr;       // (front, 64-column block) of every big front's diagonal blocks
  int n_dblk = 0;
  int* small_num = nullptr;    // LevelPlan::small_numeric, all levels concatenated
  int* pers_list = nullptr;    // Plan::pers_fronts, pers_parent, pers_pending
  int* pers_parent = nullptr;
  int* pers_pending0 = nullptr;
  int* pers_work = nullptr;    // per factorization: pending counts (n_pers) + the two queue heads
  int* pers_solve = nullptr;   // per solve: pending counts and done flags (n_pers each) + two queue heads
  int n_pers = 0;
  std::vector<int> small_off, big_off, tile_off, sfwd_off, sbwd_off, sl21_off, small_num_off;  // per level (host)
  std::vector<int> lvl_max_f_small;               // per level (host)
};

int devplan_upload(const Plan& P, DevPlan* D, cudaStream_t st);
void devplan_free(DevPlan* D);

// numeric factorization over all levels; vals = A's values (device);
// status (device int) receives the smallest failing global column, or
// INT_MAX; returns a cudaError_t code
// the build tiles' child records (once per plan, after the upload)
int launch_tile_ranges(const DevPlan& D, int ntiles, cudaStream_t st);
int launch_numeric_fp64(const Plan& P, const DevPlan& D, const double* vals, double* L,
                        double* U, double* Dinv, int* status, cudaStream_t st);
// the same factorization with FP32 fronts (TF32x3 tensor products)
// sp: the split arena (Plan::sp_len floats; its contents are produced by the
// factorization itself), or nullptr to factor without it; sp_fmt its format
// (0 TF32 hi/lo, 1 FP16 hi/scaled lo)
int launch_numeric_fp32(const Plan& P, const DevPlan& D, const float* vals, float* L,
                        float* U, float* Dinv, float* sp, int sp_fmt, int* status, cudaStream_t st);

// status value recorded when a bounded device wait of the factorization gave
// up (never a column index)
constexpr int NUMERIC_TIMEOUT = -4;

// FP32 fronts: C -= A B^T on tcgen05 (TF32x3, 128x128 tiles, TMEM
// accumulator); same modes and arguments as the mma.sync GEMM.
// gemm_tc_init() sets the kernel's shared-memory limit once and reports
// whether the kernel is usable; gemm_tc_tiles() = CTAs per front.
// variant 0: 2-stage ring, 128 producer threads, 3 CTAs per SM; variant 1:
// 3-stage ring, 256 producer threads, 2 CTAs per SM (chosen per level and
// product by the autotuner)
bool gemm_tc_init();
int gemm_tc_tiles(int rows, int cols);
// the tcgen05 GEMM fed from the split arena by bulk copies (same modes)
bool gemm_sp_init();
int gemm_sp_tiles_u(int s, int f);
void launch_gemm_sp(int fmt, int gx, int nb, const int* list, const FrontDesc* fronts, const float* sp, float* L, float* U,
                    int c_lo, int c_hi, int k_lo, int k_hi, int mode, int* status, cudaStream_t st);
void launch_gemm_tc(int variant, int gx, int nb, const int* list, const FrontDesc* fronts, float* L, float* U,
                    int c_lo, int c_hi, int k_lo, int k_hi, int mode, int* status, cudaStream_t st);

// multi-RHS solve, device vectors in permuted order: X (n x nrhs, ld) from
// B (n x nrhs, ld); W scratch of P.v_len * SOLVE_NRHS doubles, Y n *
// SOLVE_NRHS doubles
// flags (P.n_blk ints) carry release/acquire handshakes between the CTAs of
// a big front; epoch must differ from every value they hold; status gets
// SOLVE_TIMEOUT if a bounded wait gave up
constexpr int SOLVE_TIMEOUT = -2;
// Dinv: the factor's 64x64 diagonal-block inverses (FrontDesc::dinv_off)
int launch_solve_fp64(const Plan& P, const DevPlan& D, const double* L, const double* Dinv, int nrhs, double* X,
                      const double* B, int ld, double* W, double* part, int* flags, int* epoch, int* status,
                      cudaStream_t st);
// the same solve on an FP32 factor with FP32 vectors
int launch_solve_fp32(const Plan& P, const DevPlan& D, const float* L, const float* Dinv, int nrhs, float* X,
                      const float* B, int ld, float* W, float* part, int* flags, int* epoch, int* status,
                      cudaStream_t st);

// sets the polling limit and the test offset of the solve's handshake waits
// on the current device (returns a cudaError_t code)
int solve_set_wait_controls(int limit, int skew);

// Device and pinned-host allocations of the library (alloc.cpp): counted,
// and failable on request (taucs_b200_allocation_induce_failure)
cudaError_t dmalloc_raw(void** p, size_t bytes);
cudaError_t dfree(void* p);
cudaError_t hmalloc_raw(void** p, size_t bytes);
cudaError_t hfree(void* p);
template <typename T>
inline cudaError_t dmalloc(T** p, size_t bytes) { return dmalloc_raw((void**) p, bytes); }
template <typename T>
inline cudaError_t hmalloc(T** p, size_t bytes) { return hmalloc_raw((void**) p, bytes); }

// GEMM tuning table (tune.cpp): record one factor's per-level times of both
// variants (t[v][2h + kind], ms), and fill a plan's choices from the table
void tune_record(const Plan& P, int prec, const std::vector<double> (&t)[2]);
bool tune_apply(Plan* P, int prec);

// device gathers of the request server and the batch entry points
// (refine.cu): out[k] = raw[vmap[k]]; dst[i] = src[perm[i]]; dst[perm[i]] = src[i]
int gather_values_device(long nnz, const int* d_vmap, const double* d_raw, double* d_out);
int perm_gather_device(int n, const int* d_perm, const double* src, double* dst);
int perm_scatter_device(int n, const int* d_perm, const double* src, double* dst);

// launch accounting
void count_launch(long k = 1);

// Per-device one-time setup.  Function attributes such as the dynamic
// shared-memory limit belong to the device that is current when they are
// set, so every launcher runs its setup once on each device it is used on.
// Returns the setup's result for the current device (false if there is no
// current device).  Safe to call from several host threads at once.
constexpr int MAX_DEVICES = 64;
struct PerDeviceOnce {
  std::once_flag once[MAX_DEVICES];
  bool ok[MAX_DEVICES] = {};
};
bool per_device_once(PerDeviceOnce& pd, bool (*setup)());

// Optional per-kernel-class timing: when enabled, launchers bracket every
// launch of a class with CUDA events on the launch stream and record the
// algorithmic flops and bytes of that launch.
enum KernelClass { KC_SMALL = 0, KC_BUILD, KC_LEAF, KC_DINV, KC_GEMM_PANEL, KC_GEMM_U, KC_SOLVE_FWD,
                   KC_SOLVE_BWD, KC_OTHER, KC_COUNT };
bool prof_enabled();
// every profiled launch: its class, the tag set when it was issued (the
// numeric factorization tags launches with their level) and its device time
struct ProfEntry {
  int kc, tag;
  float ms;
};
void prof_tag(int tag);
std::vector<ProfEntry> prof_take_log();
void prof_begin(int kc, cudaStream_t st);
void prof_end(int kc, cudaStream_t st, double flops, double bytes);

}  // namespace tb

// Internal declarations shared by the host and device translation units of
// libtaucs_b200.so.  Nothing here is part of the C ABI.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "taucs_b200.h"

namespace tb {

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
const char* last_error();
int tprintf(const char* fmt, ...);

// --------------------------------------------------------------- symbolic
// The supernodal structure exactly as the reference's symbolic phase leaves
// it (src/taucs_sn_llt.c:3663-4001): n_sn slots, slot n_sn is the virtual
// root, emptied slots have sn_size == 0.
struct Symbolic {
  int n = 0;
  int n_sn = 0;
  std::vector<int> sn_size;        // n_sn
  std::vector<int> sn_up_size;     // n_sn
  std::vector<int> first_child;    // n_sn + 1
  std::vector<int> next_child;     // n_sn + 1
  std::vector<std::vector<int>> sn_struct;  // n_sn (reference row order)
};

// etree of a permuted lower CCS pattern: parent[j], root = n
int etree(int n, const int* colptr, const int* rowind, int* parent);
// full symbolic phase; returns TAUCS_SUCCESS, TAUCS_ERROR_MAXDEPTH or
// TAUCS_ERROR_NOMEM
int symbolic_analyze(int n, const int* colptr, const int* rowind, int max_depth,
                     Symbolic* out);

// ------------------------------------------------------------ AMD ordering
int amd_order(int n, const int* colptr, const int* rowind, int* perm, int* invperm);
// multiple minimum external degree (the reference's "genmmd" ordering)
int mmd_order(int n, const int* colptr, const int* rowind, int* perm, int* invperm);

// ------------------------------------------------------------------- plan
// Front-build tile: rows [r0, r0+TILE_R) x columns [c0, c0+TILE_C) of the
// lower part of one front.
// c0 >= 0: panel region (front-local rows r0.., columns c0..);
// c0 < 0: update-matrix region, U-local rows r0.., columns -1-c0..
struct Tile {
  int front;   // device-order front index
  int r0, c0;
  int ch_off;  // first of the tile's child records (one per child of the front)
};

// Where child ci of a front lands in one build tile, found once per plan:
// the child's columns [ja, jb) and rows [ia, ib) (child-local indices) that
// map into the tile, with the child's map offset, order m and update matrix.
struct TileChild {
  int ja, jb, ia, ib;
  int map_off, mc;
  int64_t u_off;
};

struct int2_ {
  int a, b;
};

// Dense-kernel tile for the blocked partial factorization and the update
// of U (see numeric.cu).
struct GemmTile {
  int front;
  int i0, j0;
};

// One supernode in device order.
struct FrontDesc {
  int64_t l_off;      // panel offset (doubles) in the L arena; panel f x s, ld f
  int64_t u_off;      // update matrix offset in the U arena; m x m, ld m (-1 if m == 0)
  int64_t v_off;      // solve work-vector offset (f entries per right-hand side)
  int64_t dinv_off;   // inverses of the 64x64 diagonal blocks (big fronts), -1 otherwise
  int blk_off;        // solve flags: first of ceil(s/64) per big front, -1 otherwise
  int nchunk;         // solve: row chunks of L21 for the backward partial products
  int64_t part_off;   // solve: partial sums (nchunk x s x SOLVE_NRHS doubles), -1 if none
  int s, f;           // columns, front order (m = f - s)
  int child_begin;    // range in child list
  int child_end;
  int rows_off;       // offset of the sorted global row list (f entries)
  int map_off;        // offset of this front's map into its parent (m entries)
  int acol_off;       // offset into the A-column pointer table (s + 1 entries)
  int level;
  int parent;         // device-order parent index, -1 for roots
  int sn;             // reference slot
  int64_t sp_off;     // FP32 fronts: offset (floats) of the panel's split copy in the level's split
                      // arena (layout below), -1 for fronts factored whole in shared memory
};

// Split copy of an FP32 front's panel for the tensor-core products, in one
// of two formats: 0, TF32 hi and lo parts of every value (x = hi + lo, 4-byte
// elements); 1, FP16 hi and scaled lo parts (x = hi + lo / 2048, 2-byte
// elements).  Each part is laid out as 16-byte chunks of consecutive columns
// (4 or 8) for 8 consecutive rows: element (r, k) of part p at byte
// p * sp_part_bytes + ((k / cw) * rg + r / 8) * 128 + (r % 8) * 16 + (k % cw) * esz,
// cw = sp_chunk_cols, rg = ceil(f / 8) row groups; the columns run to a
// multiple of 4 chunks (one pipeline stage of the products).
#ifdef __CUDACC__
#define TB_HD __host__ __device__
#else
#define TB_HD
#endif
TB_HD inline int sp_chunk_cols(int fmt) { return fmt ? 8 : 4; }
TB_HD inline int64_t sp_kchunks(int s, int fmt) {
  const int kst = 4 * sp_chunk_cols(fmt);
  return ((int64_t) (s + kst - 1) / kst) * 4;
}
TB_HD inline int64_t sp_rgroups(int f) { return (f + 7) / 8; }
TB_HD inline int64_t sp_part_bytes(const FrontDesc& F, int fmt) { return sp_kchunks(F.s, fmt) * sp_rgroups(F.f) * 128; }

struct LevelPlan {
  int front_begin, front_end;      // fronts of this level (device order)
  // solve: big fronts are split into 64-row blocks, one CTA each
  std::vector<int2_> solve_fwd_blocks;   // (front, row block): the n_fwd_diag diagonal blocks first
  int n_fwd_diag = 0;
  std::vector<int2_> solve_bwd_blocks;   // (front, column block), last block first
  std::vector<int2_> solve_l21_tasks;    // (front, column block << 16 | row chunk)
  // small fronts, fused kernel (sorted by order f); the first small_warp of
  // them are small enough for the one-warp-per-front solve kernels
  std::vector<int> small_fronts;
  // the small fronts that the level launches of the numeric factorization
  // take (those with a big front below them); the others are factored by
  // the persistent launch (Plan::pers_fronts).  Sorted by order f.
  std::vector<int> small_numeric;
  int small_numeric_warp = 0;      // the first ones small enough for the one-warp solve kernels
  int small_warp = 0;
  // medium/large fronts
  std::vector<int> big_fronts;
  std::vector<Tile> build_tiles;
  int max_s_big = 0;               // largest s among big fronts
  int max_m_big = 0;
};

struct Plan {
  int n = 0;
  int n_fronts = 0;
  int n_levels = 0;
  int64_t l_len = 0;               // doubles in L arena
  int64_t u_len = 0;               // doubles in U arena (peak of planned lifetimes)
  int64_t v_len = 0;               // doubles of per-front work vectors (1 rhs)
  int64_t dinv_len = 0;            // doubles of diagonal-block inverses
  int n_blk = 0;                   // solve flags
  int64_t part_len = 0;            // doubles of partial sums: the backward ones, then the forward walk's
  int64_t fpart_off = 0;           // start of the walks' tagged pairs (2 x n_blk x 64 x SOLVE_NRHS, 8 bytes each)
  int64_t sp_len = 0;              // floats of the split arena (the largest level's split copies)
  // small fronts whose whole subtree is small: first those whose subtree
  // has only fronts of order <= SMALL_WARP_F (pers_nwarp of them, factored
  // one front per warp), then the others, each part in device (level)
  // order -- children always before their parent.  Two persistent launches
  // (one per part) take them from device-side queues in this order, each
  // once its children are done.  pers_parent: the task index of the front's
  // parent when that parent is in the list too, else -1; pers_pending: the
  // front's number of children (all of them in the list).
  std::vector<int> pers_fronts, pers_parent, pers_pending;
  int pers_nwarp = 0;
  int pers_fmax = 0;               // largest order f among the second part's fronts
  int64_t nnz = 0;
  std::vector<FrontDesc> fronts;
  std::vector<int> children;       // device-order child indices
  std::vector<int> rows;           // per front: f sorted global rows
  std::vector<int> maps;           // per non-root front: m parent-local indices
  std::vector<int> acol_ptr;       // per front: s+1 offsets into a_rows/a_idx
  std::vector<int> a_rows;         // local row of each A entry
  std::vector<int> a_idx;          // index of that entry in A's value array
  std::vector<LevelPlan> levels;
  double flops = 0.0;
  double ea_bytes = 0.0;
  double solve_bytes = 0.0;
  int max_front = 0, max_s = 0;
  // GEMM variant per level and product, [2h] panel updates, [2h + 1] the
  // update matrix; index 0 for FP64 fronts, 1 for FP32 fronts.  Empty or 0:
  // the default variant; set by the autotuner from measured times.
  std::vector<uint8_t> gemm_choice[2];
};

// words of the solve's handshake array cleared by every solve call: a chain
// flag per 64-row block; one more word follows, the walks' call counter
// (never cleared)
inline size_t solve_flag_words(const Plan& P) { return (size_t) P.n_blk; }

int build_plan(const Symbolic& S, int n, const int* colptr, const int* rowind, Plan* P);

}  // namespace tb

// FP32-front GEMM on the Blackwell tensor cores (tcgen05, TF32x3).
//
// The reference's SYRK/GEMM update of a front (src/taucs_sn_llt.c:1180, and
// the trailing updates inside LAPACK's POTRF at :1131) becomes, for FP32
// fronts,
//
//     C -= A B^T      (A: rows of the panel, B: columns, K = panel columns)
//
// computed as three TF32 products per element pair, lo*hi + hi*lo + hi*hi,
// accumulated in FP32 in tensor memory, which keeps FP32-level accuracy.  One CTA
// owns a 128 x 128 tile of the lower trapezoid of C:
//
//   producers  128 or 256 threads (warps 0-3 or 0-7): each loads one row of
//              the A and B K-slabs, or half of it (coalesced, 32 threads =
//              32 consecutive rows), splits every value into TF32 hi/lo
//              once, and stores the four operand parts into a 2- or 3-stage
//              shared-memory ring in the canonical K-major, no-swizzle
//              layout (8-row x 16-byte core matrices);
//   MMA warp   allocates 128 TMEM columns; one thread issues
//              tcgen05.mma.cta_group::1.kind::tf32 (M = 128, N = the tile's
//              columns rounded up to 16, K = 8) and frees each ring stage
//              with tcgen05.commit;
//   epilogue   the producer warps read their 32 TMEM lanes (tcgen05.ld
//              32x32b) and subtract the product from C, 32 consecutive rows
//              per store.
//
// Every mbarrier wait is bounded; a wait that gives up records
// NUMERIC_TIMEOUT in the status word and the CTA winds down (no further MMAs,
// MMAs in flight are awaited, TMEM is freed), so no launch can hang.

#include <climits>
#include <cstdint>

#include "kernels.h"

namespace tb {
namespace {

constexpr int TC_BM = 128, TC_BN = 128, TC_BK = 16;
constexpr int TC_PART = TC_BM * TC_BK * 4;      // one operand part (hi or lo) of one stage: 8 KB
constexpr int TC_STAGE = 4 * TC_PART;           // A_hi, A_lo, B_hi, B_lo
constexpr int TC_TMEM_COLS = 128;
template <int STAGES>
constexpr size_t tc_smem() { return (size_t) STAGES * TC_STAGE + 1024; }   // + alignment slack
constexpr unsigned TC_WAIT_LIMIT = 1u << 22;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned) __cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait; false when it gave up
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
  for (unsigned it = 0; it < TC_WAIT_LIMIT; it++)
    if (mbar_try(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// canonical K-major, no-swizzle operand: 16-byte rows of 4 TF32 values,
// core matrices of 8 rows (128 B); the two K halves of one MMA are LBO =
// 128 B apart, consecutive 8-row groups SBO = 512 B apart (K = 16 per stage)
__device__ __forceinline__ uint64_t tc_desc(unsigned addr) {
  return (uint64_t) ((addr >> 4) & 0x3FFFu) | ((uint64_t) (128 >> 4) << 16) | ((uint64_t) (512 >> 4) << 32) |
         (1ull << 46);
}

// kind::tf32 instruction descriptor: D f32, A/B tf32, both K-major, M = 128
__device__ __forceinline__ unsigned tc_idesc(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned) (n >> 3) << 17) | ((unsigned) (TC_BM >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(unsigned tmem, uint64_t a, uint64_t b, unsigned idesc, unsigned acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void tc_commit(unsigned bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// x = hi + lo with hi = x truncated to TF32 (exact in FP32) and lo = x - hi
// (exact); the tensor core uses the top 19 bits of lo, so each product
// keeps about 21 bits, which with FP32 accumulation is FP32-level accuracy.
__device__ __forceinline__ void tf32_split(float x, unsigned& hi, unsigned& lo) {
  hi = __float_as_uint(x) & 0xffffe000u;
  lo = __float_as_uint(x - __uint_as_float(hi));
}

__device__ __forceinline__ void st_shared_v4(unsigned addr, unsigned a, unsigned b, unsigned c, unsigned d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

__device__ __forceinline__ void tmem_ld32(unsigned taddr, unsigned (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void record_timeout(int* status) { atomicMin(status, NUMERIC_TIMEOUT); }

// mode 0: panel update of columns [c_lo, min(c_hi, s)) and all rows below
//         c_lo by the panel columns [k_lo, k_hi);
// mode 1: U -= L21 L21^T (K = [0, s))
template <int STAGES, int MINB, int NPROD>
__global__ void __launch_bounds__(NPROD + 32, MINB)
k_gemm_tc(const int* __restrict__ list, const FrontDesc* __restrict__ fronts, float* __restrict__ L,
          float* __restrict__ U, int c_lo, int c_hi, int k_lo, int k_hi, int mode, int* status) {
  __shared__ __align__(8) unsigned long long bars[2 * STAGES + 1];   // full[S], empty[S], done
  __shared__ unsigned tmem_slot;
  __shared__ int abort_cta;
  extern __shared__ __align__(16) unsigned char tc_raw[];
  if (*(volatile const int*) status != INT_MAX) return;
  const FrontDesc F = fronts[list[blockIdx.y]];
  const int f = F.f, s = F.s, m = f - s;
  int rows, cols, roff, kbeg, kend, ldc;
  const float* P = L + F.l_off;
  float* Cbase;
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
  if (kend <= kbeg) return;
  int idx = blockIdx.x, c0 = 0;
  for (;;) {
    if (c0 >= cols) return;
    const int nt_c = (rows - c0 + TC_BM - 1) / TC_BM;
    if (idx < nt_c) break;
    idx -= nt_c;
    c0 += TC_BN;
  }
  const int r0 = c0 + idx * TC_BM;
  const int nr = min(TC_BM, rows - r0), nc = min(TC_BN, cols - c0);
  const int nmma = (nc + 15) & ~15;
  const float* Ag = P + (roff + r0);
  const float* Bg = P + (roff + c0);
  float* C = Cbase + r0 + (size_t) c0 * ldc;
  const int nk = (kend - kbeg + TC_BK - 1) / TC_BK;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned sbase = (smem_u32(tc_raw) + 1023u) & ~1023u;
  const unsigned full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[STAGES]),
                 done = smem_u32(&bars[2 * STAGES]);
  if (tid == 0) {
    for (int i = 0; i < STAGES; i++) {
      mbar_init(full0 + 8 * i, NPROD / 32);   // one arrival per producer warp
      mbar_init(empty0 + 8 * i, 1);
    }
    mbar_init(done, 1);
    abort_cta = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  constexpr int MW = NPROD / 32;   // the MMA warp
  if (warp == MW) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = tmem_slot;

  if (warp < MW) {
    // ---- producers: thread t loads row t % 128 of the A and B K-slabs, K
    // range [kh, kh + KT) of each slab (KT = 16 with 128 producers, 8 with 256)
    constexpr int KT = TC_BK * TC_BM / NPROD;
    const int r = tid % TC_BM, kh = (tid / TC_BM) * KT;
    const bool ra = r < nr, rb = r < nc;
    const float* arow = Ag + r;
    const float* brow = Bg + r;
    const unsigned roff_s = (unsigned) ((r >> 3) * 512 + (r & 7) * 16 + (kh / 4) * 128);
    bool ok = true;
    // the next K-slab is loaded into registers while this one is split and
    // stored, so one slab's loads are always in flight
    float av[KT], bv[KT];
    auto load = [&](int kt, float (&a)[KT], float (&b)[KT]) {
      const int k0 = kbeg + kt * TC_BK + kh;
#pragma unroll
      for (int j = 0; j < KT; j++) {
        const int k = k0 + j;
        const bool kv = k < kend;
        a[j] = (ra && kv) ? arow[(size_t) k * f] : 0.0f;
        b[j] = (rb && kv) ? brow[(size_t) k * f] : 0.0f;
      }
    };
    // one K-slab: wait for its ring slot, split and store, release it to the
    // MMA thread; the next slab's loads are issued first
    auto stage = [&](int kt, float (&a)[KT], float (&b)[KT], float (&an)[KT], float (&bn)[KT]) -> bool {
      const int stg = kt % STAGES, use = kt / STAGES;
      if (kt + 1 < nk) load(kt + 1, an, bn);
      if (use > 0) {
        // one lane polls the ring slot; the warp follows it
        int got = 1;
        if (lane == 0) got = mbar_wait(empty0 + 8 * stg, (use - 1) & 1);
        got = __shfl_sync(0xffffffffu, got, 0);
        __syncwarp();   // orders the lanes' stores after lane 0's acquire
        if (!got) return false;
      }
      const unsigned st = sbase + stg * TC_STAGE + roff_s;
#pragma unroll
      for (int c = 0; c < KT / 4; c++) {
        unsigned h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; e++) tf32_split(a[4 * c + e], h[e], l[e]);
        st_shared_v4(st + 0 * TC_PART + c * 128, h[0], h[1], h[2], h[3]);
        st_shared_v4(st + 1 * TC_PART + c * 128, l[0], l[1], l[2], l[3]);
#pragma unroll
        for (int e = 0; e < 4; e++) tf32_split(b[4 * c + e], h[e], l[e]);
        st_shared_v4(st + 2 * TC_PART + c * 128, h[0], h[1], h[2], h[3]);
        st_shared_v4(st + 3 * TC_PART + c * 128, l[0], l[1], l[2], l[3]);
      }
      // generic-proxy stores become visible to the tensor core's async
      // proxy; the warp's stores are ordered before its one arrival
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(full0 + 8 * stg);
      return true;
    };
    // two register sets in alternation, so no slab is copied between them
    float a2[KT], b2[KT];
    load(0, av, bv);
    for (int kt = 0; kt < nk && ok; kt += 2) {
      ok = stage(kt, av, bv, a2, b2);
      if (ok && kt + 1 < nk) ok = stage(kt + 1, a2, b2, av, bv);
    }
    if (!ok) {
      record_timeout(status);
      abort_cta = 1;
    }
    // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (its rows);
    // with 256 producers the two warp quartets take half the columns each.
    // C is read 32 columns ahead of the accumulator so its loads overlap
    constexpr int QUARTETS = NPROD / 128;
    const int er = (warp & 3) * 32 + lane;
    const int cq0 = (warp >> 2) * (TC_BN / QUARTETS), cq1 = min(nc, cq0 + TC_BN / QUARTETS);
    float cv[32];
    auto loadC = [&](int cb) {
#pragma unroll
      for (int j = 0; j < 32; j++) {
        const int c = cb + j;
        cv[j] = (er < nr && c < cq1 && r0 + er >= c0 + c) ? C[er + (size_t) c * ldc] : 0.0f;
      }
    };
    if (cq0 < cq1) loadC(cq0);
    int gd = 1;
    if (lane == 0) gd = mbar_wait(done, 0);
    const bool got = __shfl_sync(0xffffffffu, gd, 0) != 0;
    __syncwarp();
    if (!got) record_timeout(status);
    tc_fence_after();
    // tcgen05.ld is warp-collective: the decision must be warp-uniform
    if (__all_sync(0xffffffffu, got && ok && !*(volatile int*) &abort_cta)) {
      const unsigned tl = tmem + ((unsigned) ((warp & 3) * 32) << 16);
      for (int cb = cq0; cb < cq1; cb += 32) {
        unsigned v[32];
        tmem_ld32(tl + cb, v);
        float out[32];
#pragma unroll
        for (int j = 0; j < 32; j++) out[j] = cv[j] - __uint_as_float(v[j]);
        if (cb + 32 < cq1) loadC(cb + 32);
        if (er < nr) {
#pragma unroll
          for (int j = 0; j < 32; j++) {
            const int c = cb + j;
            if (c < cq1 && r0 + er >= c0 + c) C[er + (size_t) c * ldc] = out[j];
          }
        }
      }
    }
  } else if (lane == 0) {
    // ---- MMA issue, one thread
    const unsigned idesc = tc_idesc(nmma);
    bool ok = true;
    for (int kt = 0; kt < nk; kt++) {
      const int stg = kt % STAGES, use = kt / STAGES;
      if (!mbar_wait(full0 + 8 * stg, use & 1)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const unsigned st = sbase + stg * TC_STAGE;
#pragma unroll
      for (int j = 0; j < TC_BK / 8; j++) {
        const uint64_t ah = tc_desc(st + 0 * TC_PART + j * 256), al = tc_desc(st + 1 * TC_PART + j * 256);
        const uint64_t bh = tc_desc(st + 2 * TC_PART + j * 256), bl = tc_desc(st + 3 * TC_PART + j * 256);
        tc_mma(tmem, al, bh, idesc, (kt | j) != 0);
        tc_mma(tmem, ah, bl, idesc, 1u);
        tc_mma(tmem, ah, bh, idesc, 1u);
      }
      tc_commit(empty0 + 8 * stg);
    }
    if (!ok) {
      record_timeout(status);
      abort_cta = 1;
    }
    // done fires once every MMA issued above has completed
    tc_commit(done);
    if (!mbar_wait(done, 0)) record_timeout(status);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == MW) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS) : "memory");
  }
}

// ------------------------------------------------------------------------
// The same products with the operands already split: the panel leaves
// write every final value of a big FP32 front, split, into the split arena
// in the operand layout of the MMAs (16-byte chunks of consecutive columns
// for 8 rows; FrontDesc::sp_off), either as TF32 hi and lo (FMT 0) or as
// FP16 hi and lo scaled by 2^11 (FMT 1).  A 128-row slab of one chunk is 2 KB
// of contiguous memory there, so four chunks (K = 16 TF32 or 32 FP16
// columns) of the four operand parts (A hi/lo, B hi/lo) arrive in shared
// memory as 16 bulk copies (cp.async.bulk, completion counted in bytes on the
// stage's mbarrier), issued by 16 lanes of warp 0 -- no thread touches an
// operand value on the way.  Warp 1's lane 0 issues the MMAs: TF32,
// lo*hi + hi*lo + hi*hi into one accumulator; FP16 (kind::f16, twice the
// TF32 rate), hi*hi into one accumulator and hi*lo + lo*hi into a second,
// combined in the epilogue as acc0 + acc1 / 2048.  All four warps then run
// the epilogue from TMEM.  The tiles of the update matrix (mode 1) start at
// the row group of row s, so a tile may hold up to 7 rows of the panel above
// U; they are masked.

constexpr int SP_CHUNK = 16 * 128;             // bytes of one 16-byte-wide chunk of a 128-row slab
constexpr int SP_PARTB = 4 * SP_CHUNK;         // four chunks per stage
constexpr int SP_STAGE = 4 * SP_PARTB;         // A hi, A lo, B hi, B lo: 32 KB
template <int STAGES>
constexpr size_t sp_smem() { return (size_t) STAGES * SP_STAGE + 1024; }

// kind::f16 instruction descriptor: D f32, A/B f16, both K-major, M = 128
__device__ __forceinline__ unsigned f16_idesc(int n) {
  return (1u << 4) | ((unsigned) (n >> 3) << 17) | ((unsigned) (TC_BM >> 4) << 24);
}

__device__ __forceinline__ void f16_mma(unsigned tmem, uint64_t a, uint64_t b, unsigned idesc, unsigned acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

// K-major, no swizzle, chunk-major: the two 16-byte K halves of one MMA are
// LBO = one chunk (2 KB) apart, consecutive 8-row groups SBO = 128 B apart
__device__ __forceinline__ uint64_t sp_desc(unsigned addr) {
  return (uint64_t) ((addr >> 4) & 0x3FFFu) | ((uint64_t) (SP_CHUNK >> 4) << 16) | ((uint64_t) (128 >> 4) << 32) |
         (1ull << 46);
}

__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

template <int STAGES, int FMT>
__global__ void __launch_bounds__(128, 2)
k_gemm_sp(const int* __restrict__ list, const FrontDesc* __restrict__ fronts, const float* __restrict__ sp,
          float* __restrict__ L, float* __restrict__ U, int c_lo, int c_hi, int k_lo, int k_hi, int mode,
          int* status) {
  __shared__ __align__(8) unsigned long long bars[2 * STAGES + 1];   // full[S], empty[S], done
  __shared__ unsigned tmem_slot;
  __shared__ int abort_cta;
  extern __shared__ __align__(16) unsigned char sp_raw[];
  if (*(volatile const int*) status != INT_MAX) return;
  const FrontDesc F = fronts[list[blockIdx.y]];
  const int f = F.f, s = F.s, m = f - s;
  // tile grid origin (a row-group boundary), the valid rows/columns and K
  int base, rows, cols, lo, kbeg, kend;
  if (mode == 0) {
    const int ce = min(c_hi, s);
    if (c_lo >= ce) return;
    base = c_lo; rows = f - c_lo; cols = ce - c_lo; lo = c_lo;
    kbeg = k_lo; kend = k_hi;
  } else {
    if (m <= 0 || s <= 0) return;
    base = s & ~7; rows = f - base; cols = f - base; lo = s;
    kbeg = 0; kend = s;
  }
  if (kend <= kbeg) return;
  int idx = blockIdx.x, c0 = 0;
  for (;;) {
    if (c0 >= cols) return;
    const int nt_c = (rows - c0 + TC_BM - 1) / TC_BM;
    if (idx < nt_c) break;
    idx -= nt_c;
    c0 += TC_BN;
  }
  const int r0 = c0 + idx * TC_BM;
  const int R0 = base + r0, C0 = base + c0;            // first front row of the tile's rows / columns
  const int nr = min(TC_BM, rows - r0), nc = min(TC_BN, cols - c0);
  const int nmma = (nc + 15) & ~15;
  constexpr int CW = FMT ? 8 : 4;               // columns per chunk
  constexpr int BK = 4 * CW;                     // K per stage
  constexpr unsigned TMEM_COLS = FMT ? 2 * TC_TMEM_COLS : TC_TMEM_COLS;
  const int nk = (kend - kbeg + BK - 1) / BK;
  const int rg = (int) sp_rgroups(f);
  const unsigned char* part0 = reinterpret_cast<const unsigned char*>(sp + F.sp_off);
  const unsigned char* part1 = part0 + sp_part_bytes(F, FMT);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned sbase = (smem_u32(sp_raw) + 1023u) & ~1023u;
  const unsigned full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[STAGES]),
                 done = smem_u32(&bars[2 * STAGES]);
  if (tid == 0) {
    for (int i = 0; i < STAGES; i++) {
      mbar_init(full0 + 8 * i, 1);
      mbar_init(empty0 + 8 * i, 1);
    }
    mbar_init(done, 1);
    abort_cta = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = tmem_slot;

  if (warp == 0) {
    // ---- producer: lane q < 16 copies chunk q % 4 of operand part q / 4
    const int p = lane >> 2, c = lane & 3;
    const unsigned char* pb = (p & 1) ? part1 : part0;
    const int g0 = ((p < 2) ? R0 : C0) >> 3;
    for (int kt = 0; kt < nk; kt++) {
      const int stg = kt % STAGES, use = kt / STAGES;
      if (use > 0) {
        int got = 1;
        if (lane == 0) got = mbar_wait(empty0 + 8 * stg, (use - 1) & 1);
        got = __shfl_sync(0xffffffffu, got, 0);
        if (!got) {
          if (lane == 0) {
            record_timeout(status);
            abort_cta = 1;
          }
          break;
        }
      }
      if (lane == 0) mbar_expect_tx(full0 + 8 * stg, SP_STAGE);
      __syncwarp();
      if (lane < 16) {
        const int64_t kc = (kbeg + kt * BK) / CW + c;
        const unsigned char* src = pb + (kc * rg + g0) * 128;
        bulk_g2s(sbase + stg * SP_STAGE + p * SP_PARTB + c * SP_CHUNK, src, SP_CHUNK, full0 + 8 * stg);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issue, one thread: two MMAs of K = 2 chunks per stage
    const unsigned idesc = FMT ? f16_idesc(nmma) : tc_idesc(nmma);
    bool ok = true;
    for (int kt = 0; kt < nk; kt++) {
      const int stg = kt % STAGES, use = kt / STAGES;
      if (!mbar_wait(full0 + 8 * stg, use & 1)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const unsigned st = sbase + stg * SP_STAGE;
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const unsigned o = 2 * j * SP_CHUNK;
        const uint64_t ah = sp_desc(st + 0 * SP_PARTB + o), al = sp_desc(st + 1 * SP_PARTB + o);
        const uint64_t bh = sp_desc(st + 2 * SP_PARTB + o), bl = sp_desc(st + 3 * SP_PARTB + o);
        const unsigned first = (kt | j) != 0;
        if (FMT == 0) {
          tc_mma(tmem, al, bh, idesc, first);
          tc_mma(tmem, ah, bl, idesc, 1u);
          tc_mma(tmem, ah, bh, idesc, 1u);
        } else {
          f16_mma(tmem, ah, bh, idesc, first);
          f16_mma(tmem + TC_TMEM_COLS, ah, bl, idesc, first);
          f16_mma(tmem + TC_TMEM_COLS, al, bh, idesc, 1u);
        }
      }
      tc_commit(empty0 + 8 * stg);
    }
    if (!ok) {
      record_timeout(status);
      abort_cta = 1;
    }
    // done fires once every MMA issued above has completed
    tc_commit(done);
  }
  // ---- epilogue: warp w owns TMEM lanes (tile rows) 32 w .. 32 w + 31.
  // The first 32 columns of the old C rows are loaded before the wait for
  // the products (they do not depend on them), and each later group while
  // the group before it is stored
  const int er = warp * 32 + lane;
  const int row = R0 + er;
  const bool rv = er < nr && row >= lo;
  float* Cp = nullptr;
  int64_t ldc = 0;
  if (mode == 0) {
    Cp = L + F.l_off + row;
    ldc = f;
  } else {
    Cp = U + F.u_off + (row - s);
    ldc = m;
  }
  const int coff = (mode == 0) ? 0 : s;
  // all 32 loads of a group are issued before the first store: interleaved,
  // each load would wait for the store before it (the compiler cannot rule
  // out that they alias), one memory latency per element
  auto load_old = [&](int cb, float (&o)[32]) {
#pragma unroll
    for (int j = 0; j < 32; j++) {
      const int col = C0 + cb + j;
      o[j] = (rv && cb + j < nc && col >= lo && row >= col) ? Cp[(int64_t) (col - coff) * ldc] : 0.0f;
    }
  };
  float oldn[32];
  load_old(0, oldn);
  int gd = 1;
  if (lane == 0) gd = mbar_wait(done, 0);
  const bool got = __shfl_sync(0xffffffffu, gd, 0) != 0;
  __syncwarp();
  if (!got && lane == 0) record_timeout(status);
  tc_fence_after();
  // tcgen05.ld is warp-collective: the decision must be warp-uniform
  if (__all_sync(0xffffffffu, got && !*(volatile int*) &abort_cta)) {
    const unsigned tl = tmem + ((unsigned) (warp * 32) << 16);
    for (int cb = 0; cb < nc; cb += 32) {
      float old[32];
#pragma unroll
      for (int j = 0; j < 32; j++) old[j] = oldn[j];
      if (cb + 32 < nc) load_old(cb + 32, oldn);
      unsigned v[32];
      tmem_ld32(tl + cb, v);
      if (FMT) {
        unsigned v1[32];
        tmem_ld32(tl + TC_TMEM_COLS + cb, v1);
#pragma unroll
        for (int j = 0; j < 32; j++)
          v[j] = __float_as_uint(__uint_as_float(v[j]) + __uint_as_float(v1[j]) * (1.0f / 2048.0f));
      }
      if (rv) {
#pragma unroll
        for (int j = 0; j < 32; j++) {
          const int col = C0 + cb + j;
          if (cb + j < nc && col >= lo && row >= col) Cp[(int64_t) (col - coff) * ldc] = old[j] - __uint_as_float(v[j]);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

}  // namespace

bool gemm_sp_init() {
  static PerDeviceOnce pd;
  return per_device_once(pd, [] {
    return cudaFuncSetAttribute(k_gemm_sp<3, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sp_smem<3>()) ==
               cudaSuccess &&
           cudaFuncSetAttribute(k_gemm_sp<3, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sp_smem<3>()) ==
               cudaSuccess;
  });
}

// tiles of one front in mode 1 start at the row group of row s
int gemm_sp_tiles_u(int s, int f) {
  const int n = f - (s & ~7);
  return gemm_tc_tiles(n, n);
}

void launch_gemm_sp(int fmt, int gx, int nb, const int* list, const FrontDesc* fronts, const float* sp, float* L,
                    float* U, int c_lo, int c_hi, int k_lo, int k_hi, int mode, int* status, cudaStream_t st) {
  if (fmt)
    k_gemm_sp<3, 1><<<dim3(gx, nb), 128, sp_smem<3>(), st>>>(list, fronts, sp, L, U, c_lo, c_hi, k_lo, k_hi, mode,
                                                             status);
  else
    k_gemm_sp<3, 0><<<dim3(gx, nb), 128, sp_smem<3>(), st>>>(list, fronts, sp, L, U, c_lo, c_hi, k_lo, k_hi, mode,
                                                             status);
}

// variant 0: two-stage ring (65 KB), 128 producers, three CTAs per SM;
// variant 1: three-stage ring (97 KB), 256 producers, two CTAs per SM
bool gemm_tc_init() {
  // once per device (request-server workers reach this concurrently)
  static PerDeviceOnce pd;
  return per_device_once(pd, [] {
    const cudaError_t e0 = cudaFuncSetAttribute(k_gemm_tc<2, 3, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int) tc_smem<2>());
    const cudaError_t e1 = cudaFuncSetAttribute(k_gemm_tc<3, 2, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int) tc_smem<3>());
    return e0 == cudaSuccess && e1 == cudaSuccess;
  });
}

int gemm_tc_tiles(int rows, int cols) {
  int t = 0;
  for (int c0 = 0; c0 < cols; c0 += TC_BN) t += (rows - c0 + TC_BM - 1) / TC_BM;
  return t;
}

void launch_gemm_tc(int variant, int gx, int nb, const int* list, const FrontDesc* fronts, float* L, float* U,
                    int c_lo, int c_hi, int k_lo, int k_hi, int mode, int* status, cudaStream_t st) {
  if (variant == 1)
    k_gemm_tc<3, 2, 256><<<dim3(gx, nb), 256 + 32, tc_smem<3>(), st>>>(list, fronts, L, U, c_lo, c_hi, k_lo, k_hi,
                                                                       mode, status);
  else
    k_gemm_tc<2, 3, 128><<<dim3(gx, nb), 128 + 32, tc_smem<2>(), st>>>(list, fronts, L, U, c_lo, c_hi, k_lo, k_hi,
                                                                       mode, status);
}

}  // namespace tb

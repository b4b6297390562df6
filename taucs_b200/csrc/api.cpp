// C ABI entry points of libtaucs_b200.so: the reference's factor / solve /
// free / convert interface (src/taucs_sn_llt.c:2892-3241 generic dispatch,
// :1979-2209 double instantiations, :2844-2885 solve, :803-1006 helpers) and
// taucs_linsolve (src/taucs_linsolve.c:189-622), implemented over the device
// plan and kernels.  There is no CPU numeric path: when CUDA is unavailable
// the numeric functions fail with the reference's error returns.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>

#include "factor.h"

namespace tb {

static thread_local cudaStream_t g_stream = nullptr;
cudaStream_t current_stream() { return g_stream; }

static std::atomic<long> g_launches{0};
void count_launch(long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

bool cuda_ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return false;
}

template <class T>
static bool dev_upload(T** dst, const T* src, size_t n, cudaStream_t st) {
  if (n == 0) n = 1;
  if (!cuda_ok(tb::dmalloc((void**) dst, n * sizeof(T)), "cudaMalloc")) return false;
  if (src) return cuda_ok(cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
  return true;
}

int devplan_upload(const Plan& P, DevPlan* D, cudaStream_t st) {
  std::vector<int> small, big, small_num;
  std::vector<Tile> tiles;
  std::vector<int2_> sf, sb, sl;
  D->small_off.clear(); D->big_off.clear(); D->tile_off.clear(); D->sfwd_off.clear(); D->sbwd_off.clear();
  D->sl21_off.clear(); D->small_num_off.clear();
  for (const LevelPlan& LP : P.levels) {
    D->small_num_off.push_back((int) small_num.size());
    small_num.insert(small_num.end(), LP.small_numeric.begin(), LP.small_numeric.end());
    D->small_off.push_back((int) small.size());
    D->big_off.push_back((int) big.size());
    D->tile_off.push_back((int) tiles.size());
    D->sfwd_off.push_back((int) sf.size());
    D->sbwd_off.push_back((int) sb.size());
    D->sl21_off.push_back((int) sl.size());
    small.insert(small.end(), LP.small_fronts.begin(), LP.small_fronts.end());
    big.insert(big.end(), LP.big_fronts.begin(), LP.big_fronts.end());
    tiles.insert(tiles.end(), LP.build_tiles.begin(), LP.build_tiles.end());
    sf.insert(sf.end(), LP.solve_fwd_blocks.begin(), LP.solve_fwd_blocks.end());
    sb.insert(sb.end(), LP.solve_bwd_blocks.begin(), LP.solve_bwd_blocks.end());
    sl.insert(sl.end(), LP.solve_l21_tasks.begin(), LP.solve_l21_tasks.end());
  }
  // each tile's child records follow one another, one per child of its front
  int64_t nrec = 0;
  for (Tile& t : tiles) {
    t.ch_off = (int) nrec;
    nrec += P.fronts[t.front].child_end - P.fronts[t.front].child_begin;
  }
  std::vector<int2_> dblk;
  for (int i = 0; i < (int) P.fronts.size(); i++)
    if (P.fronts[i].dinv_off >= 0)
      for (int b = 0; b * PANEL_NB < P.fronts[i].s; b++) dblk.push_back(int2_{i, b});
  D->n_dblk = (int) dblk.size();
  D->n_pers = (int) P.pers_fronts.size();
  bool ok = dev_upload(&D->fronts, P.fronts.data(), P.fronts.size(), st)
         && dev_upload(&D->small_num, small_num.data(), small_num.size(), st)
         && dev_upload(&D->pers_list, P.pers_fronts.data(), P.pers_fronts.size(), st)
         && dev_upload(&D->pers_parent, P.pers_parent.data(), P.pers_parent.size(), st)
         && dev_upload(&D->pers_pending0, P.pers_pending.data(), P.pers_pending.size(), st)
         && dev_upload(&D->pers_work, (const int*) nullptr, P.pers_fronts.size() + 2, st)
         && dev_upload(&D->pers_solve, (const int*) nullptr, 2 * P.pers_fronts.size() + 2, st)
         && dev_upload(&D->dblk, dblk.data(), dblk.size(), st)
         && dev_upload(&D->children, P.children.data(), P.children.size(), st)
         && dev_upload(&D->rows, P.rows.data(), P.rows.size(), st)
         && dev_upload(&D->maps, P.maps.data(), P.maps.size(), st)
         && dev_upload(&D->acol_ptr, P.acol_ptr.data(), P.acol_ptr.size(), st)
         && dev_upload(&D->a_rows, P.a_rows.data(), P.a_rows.size(), st)
         && dev_upload(&D->a_idx, P.a_idx.data(), P.a_idx.size(), st)
         && dev_upload(&D->small_list, small.data(), small.size(), st)
         && dev_upload(&D->big_list, big.data(), big.size(), st)
         && dev_upload(&D->tiles, tiles.data(), tiles.size(), st)
         && dev_upload(&D->sfwd, sf.data(), sf.size(), st)
         && dev_upload(&D->sbwd, sb.data(), sb.size(), st)
         && dev_upload(&D->sl21, sl.data(), sl.size(), st)
         && dev_upload(&D->tile_ch, (const TileChild*) nullptr, (size_t) std::max<int64_t>(nrec, 1), st);
  // the records, found once per plan on the device
  if (ok && !tiles.empty()) ok = cuda_ok((cudaError_t) launch_tile_ranges(*D, (int) tiles.size(), st), "tile ranges");
  if (ok) ok = cuda_ok(cudaStreamSynchronize(st), "plan upload");
  return ok ? 0 : -1;
}

void devplan_free(DevPlan* D) {
  tb::dfree(D->fronts); tb::dfree(D->children); tb::dfree(D->rows); tb::dfree(D->maps);
  tb::dfree(D->acol_ptr); tb::dfree(D->a_rows); tb::dfree(D->a_idx);
  tb::dfree(D->small_list); tb::dfree(D->big_list); tb::dfree(D->tiles); tb::dfree(D->tile_ch);
  tb::dfree(D->sfwd); tb::dfree(D->sbwd); tb::dfree(D->sl21); tb::dfree(D->dblk);
  tb::dfree(D->small_num); tb::dfree(D->pers_list); tb::dfree(D->pers_parent); tb::dfree(D->pers_pending0);
  tb::dfree(D->pers_work); tb::dfree(D->pers_solve);
  *D = DevPlan();
}

static bool graphs_enabled() {
  static const bool on = [] {
    const char* e = getenv("TAUCS_B200_NO_GRAPHS");
    return !(e && *e && strcmp(e, "0") != 0);
  }();
  return on;
}

void drop_graphs(Factor* F) {
  for (auto& kv : F->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  F->graphs.clear();
}

int run_graphed(Factor* F, const GraphKey& key, cudaStream_t st, const std::function<int(cudaStream_t)>& record) {
  if (!graphs_enabled() || prof_enabled()) return record(st);
  Factor::Graph& g = F->graphs[key];
  if (!g.seen) {
    g.seen = true;
    if (!F->graph_first_use) return record(st);
  }
  if (!g.exec) {
    if (!F->cap_stream && cudaStreamCreateWithFlags(&F->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
      F->cap_stream = nullptr;
      return record(st);
    }
    // recorded on a private stream (the legacy default stream cannot be
    // captured); replays are ordered on st
    cudaGraph_t graph = nullptr;
    const long l0 = g_launches.load();
    int rc = (int) cudaStreamBeginCapture(F->cap_stream, cudaStreamCaptureModeThreadLocal);
    if (rc == 0) {
      rc = record(F->cap_stream);
      const cudaError_t ec = cudaStreamEndCapture(F->cap_stream, &graph);
      if (rc == 0) rc = (int) ec;
    }
    const long nl = g_launches.load() - l0;
    count_launch(-nl);   // recorded, not run
    if (rc == 0 && graph) rc = (int) cudaGraphInstantiate(&g.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (rc != 0 || !g.exec) {
      g.exec = nullptr;
      cudaGetLastError();
      return record(st);
    }
    g.launches = nl;
  }
  count_launch(g.launches);
  return (int) cudaGraphLaunch(g.exec, st);
}

void invalidate_numeric(Factor* F) {
  F->has_numeric = false;
  F->has_numeric32 = false;
}

void free_numeric(Factor* F) {
  drop_graphs(F);
  tb::dfree(F->dL); F->dL = nullptr;
  tb::dfree(F->dU); F->dU = nullptr;
  tb::dfree(F->dDinv); F->dDinv = nullptr;
  tb::dfree(F->dL32); F->dL32 = nullptr;
  tb::dfree(F->dSp32); F->dSp32 = nullptr;
  tb::dfree(F->dU32); F->dU32 = nullptr;
  tb::dfree(F->dDinv32); F->dDinv32 = nullptr;
  F->has_numeric = false;
  F->has_numeric32 = false;
}

static void free_device(Factor* F) {
  free_numeric(F);
  tb::dfree(F->batch.d_cvmap); F->batch.d_cvmap = nullptr;
  tb::dfree(F->batch.d_cperm); F->batch.d_cperm = nullptr;
  tb::dfree(F->batch.d_raw); F->batch.d_raw = nullptr;
  tb::dfree(F->batch.d_b); F->batch.d_b = nullptr;
  tb::dfree(F->batch.d_x); F->batch.d_x = nullptr;
  tb::hfree(F->batch.h_raw); F->batch.h_raw = nullptr;
  if (F->cap_stream) cudaStreamDestroy(F->cap_stream);
  F->cap_stream = nullptr;
  if (F->dev_ready) devplan_free(&F->dp);
  tb::dfree(F->dA); F->dA = nullptr;
  tb::dfree(F->dstatus); F->dstatus = nullptr;
  tb::dfree(F->dW); F->dW = nullptr;
  tb::dfree(F->dpart); F->dpart = nullptr;
  tb::dfree(F->dX); F->dX = nullptr;
  tb::dfree(F->dscale); F->dscale = nullptr;
  tb::dfree(F->dcolptr); F->dcolptr = nullptr;
  tb::dfree(F->drowind); F->drowind = nullptr;
  tb::dfree(F->dA32); F->dA32 = nullptr;
  tb::dfree(F->dW32); F->dW32 = nullptr;
  tb::dfree(F->dpart32); F->dpart32 = nullptr;
  tb::dfree(F->dV32); F->dV32 = nullptr;
  tb::dfree(F->dcolidx); F->dcolidx = nullptr;
  tb::dfree(F->ddiagpos); F->ddiagpos = nullptr;
  tb::dfree(F->dcsr_ptr); F->dcsr_ptr = nullptr;
  tb::dfree(F->dcsr_col); F->dcsr_col = nullptr;
  tb::dfree(F->dcsr_val); F->dcsr_val = nullptr;
  tb::dfree(F->dR); F->dR = nullptr;
  tb::dfree(F->dXi); F->dXi = nullptr;
  tb::dfree(F->dseg); F->dseg = nullptr;
  tb::dfree(F->dXr); F->dXr = nullptr;
  tb::dfree(F->dBr); F->dBr = nullptr;
  tb::dfree(F->dnorm); F->dnorm = nullptr;
  if (F->hnorm) tb::hfree(F->hnorm);
  F->hnorm = nullptr;
  tb::dfree(F->dpcg); F->dpcg = nullptr;
  tb::dfree(F->ddot_part); F->ddot_part = nullptr;
  tb::dfree(F->ddot); F->ddot = nullptr;
  if (F->hdot) tb::hfree(F->hdot);
  F->hdot = nullptr;
  F->refine_ready = false;
  tb::dfree(F->dflags); F->dflags = nullptr;
  if (F->hstatus) tb::hfree(F->hstatus);
  F->hstatus = nullptr;
  F->dev_ready = false;
}

// device plan and per-handle buffers, allocated on the first numeric call
int ensure_device(Factor* F) {
  if (F->dev_ready) return 0;
  int dev = 0;
  if (!cuda_ok(cudaGetDevice(&dev), "cudaGetDevice")) return -1;
  cudaDeviceProp prop;
  if (!cuda_ok(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties")) return -1;
  if (prop.major < 10) {
    set_error("this library is built for sm_100a (B200); the current device is not");
    return -1;
  }
  F->device = dev;
  cudaStream_t st = current_stream();
  if (devplan_upload(F->plan, &F->dp, st)) { devplan_free(&F->dp); return -1; }
  F->dev_ready = true;
  const Plan& P = F->plan;
  bool ok = dev_upload(&F->dA, (const double*) nullptr, (size_t) P.nnz, st)
         && dev_upload(&F->dstatus, (const int*) nullptr, 2, st)
         && dev_upload(&F->dflags, (const int*) nullptr, solve_flag_words(P) + 1, st)
         && cuda_ok(cudaMemsetAsync(F->dflags, 0, sizeof(int) * (solve_flag_words(P) + 1), st), "flags")
         && dev_upload(&F->dW, (const double*) nullptr, (size_t) P.v_len * SOLVE_NRHS, st)
         && dev_upload(&F->dpart, (const double*) nullptr, (size_t) P.part_len, st)
         && dev_upload(&F->dX, (const double*) nullptr, (size_t) F->n * SOLVE_NRHS, st)
         && dev_upload(&F->dcolptr, F->colptr.data(), F->colptr.size(), st)
         && dev_upload(&F->drowind, F->rowind.data(), F->rowind.size(), st)
         && cuda_ok(tb::hmalloc((void**) &F->hstatus, 2 * sizeof(int)), "cudaMallocHost");
  if (ok) ok = cuda_ok(cudaStreamSynchronize(st), "upload");
  if (!ok) { free_device(F); return -1; }
  return 0;
}

static bool pattern_matches(const Factor* F, const taucs_ccs_matrix* A) {
  if (A->n != F->n) return false;
  if (memcmp(A->colptr, F->colptr.data(), sizeof(int) * (F->n + 1))) return false;
  return !memcmp(A->rowind, F->rowind.data(), sizeof(int) * (size_t) F->colptr[F->n]);
}

static bool check_matrix(const taucs_ccs_matrix* A, const char* who) {
  if (!A) { set_error(std::string(who) + ": NULL matrix"); return false; }
  if (!(A->flags & TAUCS_DOUBLE)) { set_error(std::string(who) + ": only TAUCS_DOUBLE matrices are supported"); return false; }
  if (!(A->flags & (TAUCS_SYMMETRIC | TAUCS_HERMITIAN)) || !(A->flags & TAUCS_LOWER)) {
    set_error(std::string(who) + ": the lower triangle of a symmetric matrix is required");
    return false;
  }
  return true;
}

Factor* symbolic(taucs_ccs_matrix* A, int max_depth) {
  if (!check_matrix(A, "taucs_ccs_factor_llt_symbolic")) return nullptr;
  double wt = taucs_wtime();
  Factor* F = new (std::nothrow) Factor();
  if (!F) return nullptr;
  F->n = A->n;
  int rc = symbolic_analyze(A->n, A->colptr, A->rowind, max_depth, &F->sym);
  if (rc != TAUCS_SUCCESS) { delete F; return nullptr; }
  rc = build_plan(F->sym, A->n, A->colptr, A->rowind, &F->plan);
  if (rc != TAUCS_SUCCESS) { delete F; return nullptr; }
  // GEMM variants measured on earlier factors of similar shape
  tune_apply(&F->plan, 0);
  tune_apply(&F->plan, 1);
  F->colptr.assign(A->colptr, A->colptr + A->n + 1);
  F->rowind.assign(A->rowind, A->rowind + A->colptr[A->n]);
  tprintf("\t\tSymbolic Analysis            = % 10.3f seconds\n", taucs_wtime() - wt);
  tprintf("\t\tRelaxed  Analysis of LL^T: %.2e flops, %d supernodes, %d levels\n", F->plan.flops,
          F->plan.n_fronts, F->plan.n_levels);
  return F;
}

int numeric_fp64_device(Factor* F, const double* d_vals, bool wait) {
  if (ensure_device(F)) return -1;
  cudaStream_t st = current_stream();
  const Plan& P = F->plan;
  if (!F->dL && !cuda_ok(tb::dmalloc(&F->dL, sizeof(double) * (size_t) P.l_len), "cudaMalloc(L)")) return -1;
  if (!F->dU && !cuda_ok(tb::dmalloc(&F->dU, sizeof(double) * (size_t) P.u_len), "cudaMalloc(U)")) {
    free_numeric(F);
    return -1;
  }
  if (!F->dDinv && !cuda_ok(tb::dmalloc(&F->dDinv, sizeof(double) * (size_t) P.dinv_len), "cudaMalloc(Dinv)")) {
    free_numeric(F);
    return -1;
  }
  F->dvals_cur = d_vals;
  int e = run_graphed(F, GraphKey{1, (uint64_t) d_vals, 0, 0, 0, 0}, st, [&](cudaStream_t s) {
    return launch_numeric_fp64(P, F->dp, d_vals, F->dL, F->dU, F->dDinv, F->dstatus, s);
  });
  if (!cuda_ok((cudaError_t) e, "numeric launch")) return -1;
  if (!cuda_ok(cudaMemcpyAsync(F->hstatus, F->dstatus, sizeof(int), cudaMemcpyDeviceToHost, st), "status")) return -1;
  F->has_numeric = true;
  if (!wait) return 0;
  if (!cuda_ok(cudaStreamSynchronize(st), "numeric factorization")) return -1;
  if (numeric_status_check(*F->hstatus, "LL^T Factorization") != 0) {
    free_numeric(F);
    return -1;
  }
  return 0;
}

int numeric_status_check(int word, const char* what) {
  if (word == INT_MAX) return 0;
  if (word == NUMERIC_TIMEOUT) {
    set_error(std::string(what) + ": a bounded wait between thread blocks timed out; the factor is not valid");
    tprintf("\t\t%s: a bounded device wait timed out\n", what);
    return -1;
  }
  set_error(std::string(what) + ": matrix is not positive definite (nonpositive pivot in column " +
            std::to_string(word) + ")");
  tprintf("\t\t%s: Matrix is not positive definite.\n", what);
  tprintf("\t\t                    nonpositive pivot in column %d\n", word);
  return 1;
}


int numeric_device(Factor* F, const double* d_vals, bool wait) {
  if (F->precision == 1) {
    // FP32 fronts; only a nonpositive FP32 pivot falls back to the FP64
    // factor (a timed-out wait or a CUDA error is reported as it is)
    invalidate_numeric(F);
    const int r = numeric_fp32_device(F, d_vals);
    if (r <= 0) return r;
    tprintf("\t\tFP32 factorization failed; refactoring in FP64\n");
    return numeric_fp64_device(F, d_vals, true);
  }
  return numeric_fp64_device(F, d_vals, wait);
}

int numeric_host(Factor* F, taucs_ccs_matrix* A) {
  if (!check_matrix(A, "taucs_ccs_factor_llt_numeric")) return -1;
  if (!pattern_matches(F, A)) {
    set_error("taucs_ccs_factor_llt_numeric: the matrix pattern differs from the analysed one");
    return -1;
  }
  if (ensure_device(F)) return -1;
  cudaStream_t st = current_stream();
  double wt = taucs_wtime();
  if (!cuda_ok(cudaMemcpyAsync(F->dA, A->values.d, sizeof(double) * (size_t) F->plan.nnz,
                               cudaMemcpyHostToDevice, st), "values upload")) return -1;
  int rc = numeric_device(F, F->dA, true);
  tprintf("\t\tSupernodal Multifrontal LL^T = % 10.3f seconds\n", taucs_wtime() - wt);
  return rc;
}

int solve_device(Factor* F, int nrhs, double* dX, const double* dB, int ld) {
  if (!F->has_numeric) { set_error("solve: the factor has no numeric part"); return -1; }
  cudaStream_t st = current_stream();
  if (!cuda_ok(cudaMemsetAsync(F->dstatus + 1, 0, sizeof(int), st), "solve status")) return -1;
  int e = run_graphed(F, GraphKey{3, (uint64_t) nrhs, (uint64_t) dX, (uint64_t) dB, (uint64_t) ld, 0}, st,
                      [&](cudaStream_t s) {
                        return launch_solve_fp64(F->plan, F->dp, F->dL, F->dDinv, nrhs, dX, dB, ld, F->dW, F->dpart,
                                                 F->dflags, &F->epoch, F->dstatus + 1, s);
                      });
  return cuda_ok((cudaError_t) e, "solve launch") ? 0 : -1;
}

// reads the solve status word after the stream has drained
static int solve_status(Factor* F, cudaStream_t st) {
  if (!cuda_ok(cudaMemcpyAsync(F->hstatus + 1, F->dstatus + 1, sizeof(int), cudaMemcpyDeviceToHost, st), "status"))
    return -1;
  if (!cuda_ok(cudaStreamSynchronize(st), "solve")) return -1;
  if (F->hstatus[1] != 0) {
    set_error("solve: a bounded wait between thread blocks timed out");
    return -1;
  }
  return 0;
}

int solve_refine_host(Factor* F, taucs_ccs_matrix* A, int nrhs, double* X, const double* B, double tol, int maxits,
                      double* res);

int solve_host(Factor* F, int nrhs, double* X, const double* B) {
  if (F && !F->has_numeric && F->has_numeric32)   // FP32 factor: refined to a 1e-12 scaled residual
    return solve_refine_host(F, nullptr, nrhs, X, B, 1e-12, 10, nullptr) < 0 ? -1 : 0;
  if (!F || !F->has_numeric) { set_error("solve: the factor has no numeric part"); return -1; }
  cudaStream_t st = current_stream();
  const int n = F->n;
  for (int q0 = 0; q0 < nrhs; q0 += SOLVE_NRHS) {
    const int nq = std::min(SOLVE_NRHS, nrhs - q0);
    if (!cuda_ok(cudaMemcpyAsync(F->dX, B + (size_t) q0 * n, sizeof(double) * (size_t) n * nq,
                                 cudaMemcpyHostToDevice, st), "rhs upload")) return -1;
    if (solve_device(F, nq, F->dX, F->dX, n)) return -1;
    if (!cuda_ok(cudaMemcpyAsync(X + (size_t) q0 * n, F->dX, sizeof(double) * (size_t) n * nq,
                                 cudaMemcpyDeviceToHost, st), "solution download")) return -1;
  }
  return solve_status(F, st);
}

// Panel offsets in the reference's slot layout: s x f doubles per slot.
static long ref_panel_offsets(const Symbolic& S, long* vptr) {
  long tot = 0;
  for (int sn = 0; sn < S.n_sn; sn++) { vptr[sn] = tot; tot += (long) S.sn_size[sn] * S.sn_up_size[sn]; }
  vptr[S.n_sn] = tot;
  return tot;
}

// L panels in the reference's row order (f x s per slot, ld f) written into
// out (ref_panel_offsets layout).  The FP64 factor when there is one, else the
// FP32 factor (of the scaled matrix D A D) widened to double.  The device
// arena is copied one level at a time, so the host holds out plus one
// level's panels.
static int download_ref_panels_into(Factor* F, const long* vptr, double* out) {
  const bool f64 = F->has_numeric;
  if (!f64 && !F->has_numeric32) return -1;
  const Plan& P = F->plan;
  const Symbolic& S = F->sym;
  cudaStream_t st = current_stream();
  std::vector<double> hL;
  std::vector<float> hL32;
  std::vector<int> local;
  for (const LevelPlan& LP : P.levels) {
    if (LP.front_begin >= LP.front_end) continue;
    // a level's panels are contiguous in the L arena
    int64_t lo = INT64_MAX, hi = 0;
    for (int i = LP.front_begin; i < LP.front_end; i++) {
      const FrontDesc& Fd = P.fronts[i];
      lo = std::min(lo, Fd.l_off);
      hi = std::max(hi, Fd.l_off + (int64_t) Fd.f * Fd.s);
    }
    const size_t cnt = (size_t) (hi - lo);
    bool ok;
    if (f64) {
      hL.resize(cnt);
      ok = cuda_ok(cudaMemcpyAsync(hL.data(), F->dL + lo, sizeof(double) * cnt, cudaMemcpyDeviceToHost, st), "L download");
    } else {
      hL32.resize(cnt);
      ok = cuda_ok(cudaMemcpyAsync(hL32.data(), F->dL32 + lo, sizeof(float) * cnt, cudaMemcpyDeviceToHost, st), "L download");
    }
    if (!ok || !cuda_ok(cudaStreamSynchronize(st), "L download")) return -1;
    for (int i = LP.front_begin; i < LP.front_end; i++) {
      const FrontDesc& Fd = P.fronts[i];
      const int sn = Fd.sn, s = Fd.s, f = Fd.f;
      const std::vector<int>& st_ = S.sn_struct[sn];
      const int* rw = P.rows.data() + Fd.rows_off;
      local.resize(f);
      for (int k = 0; k < f; k++) local[k] = (int) (std::lower_bound(rw, rw + f, st_[k]) - rw);
      const size_t base = (size_t) (Fd.l_off - lo);
      double* o = out + vptr[sn];
      for (int jp = 0; jp < s; jp++) {
        const int lj = local[jp];
        for (int ip = 0; ip < jp; ip++) o[(size_t) jp * f + ip] = 0.0;
        for (int ip = jp; ip < f; ip++) {
          const int li = local[ip];
          const size_t at = base + li + (size_t) lj * f;
          o[(size_t) jp * f + ip] = (li >= lj) ? (f64 ? hL[at] : (double) hL32[at]) : 0.0;
        }
      }
    }
  }
  return 0;
}

static int download_ref_panels(Factor* F, std::vector<long>& vptr, std::vector<double>& vals) {
  if (!F->has_numeric) return -1;
  vptr.assign(F->sym.n_sn + 1, 0);
  const long tot = ref_panel_offsets(F->sym, vptr.data());
  vals.assign(std::max(tot, 1L), 0.0);
  return download_ref_panels_into(F, vptr.data(), vals.data());
}

static int order_identity(int n, int* p, int* ip) {
  for (int i = 0; i < n; i++) p[i] = ip[i] = i;
  return 0;
}

}  // namespace tb

using namespace tb;

extern "C" {

int taucs_b200_set_stream(void* s) {
  g_stream = (cudaStream_t) s;
  return 0;
}

// Autotuner: for the factor's precision, runs the numeric factorization
// once with every GEMM launch in each variant (after an untimed run), times
// every launch with CUDA events, and keeps per level and product the variant
// that took less device time.  The choice lives in the plan and applies to
// every later numeric factorization of this handle.
int taucs_b200_autotune(void* L, const double* d_values, int* choices) {
  Factor* F = (Factor*) L;
  if (!F || !d_values) return -1;
  if (ensure_device(F)) return -1;
  const int H = F->plan.n_levels, pi = F->precision == 1 ? 1 : 0;
  std::vector<double> t[2];
  for (int v = 0; v < 2; v++) {
    t[v].assign(2 * H, 0.0);
    F->plan.gemm_choice[pi].assign(2 * H, (uint8_t) v);
    drop_graphs(F);
    for (int rep = 0; rep < 2; rep++) {
      taucs_b200_profile(1);
      const int rc = numeric_device(F, d_values, true);
      std::vector<ProfEntry> log = prof_take_log();
      taucs_b200_profile(0);
      if (rc) {
        F->plan.gemm_choice[pi].clear();
        return -1;
      }
      if (rep == 0) continue;
      for (const ProfEntry& e : log) {
        if (e.tag < 0 || e.tag >= H) continue;
        if (e.kc == KC_GEMM_PANEL) t[v][2 * e.tag] += e.ms;
        if (e.kc == KC_GEMM_U) t[v][2 * e.tag + 1] += e.ms;
      }
    }
  }
  tune_record(F->plan, pi, t);
  std::vector<uint8_t>& c = F->plan.gemm_choice[pi];
  double before = 0.0, after = 0.0;
  for (int i = 0; i < 2 * H; i++) {
    c[i] = t[1][i] < t[0][i] ? 1 : 0;
    before += t[0][i];
    after += t[c[i]][i];
    if (choices) choices[i] = c[i];
  }
  drop_graphs(F);
  tprintf("\t\tautotune (%s fronts): GEMM time %.2f ms with the default variants, %.2f ms with the chosen ones\n",
          pi ? "FP32" : "FP64", before, after);
  return 0;
}

int taucs_b200_get_gemm_choices(void* L, int precision, int* choices) {
  Factor* F = (Factor*) L;
  if (!F || (precision != 0 && precision != 1) || !choices) return -1;
  const std::vector<uint8_t>& c = F->plan.gemm_choice[precision];
  for (int i = 0; i < 2 * F->plan.n_levels; i++) choices[i] = (size_t) i < c.size() ? c[i] : 0;
  return 0;
}

int taucs_b200_set_gemm_choices(void* L, int precision, int count, const int* choices) {
  Factor* F = (Factor*) L;
  if (!F || (precision != 0 && precision != 1) || count < 0 || (count > 0 && !choices)) return -1;
  const int H = F->plan.n_levels;
  if (count != 0 && count != 2 * H) {
    set_error("taucs_b200_set_gemm_choices: expected 2 x levels (" + std::to_string(2 * H) + ") choices");
    return -1;
  }
  std::vector<uint8_t>& c = F->plan.gemm_choice[precision];
  c.assign((size_t) count, 0);
  for (int i = 0; i < count; i++) {
    if (choices[i] != 0 && choices[i] != 1) {
      c.clear();
      set_error("taucs_b200_set_gemm_choices: a choice is neither 0 nor 1");
      return -1;
    }
    c[i] = (uint8_t) choices[i];
  }
  drop_graphs(F);
  return 0;
}

int taucs_b200_debug_waits(int limit, int skew) {
  if (limit < 0) return -1;
  return cuda_ok((cudaError_t) solve_set_wait_controls(limit, skew), "taucs_b200_debug_waits") ? 0 : -1;
}

long taucs_b200_launch_count(int reset) {
  return reset ? g_launches.exchange(0) : g_launches.load();
}

void* taucs_dccs_factor_llt_symbolic_maxdepth(taucs_ccs_matrix* A, int max_depth) {
  return symbolic(A, max_depth);
}
void* taucs_dccs_factor_llt_symbolic(taucs_ccs_matrix* A) { return symbolic(A, 0); }
void* taucs_ccs_factor_llt_symbolic_maxdepth(taucs_ccs_matrix* A, int max_depth) { return symbolic(A, max_depth); }
void* taucs_ccs_factor_llt_symbolic(taucs_ccs_matrix* A) { return symbolic(A, 0); }

int taucs_dccs_factor_llt_numeric(taucs_ccs_matrix* A, void* L) {
  if (!L) return -1;
  return numeric_host((Factor*) L, A);
}
int taucs_ccs_factor_llt_numeric(taucs_ccs_matrix* A, void* L) { return taucs_dccs_factor_llt_numeric(A, L); }

void* taucs_dccs_factor_llt_mf_maxdepth(taucs_ccs_matrix* A, int max_depth) {
  Factor* F = symbolic(A, max_depth);
  if (!F) return nullptr;
  if (numeric_host(F, A)) {
    free_device(F);
    delete F;
    return nullptr;
  }
  return F;
}
void* taucs_dccs_factor_llt_mf(taucs_ccs_matrix* A) { return taucs_dccs_factor_llt_mf_maxdepth(A, 0); }
void* taucs_ccs_factor_llt_mf_maxdepth(taucs_ccs_matrix* A, int max_depth) { return taucs_dccs_factor_llt_mf_maxdepth(A, max_depth); }
void* taucs_ccs_factor_llt_mf(taucs_ccs_matrix* A) { return taucs_dccs_factor_llt_mf_maxdepth(A, 0); }

int taucs_dsupernodal_solve_llt(void* L, void* x, void* b) {
  if (!L || !x || !b) return -1;
  return solve_host((Factor*) L, 1, (double*) x, (const double*) b);
}
int taucs_supernodal_solve_llt(void* L, void* x, void* b) { return taucs_dsupernodal_solve_llt(L, x, b); }

int taucs_b200_solve_many(void* L, int nrhs, double* X, const double* B) {
  if (!L || nrhs < 0) return -1;
  if (nrhs == 0) return 0;
  return solve_host((Factor*) L, nrhs, X, B);
}

int taucs_b200_factor_numeric_device(void* L, const double* d_values) {
  if (!L) return -1;
  return numeric_device((Factor*) L, d_values, true);
}

int taucs_b200_factor_numeric_device_async(void* L, const double* d_values) {
  if (!L) return -1;
  return numeric_device((Factor*) L, d_values, false);
}

int taucs_b200_factor_status(void* vL) {
  Factor* F = (Factor*) vL;
  if (!F || (!F->has_numeric && !F->has_numeric32)) return -1;
  if (!F->has_numeric) return 0;
  if (!cuda_ok(cudaStreamSynchronize(current_stream()), "status")) return -1;
  if (numeric_status_check(*F->hstatus, "LL^T Factorization") != 0) { free_numeric(F); return -1; }
  return 0;
}

int taucs_b200_solve_device(void* L, int nrhs, double* d_X, const double* d_B, int ld) {
  if (!L || nrhs < 0 || ld < ((Factor*) L)->n) return -1;
  if (nrhs == 0) return 0;
  return solve_device((Factor*) L, nrhs, d_X, d_B, ld);
}

void taucs_dsupernodal_factor_free(void* L) {
  Factor* F = (Factor*) L;
  if (!F) return;
  free_device(F);
  delete F;
}
void taucs_supernodal_factor_free(void* L) { taucs_dsupernodal_factor_free(L); }

void taucs_dsupernodal_factor_free_numeric(void* L) {
  if (L) free_numeric((Factor*) L);
}
void taucs_supernodal_factor_free_numeric(void* L) { taucs_dsupernodal_factor_free_numeric(L); }

taucs_ccs_matrix* taucs_dsupernodal_factor_to_ccs(void* vL) {
  Factor* F = (Factor*) vL;
  if (!F) return nullptr;
  std::vector<long> vp;
  std::vector<double> v;
  if (download_ref_panels(F, vp, v)) return nullptr;
  const Symbolic& S = F->sym;
  const int n = F->n;
  // same traversal and zero dropping as src/taucs_sn_llt.c:851-978
  std::vector<int> len(n, 0);
  long nnz = 0;
  for (int sn = 0; sn < S.n_sn; sn++) {
    const int s = S.sn_size[sn], f = S.sn_up_size[sn];
    const double* pan = v.data() + vp[sn];
    for (int jp = 0; jp < s; jp++) {
      int j = S.sn_struct[sn][jp];
      for (int ip = jp; ip < f; ip++)
        if (pan[(size_t) jp * f + ip] != 0.0) { len[j]++; nnz++; }
    }
  }
  taucs_ccs_matrix* C = taucs_ccs_create(n, n, (int) nnz, TAUCS_DOUBLE | TAUCS_TRIANGULAR | TAUCS_LOWER);
  if (!C) return nullptr;
  C->colptr[0] = 0;
  for (int j = 0; j < n; j++) C->colptr[j + 1] = C->colptr[j] + len[j];
  for (int sn = 0; sn < S.n_sn; sn++) {
    const int s = S.sn_size[sn], f = S.sn_up_size[sn];
    const double* pan = v.data() + vp[sn];
    for (int jp = 0; jp < s; jp++) {
      int j = S.sn_struct[sn][jp];
      int next = C->colptr[j];
      for (int ip = jp; ip < f; ip++) {
        const double x = pan[(size_t) jp * f + ip];
        if (x == 0.0) continue;
        C->rowind[next] = S.sn_struct[sn][ip];
        C->values.d[next] = x;
        next++;
      }
    }
  }
  return C;
}
taucs_ccs_matrix* taucs_supernodal_factor_to_ccs(void* L) { return taucs_dsupernodal_factor_to_ccs(L); }

double* taucs_dsupernodal_factor_get_diag(void* vL) {
  Factor* F = (Factor*) vL;
  if (!F || !F->has_numeric) return nullptr;
  const Plan& P = F->plan;
  double* diag = (double*) malloc(sizeof(double) * (size_t) std::max(F->n, 1));
  if (!diag) return nullptr;
  cudaStream_t st = current_stream();
  // one strided copy per front: the diagonal of the panel has stride f+1
  for (const FrontDesc& Fd : P.fronts) {
    const int* rw = P.rows.data() + Fd.rows_off;
    std::vector<double> d(Fd.s);
    if (!cuda_ok(cudaMemcpy2DAsync(d.data(), sizeof(double), F->dL + Fd.l_off, sizeof(double) * (Fd.f + 1),
                                   sizeof(double), Fd.s, cudaMemcpyDeviceToHost, st), "diag")) {
      free(diag);
      return nullptr;
    }
    cudaStreamSynchronize(st);
    for (int c = 0; c < Fd.s; c++) diag[rw[c]] = d[c];
  }
  return diag;
}
void* taucs_supernodal_factor_get_diag(void* L) { return taucs_dsupernodal_factor_get_diag(L); }

int taucs_b200_factor_info(void* vL, taucs_b200_info* info) {
  Factor* F = (Factor*) vL;
  if (!F || !info) return -1;
  const Plan& P = F->plan;
  const Symbolic& S = F->sym;
  info->n = F->n;
  info->n_sn = S.n_sn;
  info->n_live = P.n_fronts;
  info->n_levels = P.n_levels;
  long sl = 0, lv = 0;
  for (int sn = 0; sn < S.n_sn; sn++) { sl += S.sn_up_size[sn]; lv += (long) S.sn_size[sn] * S.sn_up_size[sn]; }
  info->struct_len = sl;
  info->l_values = lv;
  info->flops = P.flops;
  info->l_bytes = 8.0 * (double) P.l_len;
  info->u_bytes = 8.0 * (double) P.u_len;
  info->ea_bytes = P.ea_bytes;
  info->solve_bytes = P.solve_bytes;
  info->max_front = P.max_front;
  info->max_sn_size = P.max_s;
  return 0;
}

int taucs_b200_export_symbolic(void* vL, int* sn_size, int* sn_up_size, int* first_child, int* next_child,
                               long* struct_ptr, int* struct_idx) {
  Factor* F = (Factor*) vL;
  if (!F) return -1;
  const Symbolic& S = F->sym;
  long p = 0;
  for (int sn = 0; sn < S.n_sn; sn++) {
    sn_size[sn] = S.sn_size[sn];
    sn_up_size[sn] = S.sn_up_size[sn];
  }
  for (int sn = 0; sn <= S.n_sn; sn++) {
    first_child[sn] = S.first_child[sn];
    next_child[sn] = S.next_child[sn];
  }
  for (int sn = 0; sn < S.n_sn; sn++) {
    struct_ptr[sn] = p;
    for (int k = 0; k < S.sn_up_size[sn]; k++) struct_idx[p + k] = S.sn_struct[sn][k];
    p += S.sn_up_size[sn];
  }
  struct_ptr[S.n_sn] = p;
  return 0;
}

int taucs_b200_export_layout(void* vL, long long* fronts, long long* totals) {
  const Factor* F = (const Factor*) vL;
  if (!F) return -1;
  const Plan& P = F->plan;
  if (fronts)
    for (int i = 0; i < P.n_fronts; i++) {
      const FrontDesc& D = P.fronts[i];
      long long* o = fronts + (size_t) i * 14;
      o[0] = D.level; o[1] = D.parent; o[2] = D.s; o[3] = D.f;
      o[4] = D.l_off; o[5] = D.u_off; o[6] = D.v_off; o[7] = D.dinv_off;
      o[8] = D.blk_off; o[9] = D.part_off; o[10] = D.nchunk; o[11] = D.sn;
      o[12] = D.rows_off; o[13] = D.map_off;
    }
  if (totals) {
    totals[0] = P.l_len; totals[1] = P.u_len; totals[2] = P.v_len;
    totals[3] = P.dinv_len; totals[4] = P.part_len; totals[5] = P.n_blk;
    totals[6] = (long long) P.rows.size(); totals[7] = (long long) P.maps.size();
  }
  return 0;
}

int taucs_b200_export_rows_maps(void* vL, int* rows, int* maps) {
  const Factor* F = (const Factor*) vL;
  if (!F) return -1;
  if (rows) std::copy(F->plan.rows.begin(), F->plan.rows.end(), rows);
  if (maps) std::copy(F->plan.maps.begin(), F->plan.maps.end(), maps);
  return 0;
}

int taucs_b200_export_solve_blocks(void* vL, int h, int* fwd, int* n_fwd, int* n_diag, int* bwd, int* n_bwd) {
  const Factor* F = (const Factor*) vL;
  if (!F || h < 0 || h >= F->plan.n_levels) return -1;
  const LevelPlan& LP = F->plan.levels[h];
  if (n_fwd) *n_fwd = (int) LP.solve_fwd_blocks.size();
  if (n_diag) *n_diag = LP.n_fwd_diag;
  if (n_bwd) *n_bwd = (int) LP.solve_bwd_blocks.size();
  for (size_t i = 0; fwd && i < LP.solve_fwd_blocks.size(); i++) {
    fwd[2 * i] = LP.solve_fwd_blocks[i].a;
    fwd[2 * i + 1] = LP.solve_fwd_blocks[i].b;
  }
  for (size_t i = 0; bwd && i < LP.solve_bwd_blocks.size(); i++) {
    bwd[2 * i] = LP.solve_bwd_blocks[i].a;
    bwd[2 * i + 1] = LP.solve_bwd_blocks[i].b;
  }
  return 0;
}

int taucs_b200_export_persistent(void* vL, int* tasks, int* parent_task, int* pending) {
  const Factor* F = (const Factor*) vL;
  if (!F) return -1;
  const Plan& P = F->plan;
  const int n = (int) P.pers_fronts.size();
  for (int t = 0; t < n; t++) {
    if (tasks) tasks[t] = P.pers_fronts[t];
    if (parent_task) parent_task[t] = P.pers_parent[t];
    if (pending) pending[t] = P.pers_pending[t];
  }
  return n;
}

int taucs_b200_export_values(void* vL, long* val_ptr, double* vals) {
  Factor* F = (Factor*) vL;
  if (!F) return -1;
  if (!F->has_numeric && !F->has_numeric32) {
    set_error("taucs_b200_export_values: the factor has no numeric part");
    return -1;
  }
  ref_panel_offsets(F->sym, val_ptr);
  return download_ref_panels_into(F, val_ptr, vals);
}

int taucs_b200_etree(taucs_ccs_matrix* A, int* parent) {
  if (!A || !parent) return -1;
  return etree(A->n, A->colptr, A->rowind, parent);
}

void taucs_ccs_order(taucs_ccs_matrix* A, int** perm, int** invperm, char* which) {
  *perm = *invperm = nullptr;
  if (!A || !which) return;
  const int n = A->n;
  int* p = (int*) malloc(sizeof(int) * (size_t) std::max(n, 1));
  int* ip = (int*) malloc(sizeof(int) * (size_t) std::max(n, 1));
  if (!p || !ip) { free(p); free(ip); return; }
  int rc = -1;
  if (!strcmp(which, "identity")) {
    rc = order_identity(n, p, ip);
  } else if (!strcmp(which, "random")) {
    std::mt19937 gen(12345u);
    for (int i = 0; i < n; i++) p[i] = i;
    std::shuffle(p, p + n, gen);
    for (int i = 0; i < n; i++) ip[p[i]] = i;
    rc = 0;
  } else if (!strcmp(which, "amd")) {
    if (!(A->flags & (TAUCS_SYMMETRIC | TAUCS_HERMITIAN)) || !(A->flags & TAUCS_LOWER)) {
      tprintf("taucs_ccs_amd: the lower part of a symmetric matrix must be represented.\n");
    } else {
      rc = amd_order(n, A->colptr, A->rowind, p, ip);
    }
  } else if (!strcmp(which, "genmmd")) {
    // src/taucs_ccs_order.c:262-442
    if (!(A->flags & (TAUCS_SYMMETRIC | TAUCS_HERMITIAN))) {
      tprintf("taucs_ccs_genmmd: GENMMD ordering only works on symmetric matrices.\n");
    } else if (!(A->flags & TAUCS_LOWER)) {
      tprintf("taucs_ccs_genmmd: the lower part of the matrix must be represented.\n");
    } else {
      rc = mmd_order(n, A->colptr, A->rowind, p, ip);
    }
  } else {
    tprintf("taucs_ccs_order: ordering %s is not available in this build\n", which);
  }
  if (rc) { free(p); free(ip); return; }
  *perm = p;
  *invperm = ip;
}

}  // extern "C"

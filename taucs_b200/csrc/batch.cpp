// Batches: many independent SPD systems factored and solved as one.
//
// The reference factors one system per call (taucs_ccs_factor_llt_mf,
// src/taucs_sn_llt.c:2894-3006); thousands of small systems would each pay
// for a full traversal of their own tree of fronts.  Here the systems, each
// in its own AMD ordering, are laid side by side as the diagonal blocks of
// one matrix.  Each system is analysed on its own and the systems'
// supernodal trees are joined under one virtual root, so every system keeps
// exactly the supernodes of its own analysis (the reference's symbolic
// phase applied to the block-diagonal matrix as a whole amalgamates less: on
// a forest it leaves many more, smaller supernodes).  The level plan then
// puts the fronts of all systems of the same height into the same launches:
// one level-scheduled launch sequence (recorded once as a CUDA graph)
// factors every system of the batch, and one solves them all.  The
// systems' rows form the factor's segments, so refinement measures and
// meets the scaled-residual target of every system on its own.

#include <algorithm>
#include <atomic>
#include <string>
#include <thread>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "factor.h"

namespace tb {

int numeric_device(Factor* F, const double* d_vals, bool wait);
int solve_refine_device(Factor* F, int nrhs, double* dX, const double* dB, int ld, double tol, int maxits,
                        double* res);

}  // namespace tb

using namespace tb;

extern "C" void* taucs_b200_batch_analyze(int count, taucs_ccs_matrix* const* A) {
  if (count < 1 || !A) { set_error("batch_analyze: no systems"); return nullptr; }
  int64_t N = 0, NNZ = 0;
  for (int s = 0; s < count; s++) {
    if (!A[s] || !(A[s]->flags & TAUCS_DOUBLE) || !(A[s]->flags & TAUCS_LOWER) || A[s]->n < 1) {
      set_error("batch_analyze: system " + std::to_string(s) + " is not a lower-triangle double matrix");
      return nullptr;
    }
    N += A[s]->n;
    NNZ += A[s]->colptr[A[s]->n];
  }
  if (N > INT_MAX || NNZ > INT_MAX) { set_error("batch_analyze: the batch exceeds 2^31 rows or entries"); return nullptr; }
  std::vector<int> colptr(N + 1), rowind(NNZ), seg_ptr(count + 1, 0), perm(N), vmap(NNZ);
  std::vector<int64_t> nnz_off(count + 1, 0);
  for (int s = 0; s < count; s++) {
    seg_ptr[s + 1] = seg_ptr[s] + A[s]->n;
    nnz_off[s + 1] = nnz_off[s] + A[s]->colptr[A[s]->n];
  }
  colptr[0] = 0;
  // per system, independent of the others (host threads): AMD ordering, the
  // permuted pattern with the value map, the symbolic factor
  std::vector<Symbolic> syms(count);
  std::vector<std::string> errs(count);
  auto analyse = [&](int s) {
    taucs_ccs_matrix As = *A[s];
    const int n = As.n;
    const int64_t nnz = As.colptr[n];
    const int64_t r0 = seg_ptr[s], e0 = nnz_off[s];
    int *p = nullptr, *ip = nullptr;
    taucs_ccs_order(&As, &p, &ip, (char*) "amd");
    if (!p) { errs[s] = "ordering failed"; return; }
    // value positions travel through the permutation as values
    std::vector<double> idx((size_t) nnz);
    for (int64_t k = 0; k < nnz; k++) idx[k] = (double) k;
    As.values.d = idx.data();
    taucs_ccs_matrix* PA = taucs_ccs_permute_symmetrically(&As, p, ip);
    if (!PA) { free(p); free(ip); errs[s] = "permutation failed"; return; }
    if (symbolic_analyze(n, PA->colptr, PA->rowind, 0, &syms[s]) != TAUCS_SUCCESS) errs[s] = "symbolic analysis failed";
    for (int j = 0; j < n; j++) {
      for (int k = PA->colptr[j]; k < PA->colptr[j + 1]; k++) {
        rowind[e0 + k] = (int) r0 + PA->rowind[k];
        vmap[e0 + k] = (int) PA->values.d[k];
      }
      colptr[r0 + j + 1] = (int) (e0 + PA->colptr[j + 1]);
      perm[r0 + j] = p[j];
    }
    taucs_ccs_free(PA);
    free(p);
    free(ip);
  };
  {
    const int nth = std::max(1, std::min<int>(count, (int) std::thread::hardware_concurrency()));
    std::atomic<int> next(0);
    std::vector<std::thread> pool;
    for (int t = 0; t < nth; t++)
      pool.emplace_back([&] {
        for (int s; (s = next.fetch_add(1)) < count;) analyse(s);
      });
    for (auto& th : pool) th.join();
  }
  for (int s = 0; s < count; s++)
    if (!errs[s].empty()) {
      set_error("batch_analyze: system " + std::to_string(s) + ": " + errs[s]);
      return nullptr;
    }
  // the systems' supernodal trees under one virtual root: slots of system s
  // follow those of systems < s, rows are shifted by the system's offset,
  // and the roots of every tree become children of the joint root
  Factor* F = new (std::nothrow) Factor();
  if (!F) return nullptr;
  Symbolic& J = F->sym;
  J.n = (int) N;
  int nsn = 0;
  for (const Symbolic& S : syms) nsn += S.n_sn;
  J.n_sn = nsn;
  J.sn_size.reserve(nsn);
  J.sn_up_size.reserve(nsn);
  J.sn_struct.reserve(nsn);
  J.first_child.assign(nsn + 1, -1);
  J.next_child.assign(nsn + 1, -1);
  int o = 0, ro = 0, last_root = -1;
  for (int s = 0; s < count; s++) {
    Symbolic& S = syms[s];
    for (int k = 0; k < S.n_sn; k++) {
      J.sn_size.push_back(S.sn_size[k]);
      J.sn_up_size.push_back(S.sn_up_size[k]);
      std::vector<int> st = std::move(S.sn_struct[k]);
      for (int& r : st) r += ro;
      J.sn_struct.push_back(std::move(st));
      J.first_child[o + k] = S.first_child[k] < 0 ? -1 : o + S.first_child[k];
      J.next_child[o + k] = S.next_child[k] < 0 ? -1 : o + S.next_child[k];
    }
    // the tree's root children, linked after the previous tree's
    for (int c = S.first_child[S.n_sn]; c >= 0; c = S.next_child[c]) {
      const int g = o + c;
      if (last_root < 0) J.first_child[nsn] = g;
      else J.next_child[last_root] = g;
      J.next_child[g] = -1;
      last_root = g;
    }
    o += S.n_sn;
    ro += S.n;
    Symbolic().sn_struct.swap(S.sn_struct);
  }
  F->n = (int) N;
  if (build_plan(J, F->n, colptr.data(), rowind.data(), &F->plan) != TAUCS_SUCCESS) {
    delete F;
    set_error("batch_analyze: plan construction failed");
    return nullptr;
  }
  tune_apply(&F->plan, 0);
  tune_apply(&F->plan, 1);
  F->colptr = std::move(colptr);
  F->rowind = std::move(rowind);
  F->seg_ptr = std::move(seg_ptr);
  F->batch.nnz_off = std::move(nnz_off);
  F->batch.perm = std::move(perm);
  F->batch.vmap = std::move(vmap);
  return F;
}

static bool is_batch(const Factor* F) { return F && !F->batch.nnz_off.empty(); }

extern "C" int taucs_b200_batch_values(void* L, taucs_ccs_matrix* const* A, double* combined) {
  Factor* F = (Factor*) L;
  if (!is_batch(F) || !A || !combined) { set_error("batch_values: not a batch handle"); return -1; }
  const int count = F->nseg();
  for (int s = 0; s < count; s++) {
    const int64_t k0 = F->batch.nnz_off[s], k1 = F->batch.nnz_off[s + 1];
    if (!A[s] || A[s]->colptr[A[s]->n] != k1 - k0) {
      set_error("batch_values: system " + std::to_string(s) + " does not match the analysed pattern");
      return -1;
    }
    const double* v = A[s]->values.d;
    for (int64_t k = k0; k < k1; k++) combined[k] = v[F->batch.vmap[k]];
  }
  return 0;
}

extern "C" int taucs_b200_batch_rhs(void* L, const double* const* B, double* combined) {
  Factor* F = (Factor*) L;
  if (!is_batch(F) || !B || !combined) { set_error("batch_rhs: not a batch handle"); return -1; }
  for (int s = 0; s < F->nseg(); s++) {
    const int r0 = F->seg_ptr[s], r1 = F->seg_ptr[s + 1];
    for (int i = r0; i < r1; i++) combined[i] = B[s][F->batch.perm[i]];
  }
  return 0;
}

extern "C" int taucs_b200_batch_split(void* L, const double* combined, double* const* X) {
  Factor* F = (Factor*) L;
  if (!is_batch(F) || !X || !combined) { set_error("batch_split: not a batch handle"); return -1; }
  for (int s = 0; s < F->nseg(); s++) {
    const int r0 = F->seg_ptr[s], r1 = F->seg_ptr[s + 1];
    for (int i = r0; i < r1; i++) X[s][F->batch.perm[i]] = combined[i];
  }
  return 0;
}

// The device side of the batch entry points, set up on first use: the maps
// from the combined order to the systems' own orders concatenated, the
// device buffers, and the pinned staging area.
static int batch_device(Factor* F) {
  Factor::BatchMap& M = F->batch;
  if (M.h_raw) return 0;
  if (ensure_device(F)) return -1;
  const int64_t nnz = F->plan.nnz;
  const int n = F->n, count = F->nseg();
  std::vector<int> cvmap((size_t) nnz), cperm((size_t) n);
  for (int s = 0; s < count; s++) {
    for (int64_t k = M.nnz_off[s]; k < M.nnz_off[s + 1]; k++) cvmap[k] = (int) (M.nnz_off[s] + M.vmap[k]);
    for (int i = F->seg_ptr[s]; i < F->seg_ptr[s + 1]; i++) cperm[i] = F->seg_ptr[s] + M.perm[i];
  }
  const size_t raw = (size_t) std::max<int64_t>(nnz, n);
  cudaStream_t st = current_stream();
  bool ok = cuda_ok(dmalloc(&M.d_cvmap, sizeof(int) * std::max<int64_t>(nnz, 1)), "cudaMalloc") &&
            cuda_ok(dmalloc(&M.d_cperm, sizeof(int) * std::max(n, 1)), "cudaMalloc") &&
            cuda_ok(dmalloc(&M.d_raw, sizeof(double) * raw), "cudaMalloc") &&
            cuda_ok(dmalloc(&M.d_b, sizeof(double) * std::max(n, 1)), "cudaMalloc") &&
            cuda_ok(dmalloc(&M.d_x, sizeof(double) * std::max(n, 1)), "cudaMalloc") &&
            cuda_ok(hmalloc(&M.h_raw, sizeof(double) * raw), "cudaMallocHost") &&
            cuda_ok(cudaMemcpyAsync(M.d_cvmap, cvmap.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, st), "map") &&
            cuda_ok(cudaMemcpyAsync(M.d_cperm, cperm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st), "map") &&
            cuda_ok(cudaStreamSynchronize(st), "batch maps");
  if (!ok) {
    dfree(M.d_cvmap); dfree(M.d_cperm); dfree(M.d_raw); dfree(M.d_b); dfree(M.d_x); hfree(M.h_raw);
    M.d_cvmap = M.d_cperm = nullptr;
    M.d_raw = M.d_b = M.d_x = M.h_raw = nullptr;
    return -1;
  }
  return 0;
}

// body(s) for every system s, on up to 16 host threads
template <typename Body>
static void for_systems(int count, Body body) {
  const int nt = (int) std::min<unsigned>(16u, std::max(1u, std::thread::hardware_concurrency()));
  if (nt <= 1 || count < 64) {
    for (int s = 0; s < count; s++) body(s);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < nt; t++)
    th.emplace_back([&, t] {
      for (int s = t; s < count; s += nt) body(s);
    });
  for (auto& x : th) x.join();
}


extern "C" int taucs_b200_batch_factor(void* L, taucs_ccs_matrix* const* A) {
  Factor* F = (Factor*) L;
  if (!is_batch(F)) { set_error("batch_factor: not a batch handle"); return -1; }
  if (!A) { set_error("batch_factor: no systems"); return -1; }
  if (batch_device(F)) return -1;
  Factor::BatchMap& M = F->batch;
  const int count = F->nseg();
  for (int s = 0; s < count; s++)
    if (!A[s] || A[s]->colptr[A[s]->n] != M.nnz_off[s + 1] - M.nnz_off[s]) {
      set_error("batch_factor: system " + std::to_string(s) + " does not match the analysed pattern");
      return -1;
    }
  // the values as given, back to back in pinned memory; one copy; the
  // combined order is gathered on the device
  for_systems(count, [&](int s) {
    memcpy(M.h_raw + M.nnz_off[s], A[s]->values.d, sizeof(double) * (size_t) (M.nnz_off[s + 1] - M.nnz_off[s]));
  });
  cudaStream_t st = current_stream();
  const int64_t nnz = F->plan.nnz;
  if (!cuda_ok(cudaMemcpyAsync(M.d_raw, M.h_raw, sizeof(double) * nnz, cudaMemcpyHostToDevice, st), "values") ||
      gather_values_device(nnz, M.d_cvmap, M.d_raw, F->dA))
    return -1;
  return numeric_device(F, F->dA, true);
}

extern "C" int taucs_b200_batch_solve(void* L, double* const* X, const double* const* B, double tol, int maxits,
                                      double* res) {
  Factor* F = (Factor*) L;
  if (!is_batch(F)) { set_error("batch_solve: not a batch handle"); return -1; }
  if (!F->has_numeric && !F->has_numeric32) { set_error("batch_solve: no numeric factor"); return -1; }
  if (!X || !B) { set_error("batch_solve: no vectors"); return -1; }
  if (batch_device(F)) return -1;
  Factor::BatchMap& M = F->batch;
  const int n = F->n, count = F->nseg();
  // right-hand sides as given, back to back; permuted on the device
  for_systems(count, [&](int s) {
    memcpy(M.h_raw + F->seg_ptr[s], B[s], sizeof(double) * (size_t) (F->seg_ptr[s + 1] - F->seg_ptr[s]));
  });
  cudaStream_t st = current_stream();
  if (!cuda_ok(cudaMemcpyAsync(M.d_raw, M.h_raw, sizeof(double) * n, cudaMemcpyHostToDevice, st), "rhs") ||
      perm_gather_device(n, M.d_cperm, M.d_raw, M.d_b))
    return -1;
  int steps = solve_refine_device(F, 1, M.d_x, M.d_b, n, tol, maxits < 0 ? 0 : maxits, res);
  if (steps < 0) return -1;
  if (perm_scatter_device(n, M.d_cperm, M.d_x, M.d_raw) ||
      !cuda_ok(cudaMemcpyAsync(M.h_raw, M.d_raw, sizeof(double) * n, cudaMemcpyDeviceToHost, st), "solution") ||
      !cuda_ok(cudaStreamSynchronize(st), "batch solve"))
    return -1;
  for_systems(count, [&](int s) {
    memcpy(X[s], M.h_raw + F->seg_ptr[s], sizeof(double) * (size_t) (F->seg_ptr[s + 1] - F->seg_ptr[s]));
  });
  return steps;
}

extern "C" int taucs_b200_batch_info(void* L, int* count, int* rows, long* nnz) {
  Factor* F = (Factor*) L;
  if (!is_batch(F)) return -1;
  if (count) *count = F->nseg();
  if (rows) *rows = F->n;
  if (nnz) *nnz = (long) F->plan.nnz;
  return 0;
}

// Request server: factor/solve requests admitted onto the GPU as they arrive.
//
// The reference solves one system per call on the calling thread
// (taucs_linsolve, src/taucs_linsolve.c:433-583: order, factor, solve).  A
// serving process instead receives a stream of independent requests -- new
// matrices, new coefficients on a pattern it has seen, new right-hand sides
// for a matrix it has already factored -- and should keep the GPU busy with
// several of them at once.  This server does that:
//
//  * worker threads, each with its own CUDA streams, take requests from one
//    FIFO queue as soon as they are free, so the numeric factorizations and
//    refinement solves of different requests overlap on the device
//    (continuous admission: a request that arrives while others run starts
//    as soon as a worker and device memory are free); small systems run on
//    high-priority streams so they are not queued behind the thread blocks
//    of large factorizations;
//  * a pattern cache keeps, per sparsity pattern, the AMD ordering, the map
//    from A's values to those of P A P^T, and the symbolic factor and level
//    plan (the reference's taucs_ccs_order + taucs_ccs_permute_symmetrically
//    + taucs_ccs_factor_llt_symbolic), computed once;
//  * factor instances (device buffers of one pattern) are reused; an
//    instance keeps its last numeric factor resident, so a request that
//    brings new right-hand sides for a matrix already factored only solves;
//  * admission by device memory: an instance is created only when its
//    predicted bytes fit the budget next to the instances already held;
//    otherwise idle instances are evicted (least recently used first) or the
//    request waits until running ones finish;
//  * every system is factored with FP32 fronts and refined in FP64 to the
//    request's scaled-residual tolerance (FP64 refactorization when FP32
//    fails or refinement stalls).

#include <algorithm>
#include <chrono>
#include <climits>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "factor.h"

namespace tb {

Factor* symbolic(taucs_ccs_matrix* A, int max_depth);
int numeric_device(Factor* F, const double* d_vals, bool wait);
int gather_values_device(long nnz, const int* d_vmap, const double* d_raw, double* d_out);
int solve_refine_permuted(Factor* F, int nrhs, double* d_x, const double* d_b, const int* d_perm, double tol,
                          int maxits, double* res);

// factor instances kept per pattern while the budget allows (each holds one
// resident numeric factor)
constexpr int MAX_INSTANCES_PER_PATTERN = 8;
// systems below this order run on high-priority streams, so their short
// kernels are scheduled between the thread blocks of large factorizations
constexpr int SMALL_SYSTEM_N = 100000;

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// 64-bit hash of a byte array: four independent multiply-xorshift lanes over
// 32-byte strides (so the multiplies of one lane do not wait for the others),
// folded at the end
inline uint64_t hash_mix(uint64_t h, uint64_t w) {
  h ^= w + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
  return h * 0xff51afd7ed558ccdull;
}

uint64_t hash_bytes(const void* p, size_t bytes, uint64_t h) {
  const unsigned char* c = (const unsigned char*) p;
  uint64_t l0 = h, l1 = h ^ 0x243f6a8885a308d3ull, l2 = h ^ 0x13198a2e03707344ull, l3 = h ^ 0xa4093822299f31d0ull;
  size_t i = 0;
  for (; i + 32 <= bytes; i += 32) {
    uint64_t w[4];
    memcpy(w, c + i, 32);
    l0 = hash_mix(l0, w[0]);
    l1 = hash_mix(l1, w[1]);
    l2 = hash_mix(l2, w[2]);
    l3 = hash_mix(l3, w[3]);
  }
  h = hash_mix(hash_mix(hash_mix(hash_mix(h, l0), l1), l2), l3);
  for (; i < bytes; i++) h = (h ^ c[i]) * 0x100000001b3ull;
  return h ^ (h >> 29);
}

// device bytes of one FP32 factor instance with refinement buffers
size_t predict_bytes(const Plan& P) {
  const double n = P.n, nnz = P.nnz;
  double b = 4.0 * (P.l_len + P.u_len + P.dinv_len + P.part_len)      // FP32 factor, partial sums
             + 4.0 * P.sp_len                                           // split arena
             + 4.0 * (6.0 * P.pers_fronts.size() + 4.0)                 // persistent queues
             + 8.0 * P.part_len                                         // FP64 partial sums
             + 12.0 * P.v_len * SOLVE_NRHS                              // work vectors (FP64 + FP32)
             + 8.0 * nnz * 2 + 4.0 * nnz * 6                            // A (FP64, FP32), pattern, CSR
             + 8.0 * n * SOLVE_NRHS * 4 + 4.0 * n * SOLVE_NRHS + 16.0 * n  // R, Xr, Br, X, V32, scale
             + 4.0 * ((double) P.rows.size() + P.maps.size() + P.acol_ptr.size() + 2.0 * P.a_rows.size())
             + (double) sizeof(FrontDesc) * P.fronts.size() + 4.0 * (solve_flag_words(P) + 1);
  // the build tiles and their child records
  for (const LevelPlan& LP : P.levels)
    for (const Tile& t : LP.build_tiles)
      b += sizeof(Tile) + sizeof(TileChild) * (double) (P.fronts[t.front].child_end - P.fronts[t.front].child_begin);
  return (size_t) (b * 1.05) + (2u << 20);
}

struct Pattern {
  int n = 0;
  int64_t nnz = 0;
  std::vector<int> perm;      // P A P^T row i is A's row perm[i]
  std::vector<int> vmap;      // value k of P A P^T is A's value vmap[k]
  Factor* proto = nullptr;    // symbolic factor + plan (host only)
  // device copies of perm and vmap for the device-side permutations, made
  // by the first request that needs them (dev_state 0 none, 1 ready, -1 failed)
  int* d_perm = nullptr;
  int* d_vmap = nullptr;
  std::mutex dev_mu;
  int dev_state = 0;
  size_t inst_bytes = 0;
  int state = 0;              // 0 being built, 1 ready, -1 failed
  int n_created = 0;          // instances made so far
};

struct Instance {
  Factor* F = nullptr;
  Pattern* pat = nullptr;
  uint64_t vkey = 0;          // values of the resident numeric factor
  bool has_values = false;
  bool busy = false;
  uint64_t last_use = 0;
  size_t bytes = 0;
};

struct Request {
  long id = 0;
  taucs_ccs_matrix A{};       // arrays owned by the caller until completion
  int nrhs = 0;
  const double* B = nullptr;
  double* X = nullptr;
  double tol = 1e-12;
  double t_submit = 0, t_start = 0, t_done = 0;
  int status = 0, steps = 0;
  double resid = 0;
  bool factored = false;      // false: solved on a resident factor
  bool done = false;
};

struct Worker {
  cudaStream_t stream = nullptr;      // low priority (large systems)
  cudaStream_t stream_hi = nullptr;   // high priority (small systems)
  double* h_vals = nullptr;   // pinned staging: A's values as given
  size_t h_vals_len = 0;
  double* h_b = nullptr;      // pinned staging: b and x in the caller's order
  double* h_x = nullptr;
  size_t h_vec_len = 0;
  double* d_vals = nullptr;   // device copies of the same (stream-ordered allocations)
  double* d_b = nullptr;
  double* d_x = nullptr;
};

}  // namespace

class Server {
 public:
  Server(int workers, size_t budget, int device) : budget_(budget), device_(device) {
    for (int w = 0; w < workers; w++) workers_.emplace_back(new Worker());
    for (int w = 0; w < workers; w++) threads_.emplace_back([this, w] { worker_main(w); });
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_work_.notify_all();
    cv_mem_.notify_all();
    for (auto& t : threads_) t.join();
    cudaSetDevice(device_);
    for (auto& I : instances_) taucs_supernodal_factor_free(I->F);
    for (auto& kv : patterns_) {
      if (kv.second->proto) taucs_supernodal_factor_free(kv.second->proto);
      tb::dfree(kv.second->d_perm);
      tb::dfree(kv.second->d_vmap);
    }
    for (auto& w : workers_) {
      tb::dfree(w->d_vals);
      tb::dfree(w->d_b);
      tb::dfree(w->d_x);
      if (w->stream) cudaStreamDestroy(w->stream);
      if (w->stream_hi) cudaStreamDestroy(w->stream_hi);
      if (w->h_vals) tb::hfree(w->h_vals);
      if (w->h_b) tb::hfree(w->h_b);
      if (w->h_x) tb::hfree(w->h_x);
    }
    for (auto& kv : reqs_) delete kv.second;
  }

  long submit(const taucs_ccs_matrix* A, int nrhs, const double* B, double* X, double tol) {
    Request* r = new Request();
    r->A = *A;
    r->nrhs = nrhs;
    r->B = B;
    r->X = X;
    r->tol = tol;
    r->t_submit = now_s();
    {
      std::lock_guard<std::mutex> lk(mu_);
      r->id = next_id_++;
      reqs_[r->id] = r;
      queue_.push_back(r);
    }
    cv_work_.notify_one();
    return r->id;
  }

  int wait(long id, double* latency, int* steps, double* resid, int* factored) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return -2;
    Request* r = it->second;
    cv_done_.wait(lk, [&] { return r->done; });
    if (latency) *latency = r->t_done - r->t_submit;
    if (steps) *steps = r->steps;
    if (resid) *resid = r->resid;
    if (factored) *factored = r->factored ? 1 : 0;
    const int st = r->status;
    reqs_.erase(it);
    delete r;
    return st;
  }

  void stats(taucs_b200_server_info* s) {
    std::lock_guard<std::mutex> lk(mu_);
    s->patterns = (int) patterns_.size();
    s->instances = (int) instances_.size();
    s->bytes_in_use = (double) in_use_;
    s->budget_bytes = (double) budget_;
    s->factorizations = n_factor_;
    s->resident_solves = n_resident_;
    s->evictions = n_evict_;
    s->waits_for_memory = n_memwait_;
    s->failed = n_failed_;
    s->queued = (long) queue_.size();
  }

 private:
  void worker_main(int w) {
    Worker& W = *workers_[w];
    cudaSetDevice(device_);
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    cudaStreamCreateWithPriority(&W.stream, cudaStreamNonBlocking, lo);
    cudaStreamCreateWithPriority(&W.stream_hi, cudaStreamNonBlocking, hi);
    for (;;) {
      Request* r;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_work_.wait(lk, [&] { return stop_ || !queue_.empty(); });
        if (stop_ && queue_.empty()) return;
        r = queue_.front();
        queue_.pop_front();
      }
      r->t_start = now_s();
      const int st = process(r, W);
      {
        std::lock_guard<std::mutex> lk(mu_);
        r->status = st;
        r->t_done = now_s();
        r->done = true;
        if (st) n_failed_++;
      }
      cv_done_.notify_all();
    }
  }

  // staging buffers of a worker, grown to the largest request it has seen;
  // the device ones come from the stream-ordered allocator (no device-wide
  // synchronisation) and are ready when the stream has drained
  bool grow(Worker& W, size_t nvals, size_t nvec, cudaStream_t st) {
    if (nvals <= W.h_vals_len && nvec <= W.h_vec_len) return true;
    if (nvals > W.h_vals_len) {
      if (W.h_vals) tb::hfree(W.h_vals);
      cudaFreeAsync(W.d_vals, st);
      W.h_vals = nullptr;
      W.d_vals = nullptr;
      if (tb::hmalloc((void**) &W.h_vals, sizeof(double) * nvals) != cudaSuccess ||
          cudaMallocAsync((void**) &W.d_vals, sizeof(double) * nvals, st) != cudaSuccess)
        return false;
      W.h_vals_len = nvals;
    }
    if (nvec > W.h_vec_len) {
      if (W.h_b) tb::hfree(W.h_b);
      if (W.h_x) tb::hfree(W.h_x);
      cudaFreeAsync(W.d_b, st);
      cudaFreeAsync(W.d_x, st);
      W.h_b = W.h_x = nullptr;
      W.d_b = W.d_x = nullptr;
      if (tb::hmalloc((void**) &W.h_b, sizeof(double) * nvec) != cudaSuccess ||
          tb::hmalloc((void**) &W.h_x, sizeof(double) * nvec) != cudaSuccess ||
          cudaMallocAsync((void**) &W.d_b, sizeof(double) * nvec, st) != cudaSuccess ||
          cudaMallocAsync((void**) &W.d_x, sizeof(double) * nvec, st) != cudaSuccess)
        return false;
      W.h_vec_len = nvec;
    }
    return cudaStreamSynchronize(st) == cudaSuccess;
  }

  // device copies of the pattern's permutation and value map, uploaded once
  // (their bytes count against the budget like an instance's)
  bool pattern_device(Pattern* P, cudaStream_t st) {
    std::lock_guard<std::mutex> lk(P->dev_mu);
    if (P->dev_state == 0) {
      const size_t bytes = sizeof(int) * (P->perm.size() + P->vmap.size());
      bool ok = tb::dmalloc((void**) &P->d_perm, sizeof(int) * std::max<size_t>(P->perm.size(), 1)) == cudaSuccess &&
                tb::dmalloc((void**) &P->d_vmap, sizeof(int) * std::max<size_t>(P->vmap.size(), 1)) == cudaSuccess &&
                cudaMemcpyAsync(P->d_perm, P->perm.data(), sizeof(int) * P->perm.size(), cudaMemcpyHostToDevice,
                                st) == cudaSuccess &&
                cudaMemcpyAsync(P->d_vmap, P->vmap.data(), sizeof(int) * P->vmap.size(), cudaMemcpyHostToDevice,
                                st) == cudaSuccess &&
                cudaStreamSynchronize(st) == cudaSuccess;
      P->dev_state = ok ? 1 : -1;
      if (ok) {
        std::lock_guard<std::mutex> lk2(mu_);
        in_use_ += bytes;
      } else {
        set_error("server: could not upload a pattern's permutation to the device");
      }
    }
    return P->dev_state == 1;
  }

  int process(Request* r, Worker& W) {
    const taucs_ccs_matrix& A = r->A;
    const int n = A.n;
    const int64_t nnz = A.colptr[n];
    cudaStream_t st = n < SMALL_SYSTEM_N ? W.stream_hi : W.stream;
    taucs_b200_set_stream(st);
    Pattern* P = get_pattern(A);
    if (!P) return -1;
    const uint64_t vkey = hash_bytes(A.values.d, sizeof(double) * nnz, (uint64_t) P);
    bool hit = false;
    Instance* I = acquire(P, vkey, &hit);
    if (!I) return -1;
    const size_t nvec = (size_t) n * r->nrhs;
    int rc = grow(W, (size_t) nnz, nvec, st) && pattern_device(P, st) ? 0 : -1;
    Factor* F = I->F;
    if (!rc && !hit) {
      // A's values as given go to the device in one sequential copy; the
      // values of P A P^T are gathered there through the pattern's value
      // map, then FP32 fronts
      memcpy(W.h_vals, A.values.d, sizeof(double) * nnz);
      rc = ensure_device(F);
      if (!rc && cudaMemcpyAsync(W.d_vals, W.h_vals, sizeof(double) * nnz, cudaMemcpyHostToDevice, st) != cudaSuccess)
        rc = -1;
      if (!rc) rc = gather_values_device(nnz, P->d_vmap, W.d_vals, F->dA);
      F->precision = 1;
      if (!rc) rc = numeric_device(F, F->dA, true);
      r->factored = true;
    }
    if (!rc) {
      // b in the caller's order to the device; P b, the refinement in the
      // instance's own vectors (8 columns at a time, so its recorded launch
      // sequences are replayed by every worker) and x = P^T y on the device
      memcpy(W.h_b, r->B, sizeof(double) * nvec);
      if (cudaMemcpyAsync(W.d_b, W.h_b, sizeof(double) * nvec, cudaMemcpyHostToDevice, st) != cudaSuccess) rc = -1;
      std::vector<double> res(r->nrhs, 0.0);
      const int s = rc ? -1 : solve_refine_permuted(F, r->nrhs, W.d_x, W.d_b, P->d_perm, r->tol, 10, res.data());
      if (s < 0) rc = -1;
      if (!rc && (cudaMemcpyAsync(W.h_x, W.d_x, sizeof(double) * nvec, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                  cudaStreamSynchronize(st) != cudaSuccess))
        rc = -1;
      if (!rc) memcpy(r->X, W.h_x, sizeof(double) * nvec);
      r->steps = s;
      r->resid = *std::max_element(res.begin(), res.end());
    }
    release(I, rc == 0, vkey);
    return rc;
  }

  // ordering, value map and symbolic factor of A's pattern, built once
  Pattern* get_pattern(const taucs_ccs_matrix& A) {
    const int n = A.n;
    const int64_t nnz = A.colptr[n];
    uint64_t key = hash_bytes(A.colptr, sizeof(int) * (size_t) (n + 1), 0x243f6a8885a308d3ull ^ (uint64_t) n);
    key = hash_bytes(A.rowind, sizeof(int) * (size_t) nnz, key);
    Pattern* P;
    {
      std::unique_lock<std::mutex> lk(mu_);
      auto it = patterns_.find(key);
      if (it != patterns_.end()) {
        P = it->second.get();
        cv_pat_.wait(lk, [&] { return P->state != 0; });
        return P->state == 1 ? P : nullptr;
      }
      patterns_[key].reset(new Pattern());
      P = patterns_[key].get();
    }
    int ok = 0;
    P->n = n;
    P->nnz = nnz;
    int *perm = nullptr, *iperm = nullptr;
    taucs_ccs_matrix Ai = A;
    taucs_ccs_order(&Ai, &perm, &iperm, (char*) "amd");
    if (perm) {
      // value positions travel through the permutation as values
      std::vector<double> idx((size_t) nnz);
      for (int64_t k = 0; k < nnz; k++) idx[k] = (double) k;
      Ai.values.d = idx.data();
      taucs_ccs_matrix* PA = taucs_ccs_permute_symmetrically(&Ai, perm, iperm);
      if (PA) {
        P->perm.assign(perm, perm + n);
        P->vmap.resize((size_t) nnz);
        for (int64_t k = 0; k < nnz; k++) P->vmap[k] = (int) PA->values.d[k];
        P->proto = symbolic(PA, 0);
        if (P->proto) {
          P->inst_bytes = predict_bytes(P->proto->plan);
          ok = 1;
        }
        taucs_ccs_free(PA);
      }
    }
    free(perm);
    free(iperm);
    {
      std::lock_guard<std::mutex> lk(mu_);
      P->state = ok ? 1 : -1;
    }
    cv_pat_.notify_all();
    return ok ? P : nullptr;
  }

  // An instance for one request, in this order of preference: the idle
  // instance that holds exactly these values (solve only); an idle instance
  // of the pattern without values; the least recently used idle instance of
  // the pattern; a new instance while the pattern has fewer than
  // MAX_INSTANCES_PER_PATTERN and the budget allows; after evicting idle
  // instances of other patterns, least recently used first, a new instance;
  // otherwise wait for a running request to finish.
  Instance* acquire(Pattern* P, uint64_t vkey, bool* hit) {
    std::unique_lock<std::mutex> lk(mu_);
    if (P->inst_bytes > budget_) {
      set_error("server: one instance of this pattern needs more device memory than the budget");
      return nullptr;
    }
    bool waited = false;
    for (;;) {
      Instance *empty = nullptr, *lru = nullptr;
      int count = 0;
      for (auto& I : instances_) {
        if (I->pat != P) continue;
        count++;
        if (I->busy) continue;
        if (I->has_values && I->vkey == vkey) {
          I->busy = true;
          I->last_use = ++tick_;
          *hit = true;
          n_resident_++;
          return I.get();
        }
        if (!I->has_values && !empty) empty = I.get();
        if (I->has_values && (!lru || I->last_use < lru->last_use)) lru = I.get();
      }
      // an idle instance of the pattern is reused before a new one is made:
      // a new instance starts cold (device buffers, launch graphs), so
      // instances are only added while all of the pattern's are busy
      Instance* take = empty ? empty : lru;
      if (!take && count < MAX_INSTANCES_PER_PATTERN && in_use_ + P->inst_bytes <= budget_)
        return create(P, lk, hit);
      if (take) {
        take->busy = true;
        take->has_values = false;
        take->last_use = ++tick_;
        *hit = false;
        n_factor_++;
        return take;
      }
      if (in_use_ + P->inst_bytes <= budget_) return create(P, lk, hit);
      // evict the least recently used idle instance of another pattern
      auto victim = instances_.end();
      for (auto it = instances_.begin(); it != instances_.end(); ++it)
        if (!(*it)->busy && (*it)->F && (*it)->pat != P &&
            (victim == instances_.end() || (*it)->last_use < (*victim)->last_use))
          victim = it;
      if (victim != instances_.end()) {
        std::unique_ptr<Instance> V = std::move(*victim);
        instances_.erase(victim);
        in_use_ -= V->bytes;
        n_evict_++;
        lk.unlock();
        taucs_supernodal_factor_free(V->F);
        lk.lock();
        continue;
      }
      if (!waited) n_memwait_++;
      waited = true;
      if (stop_) return nullptr;
      cv_mem_.wait(lk);
    }
  }

  // a new instance of P (host copy of the symbolic factor; device buffers
  // are allocated by its first factorization); called with mu_ held
  Instance* create(Pattern* P, std::unique_lock<std::mutex>& lk, bool* hit) {
    in_use_ += P->inst_bytes;
    std::unique_ptr<Instance> I(new Instance());
    I->pat = P;
    I->busy = true;
    I->bytes = P->inst_bytes;
    I->last_use = ++tick_;
    Instance* raw = I.get();
    instances_.push_back(std::move(I));
    // the pattern's first instance runs every launch sequence once eagerly
    // (module loading and kernel attributes happen outside any capture); the
    // later ones record their graphs on first use
    const bool first = P->n_created++ == 0;
    lk.unlock();
    Factor* F = new Factor();
    F->n = P->proto->n;
    F->sym = P->proto->sym;
    F->plan = P->proto->plan;
    F->colptr = P->proto->colptr;
    F->rowind = P->proto->rowind;
    F->precision = 1;
    F->graph_first_use = !first;
    lk.lock();
    raw->F = F;
    *hit = false;
    n_factor_++;
    return raw;
  }

  void release(Instance* I, bool ok, uint64_t vkey) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      I->busy = false;
      I->has_values = ok && (I->F->has_numeric32 || I->F->has_numeric);
      I->vkey = vkey;
      I->last_use = ++tick_;
    }
    cv_mem_.notify_all();
  }

  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_, cv_mem_, cv_pat_;
  std::deque<Request*> queue_;
  std::unordered_map<long, Request*> reqs_;
  std::unordered_map<uint64_t, std::unique_ptr<Pattern>> patterns_;
  std::vector<std::unique_ptr<Instance>> instances_;
  std::vector<std::unique_ptr<Worker>> workers_;
  std::vector<std::thread> threads_;
  size_t budget_, in_use_ = 0;
  int device_;
  bool stop_ = false;
  long next_id_ = 1;
  uint64_t tick_ = 0;
  long n_factor_ = 0, n_resident_ = 0, n_evict_ = 0, n_memwait_ = 0, n_failed_ = 0;
};

}  // namespace tb

using tb::Server;

extern "C" void* taucs_b200_server_create(int workers, double hbm_budget_bytes) {
  if (workers < 1 || hbm_budget_bytes <= 0) return nullptr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  return new (std::nothrow) Server(workers, (size_t) hbm_budget_bytes, dev);
}

extern "C" long taucs_b200_server_submit(void* S, const taucs_ccs_matrix* A, int nrhs, const double* B, double* X,
                                         double tol) {
  if (!S || !A || nrhs < 1 || !B || !X || !(A->flags & TAUCS_DOUBLE) || !(A->flags & TAUCS_LOWER)) return -1;
  return ((Server*) S)->submit(A, nrhs, B, X, tol);
}

extern "C" int taucs_b200_server_wait(void* S, long id, double* latency_s, int* steps, double* residual,
                                      int* factored) {
  if (!S) return -2;
  return ((Server*) S)->wait(id, latency_s, steps, residual, factored);
}

extern "C" int taucs_b200_server_stats(void* S, taucs_b200_server_info* out) {
  if (!S || !out) return -1;
  ((Server*) S)->stats(out);
  return 0;
}

extern "C" void taucs_b200_server_destroy(void* S) { delete (Server*) S; }

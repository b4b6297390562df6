// Device and pinned-host allocations of the library, counted so that
// allocation failures can be induced and leaks detected -- the device-memory
// counterpart of the reference's allocation tracking and failure injection
// (src/taucs_malloc.c:127-250: taucs_allocation_induce_failure, _attempts,
// _mark_clean, _assert_clean), exercised like progs/xtest_allocations.c:62-87
// (every allocation of a call made to fail in turn; the call must fail
// cleanly and leave nothing allocated).
#include <atomic>
#include <mutex>
#include <unordered_map>

#include "kernels.h"

namespace tb {

namespace {

std::mutex g_mu;
std::unordered_map<void*, size_t> g_live;   // live allocations and their sizes
double g_live_bytes = 0.0;
long g_attempts = 0;                         // attempts since the last mark
long g_induce = -1;                          // attempt index that fails, -1 none

// true when this attempt is the one to fail
bool attempt() {
  std::lock_guard<std::mutex> lk(g_mu);
  const bool fail = g_attempts == g_induce;
  if (fail) g_induce = -1;
  g_attempts++;
  return !fail;
}

void track(void* p, size_t bytes) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_live[p] = bytes;
  g_live_bytes += (double) bytes;
}

void untrack(void* p) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_live.find(p);
  if (it == g_live.end()) return;
  g_live_bytes -= (double) it->second;
  g_live.erase(it);
}

}  // namespace

cudaError_t dmalloc_raw(void** p, size_t bytes) {
  *p = nullptr;
  if (!attempt()) {
    tprintf("taucs_b200 allocation: inducing a failure of a %zu-byte device allocation\n", bytes);
    return cudaErrorMemoryAllocation;
  }
  const cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaSuccess) track(*p, bytes);
  return e;
}

cudaError_t dfree(void* p) {
  if (!p) return cudaSuccess;
  untrack(p);
  return cudaFree(p);
}

cudaError_t hmalloc_raw(void** p, size_t bytes) {
  *p = nullptr;
  if (!attempt()) {
    tprintf("taucs_b200 allocation: inducing a failure of a %zu-byte pinned host allocation\n", bytes);
    return cudaErrorMemoryAllocation;
  }
  const cudaError_t e = cudaMallocHost(p, bytes);
  if (e == cudaSuccess) track(*p, bytes);
  return e;
}

cudaError_t hfree(void* p) {
  if (!p) return cudaSuccess;
  untrack(p);
  return cudaFreeHost(p);
}

}  // namespace tb

using namespace tb;

extern "C" {

void taucs_b200_allocation_induce_failure(int i) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_induce = i;
}

int taucs_b200_allocation_attempts(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  return (int) g_attempts;
}

void taucs_b200_allocation_mark_clean(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_attempts = 0;
  g_induce = -1;
}

int taucs_b200_allocation_live(double* bytes) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (bytes) *bytes = g_live_bytes;
  return (int) g_live.size();
}

}  // extern "C"

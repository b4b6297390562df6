// Per-kernel-class device timing with CUDA events (off by default).  Used by
// benchmarks to report the achieved rate of the dominant kernel over the
// timed region; the events are recorded on the stream the kernels run on.
#include <mutex>
#include <vector>

#include "kernels.h"

namespace tb {

bool per_device_once(PerDeviceOnce& pd, bool (*setup)()) {
  int d = -1;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= MAX_DEVICES) return false;
  std::call_once(pd.once[d], [&] { pd.ok[d] = setup(); });
  return pd.ok[d];
}

namespace {

struct Rec {
  cudaEvent_t a, b;
  int kc, tag;
  double flops, bytes;
};

std::mutex g_mu;
bool g_on = false;
std::vector<Rec> g_recs;
std::vector<cudaEvent_t> g_pool;
cudaEvent_t g_open = nullptr;
double g_ms[KC_COUNT], g_flops[KC_COUNT], g_bytes[KC_COUNT];
long g_n[KC_COUNT];
std::vector<ProfEntry> g_log;   // every launch, in order
int g_tag = -1;

cudaEvent_t get_event() {
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

void drain() {
  for (Rec& r : g_recs) {
    cudaEventSynchronize(r.b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.a, r.b);
    g_ms[r.kc] += ms;
    if (g_log.size() < (size_t) 1 << 20) g_log.push_back(ProfEntry{r.kc, r.tag, ms});
    g_flops[r.kc] += r.flops;
    g_bytes[r.kc] += r.bytes;
    g_n[r.kc] += 1;
    g_pool.push_back(r.a);
    g_pool.push_back(r.b);
  }
  g_recs.clear();
}

}  // namespace

bool prof_enabled() { return g_on; }

void prof_tag(int tag) { g_tag = tag; }

std::vector<ProfEntry> prof_take_log() {
  std::lock_guard<std::mutex> lk(g_mu);
  drain();
  std::vector<ProfEntry> out;
  out.swap(g_log);
  return out;
}

void prof_begin(int kc, cudaStream_t st) {
  (void) kc;
  if (!g_on) return;
  std::lock_guard<std::mutex> lk(g_mu);
  g_open = get_event();
  cudaEventRecord(g_open, st);
}

void prof_end(int kc, cudaStream_t st, double flops, double bytes) {
  if (!g_on) return;
  std::lock_guard<std::mutex> lk(g_mu);
  cudaEvent_t b = get_event();
  cudaEventRecord(b, st);
  g_recs.push_back(Rec{g_open, b, kc, g_tag, flops, bytes});
  if (g_recs.size() > 4096) drain();
}

}  // namespace tb

using namespace tb;

extern "C" {

int taucs_b200_profile(int enable) {
  std::lock_guard<std::mutex> lk(g_mu);
  drain();
  g_on = enable != 0;
  for (int k = 0; k < KC_COUNT; k++) { g_ms[k] = g_flops[k] = g_bytes[k] = 0.0; g_n[k] = 0; }
  g_log.clear();
  return 0;
}

long taucs_b200_profile_log(int* kernel_class, float* ms, long cap) {
  std::lock_guard<std::mutex> lk(g_mu);
  drain();
  const long n = (long) g_log.size();
  for (long i = 0; i < n && i < cap; i++) {
    if (kernel_class) kernel_class[i] = g_log[i].kc;
    if (ms) ms[i] = g_log[i].ms;
  }
  return n;
}

int taucs_b200_profile_read(int kernel_class, double* ms, long* launches, double* flops, double* bytes) {
  if (kernel_class < 0 || kernel_class >= KC_COUNT) return -1;
  std::lock_guard<std::mutex> lk(g_mu);
  drain();
  if (ms) *ms = g_ms[kernel_class];
  if (launches) *launches = g_n[kernel_class];
  if (flops) *flops = g_flops[kernel_class];
  if (bytes) *bytes = g_bytes[kernel_class];
  return 0;
}

}  // extern "C"

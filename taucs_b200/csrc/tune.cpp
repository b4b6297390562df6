// Tuning table of the GEMM variants (no counterpart in the reference).
//
// taucs_b200_autotune measures, per level of one factor, the device time of
// both GEMM variants of each product (panel updates, update matrix).  The
// measurements go into a process-wide table keyed by what decides the
// outcome -- precision, product, and the shape of the level's largest
// product (rows and K, in powers of two) -- so that every later handle
// (new patterns, the request server's instances, batches) takes the faster
// variant per level from the table without tuning again, and the table can
// be written to and read from a file to carry the choices across processes.
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <tuple>

#include "kernels.h"

namespace tb {

namespace {

struct Entry {
  double ms[2] = {0.0, 0.0};
  long n[2] = {0, 0};
};

using Key = std::tuple<int, int, int, int>;   // precision, product (0 panel, 1 U), row class, K class

std::mutex g_mu;
std::map<Key, Entry> g_table;

int cls(double x) { return x <= 1.0 ? 0 : (int) std::ceil(std::log2(x)); }

// shape class of level h's product `kind`: its largest front by product size
bool level_key(const Plan& P, int h, int prec, int kind, Key* key) {
  const LevelPlan& LP = P.levels[h];
  double best = -1.0;
  int rows = 0, k = 0;
  for (int fi : LP.big_fronts) {
    const FrontDesc& F = P.fronts[fi];
    const int m = F.f - F.s;
    const int r = kind ? m : F.f, kk = F.s;
    if (kind && m <= 0) continue;
    const double sz = (double) r * r * kk;
    if (sz > best) { best = sz; rows = r; k = kk; }
  }
  if (best < 0) return false;
  *key = Key{prec, kind, cls(rows), cls(k)};
  return true;
}

}  // namespace

void tune_record(const Plan& P, int prec, const std::vector<double> (&t)[2]) {
  std::lock_guard<std::mutex> lk(g_mu);
  for (int h = 0; h < P.n_levels; h++)
    for (int kind = 0; kind < 2; kind++) {
      Key key;
      if (!level_key(P, h, prec, kind, &key)) continue;
      Entry& e = g_table[key];
      for (int v = 0; v < 2; v++) {
        const double ms = t[v][2 * h + kind];
        if (ms > 0.0) { e.ms[v] += ms; e.n[v]++; }
      }
    }
}

bool tune_apply(Plan* P, int prec) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_table.empty()) return false;
  std::vector<uint8_t> c((size_t) 2 * P->n_levels, 0);
  bool any = false;
  for (int h = 0; h < P->n_levels; h++)
    for (int kind = 0; kind < 2; kind++) {
      Key key;
      if (!level_key(*P, h, prec, kind, &key)) continue;
      auto it = g_table.find(key);
      if (it == g_table.end() || !it->second.n[0] || !it->second.n[1]) continue;
      const Entry& e = it->second;
      c[2 * h + kind] = (e.ms[1] / e.n[1] < e.ms[0] / e.n[0]) ? 1 : 0;
      any = true;
    }
  if (any) P->gemm_choice[prec] = c;
  return any;
}

}  // namespace tb

using namespace tb;

extern "C" {

int taucs_b200_tuning_save(const char* path) {
  if (!path) return -1;
  FILE* fp = fopen(path, "w");
  if (!fp) return -1;
  std::lock_guard<std::mutex> lk(g_mu);
  fprintf(fp, "# taucs_b200 GEMM tuning: precision product row_class k_class ms0 n0 ms1 n1\n");
  for (const auto& kv : g_table)
    fprintf(fp, "%d %d %d %d %.9g %ld %.9g %ld\n", std::get<0>(kv.first), std::get<1>(kv.first),
            std::get<2>(kv.first), std::get<3>(kv.first), kv.second.ms[0], kv.second.n[0], kv.second.ms[1],
            kv.second.n[1]);
  return fclose(fp) == 0 ? 0 : -1;
}

int taucs_b200_tuning_load(const char* path) {
  if (!path) return -1;
  FILE* fp = fopen(path, "r");
  if (!fp) return -1;
  char line[256];
  int loaded = 0;
  std::lock_guard<std::mutex> lk(g_mu);
  while (fgets(line, sizeof line, fp)) {
    if (line[0] == '#') continue;
    int p, k, r, c;
    double m0, m1;
    long n0, n1;
    if (sscanf(line, "%d %d %d %d %lf %ld %lf %ld", &p, &k, &r, &c, &m0, &n0, &m1, &n1) != 8) continue;
    Entry& e = g_table[Key{p, k, r, c}];
    e.ms[0] += m0; e.n[0] += n0; e.ms[1] += m1; e.n[1] += n1;
    loaded++;
  }
  fclose(fp);
  return loaded;
}

int taucs_b200_tuning_entries(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  return (int) g_table.size();
}

void taucs_b200_tuning_clear(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_table.clear();
}

}  // extern "C"

// Host-side sparse-matrix support for the C ABI: CCS create/free, symmetric
// permutation, symmetric SpMV, vector permutes, the reference's generators,
// a seeded lognormal-coefficient generator, logging and timers.
//
// Reference behaviour followed (file:line):
//   taucs_dccs_create / taucs_ccs_free ...... src/taucs_ccs_base.c:72-132
//   taucs_dccs_permute_symmetrically ........ src/taucs_ccs_ops.c:174-257
//   taucs_dccs_times_vec .................... src/taucs_ccs_ops.c:299-344
//   taucs_dvec_permute / _ipermute .......... src/taucs_vec_base.c:194-206
//   taucs_ccs_generate_mesh2d ............... src/taucs_ccs_generators.c:89-195
//   taucs_ccs_generate_mesh3d ............... src/taucs_ccs_generators.c:197-261
//   taucs_logfile / taucs_printf ............ src/taucs_logging.c:32-80
//   taucs_wtime / taucs_ctime ............... src/taucs_timer.c:250-290
// The generators must emit the same rows in the same order with the same
// values as the reference (the matrices are parity inputs).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <sys/resource.h>
#include <sys/time.h>

#include "internal.h"

namespace tb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) {
  g_last_error = msg;
  tprintf("taucs_b200: %s\n", msg.c_str());
}

const char* last_error() { return g_last_error.c_str(); }

static std::mutex g_log_mu;
static FILE* g_log = nullptr;
static bool g_log_owned = false;

int tprintf(const char* fmt, ...) {
  std::lock_guard<std::mutex> lk(g_log_mu);
  if (!g_log) return 0;
  va_list ap;
  va_start(ap, fmt);
  int r = vfprintf(g_log, fmt, ap);
  va_end(ap);
  fflush(g_log);
  return r;
}

}  // namespace tb

using namespace tb;

extern "C" {

void taucs_logfile(char* file_prefix) {
  std::lock_guard<std::mutex> lk(g_log_mu);
  if (g_log && g_log_owned) fclose(g_log);
  g_log = nullptr;
  g_log_owned = false;
  if (!file_prefix || !strcmp(file_prefix, "none")) return;
  if (!strcmp(file_prefix, "stdout")) { g_log = stdout; return; }
  if (!strcmp(file_prefix, "stderr")) { g_log = stderr; return; }
  std::string name = std::string(file_prefix) + ".log";
  g_log = fopen(name.c_str(), "w");
  g_log_owned = g_log != nullptr;
}

int taucs_printf(char* fmt, ...) {
  std::lock_guard<std::mutex> lk(g_log_mu);
  if (!g_log) return 0;
  va_list ap;
  va_start(ap, fmt);
  int r = vfprintf(g_log, fmt, ap);
  va_end(ap);
  fflush(g_log);
  return r;
}

double taucs_wtime(void) {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return (double) tv.tv_sec + 1e-6 * (double) tv.tv_usec;
}

double taucs_ctime(void) {
  struct rusage ru;
  getrusage(RUSAGE_SELF, &ru);
  return (double) ru.ru_utime.tv_sec + 1e-6 * (double) ru.ru_utime.tv_usec;
}

taucs_ccs_matrix* taucs_ccs_create(int m, int n, int nnz, int flags) {
  if (n < 0 || m < 0 || nnz < 0) return nullptr;
  if (!(flags & TAUCS_DOUBLE) && !(flags & TAUCS_SINGLE)) {
    set_error("taucs_ccs_create: only TAUCS_DOUBLE and TAUCS_SINGLE values are supported");
    return nullptr;
  }
  taucs_ccs_matrix* A = (taucs_ccs_matrix*) malloc(sizeof(taucs_ccs_matrix));
  if (!A) return nullptr;
  size_t esz = (flags & TAUCS_DOUBLE) ? sizeof(double) : sizeof(float);
  A->n = n;
  A->m = m;
  A->flags = flags;
  A->colptr = (int*) malloc(sizeof(int) * ((size_t) n + 1));
  A->rowind = (int*) malloc(sizeof(int) * (size_t) (nnz > 0 ? nnz : 1));
  A->values.v = malloc(esz * (size_t) (nnz > 0 ? nnz : 1));
  if (!A->colptr || !A->rowind || !A->values.v) {
    free(A->colptr); free(A->rowind); free(A->values.v); free(A);
    return nullptr;
  }
  A->colptr[0] = 0;
  return A;
}

taucs_ccs_matrix* taucs_dccs_create(int m, int n, int nnz) {
  return taucs_ccs_create(m, n, nnz, TAUCS_DOUBLE);
}

void taucs_ccs_free(taucs_ccs_matrix* A) {
  if (!A) return;
  free(A->colptr);
  free(A->rowind);
  free(A->values.v);
  free(A);
}

void taucs_dccs_free(taucs_ccs_matrix* A) { taucs_ccs_free(A); }

taucs_ccs_matrix* taucs_dccs_permute_symmetrically(taucs_ccs_matrix* A, int* perm, int* invperm) {
  (void) perm;
  if (!A || !invperm) return nullptr;
  if (!(A->flags & (TAUCS_SYMMETRIC | TAUCS_HERMITIAN)) || !(A->flags & TAUCS_LOWER)) {
    set_error("taucs_ccs_permute_symmetrically: lower triangle of a symmetric matrix required");
    return nullptr;
  }
  const int n = A->n;
  const int nnz = A->colptr[n];
  taucs_ccs_matrix* P = taucs_ccs_create(n, n, nnz, A->flags);
  if (!P) return nullptr;
  // entry (i, j) goes to (max(I,J), min(I,J)) with I = invperm[i], J = invperm[j];
  // within each new column, entries keep the order in which A is traversed
  std::vector<int> len(n, 0);
  for (int j = 0; j < n; j++)
    for (int ip = A->colptr[j]; ip < A->colptr[j + 1]; ip++) {
      int I = invperm[A->rowind[ip]], J = invperm[j];
      len[I < J ? I : J]++;
    }
  P->colptr[0] = 0;
  for (int j = 0; j < n; j++) P->colptr[j + 1] = P->colptr[j] + len[j];
  for (int j = 0; j < n; j++) len[j] = P->colptr[j];
  const bool dbl = (A->flags & TAUCS_DOUBLE) != 0;
  for (int j = 0; j < n; j++)
    for (int ip = A->colptr[j]; ip < A->colptr[j + 1]; ip++) {
      int I = invperm[A->rowind[ip]], J = invperm[j];
      if (I < J) { int t = I; I = J; J = t; }
      int dst = len[J]++;
      P->rowind[dst] = I;
      if (dbl) P->values.d[dst] = A->values.d[ip];
      else P->values.s[dst] = A->values.s[ip];
    }
  return P;
}

taucs_ccs_matrix* taucs_ccs_permute_symmetrically(taucs_ccs_matrix* A, int* perm, int* invperm) {
  return taucs_dccs_permute_symmetrically(A, perm, invperm);
}

void taucs_dccs_times_vec(taucs_ccs_matrix* A, double* X, double* B) {
  const int n = A->n;
  for (int i = 0; i < n; i++) B[i] = 0.0;
  const bool sym = (A->flags & (TAUCS_SYMMETRIC | TAUCS_HERMITIAN)) != 0;
  for (int j = 0; j < n; j++)
    for (int ip = A->colptr[j]; ip < A->colptr[j + 1]; ip++) {
      int i = A->rowind[ip];
      double a = A->values.d[ip];
      B[i] += X[j] * a;
      if (sym && i != j) B[j] += X[i] * a;
    }
}

void taucs_ccs_times_vec(taucs_ccs_matrix* A, void* X, void* B) {
  if (A->flags & TAUCS_DOUBLE) taucs_dccs_times_vec(A, (double*) X, (double*) B);
}

void taucs_dvec_permute(int n, double v[], double pv[], int p[]) {
  for (int i = 0; i < n; i++) pv[i] = v[p[i]];
}

void taucs_dvec_ipermute(int n, double pv[], double v[], int invp[]) {
  for (int i = 0; i < n; i++) v[invp[i]] = pv[i];
}

void taucs_vec_permute(int n, int flags, void* v, void* pv, int p[]) {
  if (flags & TAUCS_DOUBLE) taucs_dvec_permute(n, (double*) v, (double*) pv, p);
  else if (flags & TAUCS_SINGLE)
    for (int i = 0; i < n; i++) ((float*) pv)[i] = ((float*) v)[p[i]];
}

void taucs_vec_ipermute(int n, int flags, void* pv, void* v, int invp[]) {
  if (flags & TAUCS_DOUBLE) taucs_dvec_ipermute(n, (double*) pv, (double*) v, invp);
  else if (flags & TAUCS_SINGLE)
    for (int i = 0; i < n; i++) ((float*) v)[invp[i]] = ((float*) pv)[i];
}

// axpby = a x + b y (src/taucs_vec_base.c:56-92); the output may alias x or y
void taucs_vec_axpby(int n, int flags, double a, void* x, double b, void* y, void* axpby) {
  if (flags & TAUCS_DOUBLE) {
    const double *xv = (const double*) x, *yv = (const double*) y;
    double* o = (double*) axpby;
    for (int i = 0; i < n; i++) o[i] = a * xv[i] + b * yv[i];
  } else if (flags & TAUCS_SINGLE) {
    const float *xv = (const float*) x, *yv = (const float*) y;
    float* o = (float*) axpby;
    for (int i = 0; i < n; i++) o[i] = (float) a * xv[i] + (float) b * yv[i];
  }
}

// Euclidean norm (src/taucs_vec_base.c:29-53, BLAS nrm2 there), accumulated
// with a running scale so that no square overflows or underflows
double taucs_vec_norm2(int n, int flags, void* x) {
  double scale = 0.0, ssq = 1.0;
  for (int i = 0; i < n; i++) {
    const double v = (flags & TAUCS_SINGLE) ? (double) ((const float*) x)[i] : ((const double*) x)[i];
    if (v == 0.0) continue;
    const double a = std::fabs(v);
    if (scale < a) {
      ssq = 1.0 + ssq * (scale / a) * (scale / a);
      scale = a;
    } else {
      ssq += (a / scale) * (a / scale);
    }
  }
  return scale * std::sqrt(ssq);
}

taucs_ccs_matrix* taucs_ccs_generate_mesh2d(int n, char* which) {
  if (n <= 0 || !which) return nullptr;
  const int N = n * n;
  taucs_ccs_matrix* A = taucs_ccs_create(N, N, 3 * N, TAUCS_SYMMETRIC | TAUCS_LOWER | TAUCS_DOUBLE);
  if (!A) return nullptr;
  const double jump = 100.0;
  const bool aniso_y = !strcmp(which, "anisotropic_y");
  const bool aniso_x = !strcmp(which, "anisotropic_x");
  const bool dirichlet = !strcmp(which, "dirichlet");
  int ip = 0;
  for (int y = 0; y < n; y++)
    for (int x = 0; x < n; x++) {
      int j = x + y * n;
      A->colptr[j] = ip;
      // +y neighbour, then +x neighbour, then the diagonal
      if (y < n - 1) { A->rowind[ip] = x + (y + 1) * n; A->values.d[ip] = aniso_y ? -jump : -1.0; ip++; }
      if (x < n - 1) { A->rowind[ip] = (x + 1) + y * n; A->values.d[ip] = aniso_x ? -jump : -1.0; ip++; }
      A->rowind[ip] = j;
      double d;
      if (dirichlet) {
        d = 4.0;
      } else {
        double wx = aniso_x ? jump : 1.0, wy = aniso_y ? jump : 1.0;
        d = 0.0;
        if (x > 0) d += wx;
        if (y > 0) d += wy;
        if (x < n - 1) d += wx;
        if (y < n - 1) d += wy;
        if (x == 0 && y == 0) d += 1.0;
      }
      A->values.d[ip] = d;
      ip++;
    }
  A->colptr[N] = ip;
  return A;
}

taucs_ccs_matrix* taucs_ccs_generate_mesh3d(int X, int Y, int Z) {
  if (X <= 0 || Y <= 0 || Z <= 0) return nullptr;
  const int N = X * Y * Z;
  taucs_ccs_matrix* A = taucs_ccs_create(N, N, 4 * N, TAUCS_SYMMETRIC | TAUCS_LOWER | TAUCS_DOUBLE);
  if (!A) return nullptr;
  int ip = 0;
  for (int z = 0; z < Z; z++)
    for (int y = 0; y < Y; y++)
      for (int x = 0; x < X; x++) {
        int j = z * X * Y + y * X + x;
        A->colptr[j] = ip;
        if (x < X - 1) { A->rowind[ip] = j + 1; A->values.d[ip] = -1.0; ip++; }
        if (y < Y - 1) { A->rowind[ip] = j + X; A->values.d[ip] = -1.0; ip++; }
        if (z < Z - 1) { A->rowind[ip] = j + X * Y; A->values.d[ip] = -1.0; ip++; }
        double d = 0.0;
        if (x < X - 1) d += 1.0;
        if (y < Y - 1) d += 1.0;
        if (z < Z - 1) d += 1.0;
        if (x > 0) d += 1.0;
        if (y > 0) d += 1.0;
        if (z > 0) d += 1.0;
        if (x == 0 && y == 0 && z == 0) d += 1.0;
        A->rowind[ip] = j;
        A->values.d[ip] = d;
        ip++;
      }
  A->colptr[N] = ip;
  return A;
}

// ---- seeded lognormal-coefficient operator (no reference counterpart)

static inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// standard normal for stream position k (Box-Muller on two hashed uniforms)
static inline double normal_at(uint64_t seed, uint64_t k) {
  uint64_t a = splitmix64(seed ^ (2 * k));
  uint64_t b = splitmix64(seed ^ (2 * k + 1) ^ 0xD1B54A32D192ED03ull);
  double u1 = ((double) (a >> 11) + 1.0) * (1.0 / 9007199254740992.0);  // (0, 1]
  double u2 = (double) (b >> 11) * (1.0 / 9007199254740992.0);          // [0, 1)
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

taucs_ccs_matrix* taucs_b200_generate_lognormal(int X, int Y, int Z, double sigma,
                                                double ax, double ay, double az,
                                                unsigned long long seed) {
  const bool two_d = (Z == 0);
  if (two_d) Z = 1;
  if (X <= 0 || Y <= 0 || Z <= 0) return nullptr;
  const int N = X * Y * Z;
  const int per = two_d ? 3 : 4;
  taucs_ccs_matrix* A = taucs_ccs_create(N, N, per * N, TAUCS_SYMMETRIC | TAUCS_LOWER | TAUCS_DOUBLE);
  if (!A) return nullptr;
  const uint64_t NN = (uint64_t) N;
  // conductance of the edge (or boundary face) with stream id k
  auto cond = [&](uint64_t k, double scale) { return scale * std::exp(sigma * normal_at(seed, k)); };
  std::vector<double> diag(N, 0.0);
  // interior edges: id 3*j + dir for the edge from j to its +dir neighbour
  // boundary faces: id 3N + 6*j + face (face 0..5 = -x,+x,-y,+y,-z,+z)
  int ip = 0;
  for (int z = 0; z < Z; z++)
    for (int y = 0; y < Y; y++)
      for (int x = 0; x < X; x++) {
        int j = z * X * Y + y * X + x;
        A->colptr[j] = ip;
        if (x < X - 1) {
          double c = cond(3 * (uint64_t) j + 0, ax);
          A->rowind[ip] = j + 1; A->values.d[ip] = -c; ip++;
          diag[j] += c; diag[j + 1] += c;
        }
        if (y < Y - 1) {
          double c = cond(3 * (uint64_t) j + 1, ay);
          A->rowind[ip] = j + X; A->values.d[ip] = -c; ip++;
          diag[j] += c; diag[j + X] += c;
        }
        if (!two_d && z < Z - 1) {
          double c = cond(3 * (uint64_t) j + 2, az);
          A->rowind[ip] = j + X * Y; A->values.d[ip] = -c; ip++;
          diag[j] += c; diag[j + X * Y] += c;
        }
        const uint64_t fb = 3 * NN + 6 * (uint64_t) j;
        if (x == 0) diag[j] += cond(fb + 0, ax);
        if (x == X - 1) diag[j] += cond(fb + 1, ax);
        if (y == 0) diag[j] += cond(fb + 2, ay);
        if (y == Y - 1) diag[j] += cond(fb + 3, ay);
        if (!two_d) {
          if (z == 0) diag[j] += cond(fb + 4, az);
          if (z == Z - 1) diag[j] += cond(fb + 5, az);
        }
        A->rowind[ip] = j;
        A->values.d[ip] = 0.0;  // filled below once all edges are known
        ip++;
      }
  A->colptr[N] = ip;
  for (int j = 0; j < N; j++) A->values.d[A->colptr[j + 1] - 1] = diag[j];
  return A;
}

const char* taucs_b200_last_error(void) { return tb::last_error(); }

}  // extern "C"

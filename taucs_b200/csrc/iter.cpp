// taucs_conjugate_gradients: the reference's preconditioned conjugate
// gradients driver (src/taucs_iter.c:66-223) with its interface -- host
// vectors, a preconditioner callback such as taucs_supernodal_solve_llt --
// and its iteration: r = b - A x; z = M^-1 r; rho = r.z; p = z (first) or
// z + (rho / (rho_old + tiny)) p; q = A p; alpha = rho / (p.q + tiny);
// x += alpha p; r -= alpha q; stop when ||r||_2 / ||r_0||_2 <= convergetol or
// after itermax + 1 iterations.  The callback is where the work is: with this
// library's factor it is a solve on the GPU.  The vector updates and the
// product with A stay on the host, beside the caller's host vectors, as in
// the reference's interface.
//
// taucs_linsolve reaches it with taucs.solve.cg=true
// (src/taucs_linsolve.c:561-567), one right-hand side at a time, with the
// factor's solve as preconditioner.
#include <cmath>
#include <vector>

#include "internal.h"

using namespace tb;

namespace {

double two_norm(int n, const double* v) {
  double s = 0.0;
  for (int i = 0; i < n; i++) s += v[i] * v[i];
  return std::sqrt(s);
}

double dot(int n, const double* a, const double* b) {
  double s = 0.0;
  for (int i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

}  // namespace

extern "C" int taucs_conjugate_gradients(taucs_ccs_matrix* A, int (*precond_fn)(void*, void* x, void* b),
                                         void* precond_args, void* vX, void* vB, int itermax, double convergetol) {
  if (!A || !vX || !vB || !(A->flags & TAUCS_DOUBLE)) {
    set_error("taucs_conjugate_gradients: bad arguments (double matrices only)");
    return TAUCS_ERROR_BADARGS;
  }
  double* X = (double*) vX;
  const double* B = (const double*) vB;
  const int n = A->n;
  const double tiny = 0.1e-28;   // the reference's guard against a zero denominator
  std::vector<double> P(n), R(n), Q(n), Z(n);
  taucs_ccs_times_vec(A, X, R.data());
  for (int i = 0; i < n; i++) R[i] = B[i] - R[i];
  double res_norm = two_norm(n, R.data()), init_norm = res_norm;
  tprintf("cg: starting residual, 2-norm %.2e\n", init_norm);
  if (init_norm == 0.0) init_norm = 1.0;
  double ratio = 1.0, rho0 = 0.0;
  int iter = 0;
  while (ratio > convergetol && iter <= itermax) {
    iter++;
    if (precond_fn) {
      if (precond_fn(precond_args, Z.data(), R.data()) != 0) {
        set_error("taucs_conjugate_gradients: the preconditioner failed");
        return TAUCS_ERROR;
      }
    } else {
      Z = R;
    }
    const double rho = dot(n, R.data(), Z.data());
    if (iter == 1) {
      P = Z;
    } else {
      const double beta = rho / (rho0 + tiny);
      for (int i = 0; i < n; i++) P[i] = Z[i] + beta * P[i];
    }
    taucs_ccs_times_vec(A, P.data(), Q.data());
    const double alpha = rho / (dot(n, P.data(), Q.data()) + tiny);
    for (int i = 0; i < n; i++) X[i] += alpha * P[i];
    for (int i = 0; i < n; i++) R[i] -= alpha * Q[i];
    rho0 = rho;
    res_norm = two_norm(n, R.data());
    ratio = res_norm / init_norm;
    if (iter % 25 == 0)
      tprintf("cg: iteration %d (n=%d): residual reduced by %.2e, 2-norm %.2e\n", iter, n, ratio, res_norm);
  }
  if (iter > 0) {
    tprintf("cg: stopped after %d iterations (n=%d): residual reduced by %.2e, 2-norm %.2e\n", iter, n, ratio, res_norm);
    taucs_ccs_times_vec(A, X, R.data());
    for (int i = 0; i < n; i++) R[i] = B[i] - R[i];
    tprintf("cg: recomputed residual b - A x, 2-norm %.2e\n", two_norm(n, R.data()));
  }
  return TAUCS_SUCCESS;
}

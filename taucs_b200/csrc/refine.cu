// Mixed precision and iterative refinement (placeholder).
#include "factor.h"

using namespace tb;

extern "C" int taucs_b200_set_precision(void* L, int precision) {
  if (!L || precision != 0) return -1;
  ((Factor*) L)->precision = 0;
  return 0;
}

extern "C" int taucs_b200_solve_refine(void* L, taucs_ccs_matrix* A, int nrhs, double* X, const double* B,
                                       double tol, int maxits, double* res_out) {
  (void) L; (void) A; (void) nrhs; (void) X; (void) B; (void) tol; (void) maxits; (void) res_out;
  return -1;
}

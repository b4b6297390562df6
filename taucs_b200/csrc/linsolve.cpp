// taucs_linsolve: the reference's unified interface (src/taucs_linsolve.c:
// 189-622) over the device factor.  Option syntax and the "=#k" indirection
// into opt_arg follow src/taucs_linsolve.c:41-151; unknown options are
// reported and ignored.  Differences, all on purpose:
//  * the LLT factor is always the multifrontal one (the reference's default
//    is left-looking, :476-486); taucs.factor.ll is accepted and selects it;
//  * all nrhs columns are solved in one multi-RHS device solve instead of a
//    per-column loop (:556-583);
//  * taucs.gpu.precision=mixed factors in FP32 and refines in FP64.
//  * taucs.ooc=true (out-of-core LL^T) gets the same factor, held in device
//    memory, after the reference's checks of its file options.
// LU, MINRES, the orderings other than AMD and GENMMD, and preconditioners
// are outside this library; requesting them returns an error.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "factor.h"

namespace tb {
Factor* symbolic(taucs_ccs_matrix* A, int max_depth);
int numeric_host(Factor* F, taucs_ccs_matrix* A);
int solve_host(Factor* F, int nrhs, double* X, const double* B);
}  // namespace tb

using namespace tb;

namespace {

struct LinsolveFactor {
  int n;
  int flags;
  int* rowperm;
  int* colperm;
  Factor* L;
};

void lf_free(LinsolveFactor* f) {
  if (!f) return;
  if (f->L) taucs_supernodal_factor_free(f->L);
  free(f->rowperm);
  free(f->colperm);
  delete f;
}

// returns 1 if `name` matched and was parsed, 0 otherwise (src/taucs_linsolve.c:41-151)
int opt_match(const char* cmd, const char* name, const char** value, void* args[], int* argi) {
  const size_t lc = strlen(cmd), ln = strlen(name);
  if (strncmp(cmd, name, ln)) return 0;
  if (lc > ln && cmd[ln] == '.') return 0;
  if (lc > ln && cmd[ln] == '=') {
    if (cmd[ln + 1] == '#') {
      unsigned p;
      if (sscanf(cmd + ln + 2, "%u", &p) == 1 && args) {
        for (unsigned i = 0; args[i]; i++)
          if (i == p) { *argi = (int) i; *value = nullptr; return 1; }
        taucs_printf((char*) "taucs: WARNING, pointer argument out of range in [%s]\n", cmd);
      }
      taucs_printf((char*) "taucs: WARNING, illegal pointer argument in [%s]\n", cmd);
      return -1;
    }
    *argi = -1;
    *value = cmd + ln + 1;
    return 1;
  }
  taucs_printf((char*) "taucs: WARNING, illegal argument in [%s]\n", cmd);
  return -1;
}

int get_bool(const char* cmd, const char* name, void* args[], int* x) {
  const char* v;
  int ai;
  int r = opt_match(cmd, name, &v, args, &ai);
  if (r <= 0) return 0;
  if (ai >= 0) { *x = *(int*) args[ai]; return 1; }
  if (!strcmp(v, "true")) { *x = 1; return 1; }
  if (!strcmp(v, "false")) { *x = 0; return 1; }
  taucs_printf((char*) "taucs: WARNING, illegal argument in [%s]\n", cmd);
  return 0;
}

int get_double(const char* cmd, const char* name, void* args[], double* x) {
  const char* v;
  int ai;
  int r = opt_match(cmd, name, &v, args, &ai);
  if (r <= 0) return 0;
  if (ai >= 0) { *x = *(double*) args[ai]; return 1; }
  if (sscanf(v, "%le", x) == 1) return 1;
  taucs_printf((char*) "taucs: WARNING, illegal argument in [%s]\n", cmd);
  return 0;
}

int get_string(const char* cmd, const char* name, void* args[], const char** x) {
  const char* v;
  int ai;
  int r = opt_match(cmd, name, &v, args, &ai);
  if (r <= 0) return 0;
  if (ai >= 0) { *x = *(char**) args[ai]; return 1; }
  *x = v;
  return 1;
}

}  // namespace

extern "C" int taucs_linsolve(taucs_ccs_matrix* A, void** F, int nrhs, void* X, void* B, char* options[],
                              void* opt_arg[]) {
  if (!A && nrhs == 0) {
    if (F) {
      lf_free((LinsolveFactor*) *F);
      *F = nullptr;
    }
    return TAUCS_SUCCESS;
  }
  int opt_factor = 1, opt_symbolic = 1, opt_numeric = 1, opt_llt = 0, opt_lu = 0, opt_mf = 0, opt_ll = 0;
  int opt_ooc = 0, opt_cg = 0, opt_minres = 0;
  double opt_maxdepth = 0.0, opt_tol = 1e-12, opt_maxits = 10.0;
  double opt_cg_maxits = 300.0, opt_convergetol = 1e-6;   // src/taucs_linsolve.c:238-239
  const char* opt_ordering = nullptr;
  const char* opt_precision = "fp64";
  const char* opt_ooc_name = nullptr;
  double opt_ooc_memory = -1.0;
  int opt_ooc_handle = 0;
  if (options) {
    for (int i = 0; options[i]; i++) {
      const char* o = options[i];
      int u = 0;
      u |= get_bool(o, "taucs.factor", opt_arg, &opt_factor);
      u |= get_bool(o, "taucs.factor.symbolic", opt_arg, &opt_symbolic);
      u |= get_bool(o, "taucs.factor.numeric", opt_arg, &opt_numeric);
      u |= get_bool(o, "taucs.factor.LLT", opt_arg, &opt_llt);
      u |= get_bool(o, "taucs.factor.LU", opt_arg, &opt_lu);
      u |= get_bool(o, "taucs.factor.mf", opt_arg, &opt_mf);
      u |= get_bool(o, "taucs.factor.ll", opt_arg, &opt_ll);
      u |= get_string(o, "taucs.factor.ordering", opt_arg, &opt_ordering);
      u |= get_double(o, "taucs.maxdepth", opt_arg, &opt_maxdepth);
      u |= get_bool(o, "taucs.ooc", opt_arg, &opt_ooc);
      u |= get_bool(o, "taucs.solve.cg", opt_arg, &opt_cg);
      u |= get_bool(o, "taucs.solve.minres", opt_arg, &opt_minres);
      u |= get_double(o, "taucs.solve.maxits", opt_arg, &opt_cg_maxits);
      u |= get_double(o, "taucs.solve.convergetol", opt_arg, &opt_convergetol);
      u |= get_string(o, "taucs.ooc.basename", opt_arg, &opt_ooc_name);
      u |= get_double(o, "taucs.ooc.memory", opt_arg, &opt_ooc_memory);
      if (!strncmp(o, "taucs.ooc.iohandle=", 19)) {
        opt_ooc_handle = 1;
        u = 1;
      }
      u |= get_string(o, "taucs.gpu.precision", opt_arg, &opt_precision);
      u |= get_double(o, "taucs.gpu.refine.tol", opt_arg, &opt_tol);
      u |= get_double(o, "taucs.gpu.refine.maxits", opt_arg, &opt_maxits);
      if (!u) taucs_printf((char*) "taucs_linsolve: illegal option [[%s]]\n", o);
    }
  }
  (void) opt_mf;
  (void) opt_ll;
  if (opt_lu || opt_minres) {
    taucs_printf((char*) "taucs_linsolve: LU and MINRES are not provided by this library\n");
    return TAUCS_ERROR_BADARGS;
  }
  (void) opt_ooc_memory;
  if (opt_ooc && opt_factor) {
    // the reference's out-of-core LL^T (src/taucs_linsolve.c:366-402) keeps
    // the factor in a file because it may not fit in memory; here it is the
    // same multifrontal factor held in device memory.  The option checks are
    // the reference's: exactly one of a file name and an I/O handle.
    if ((opt_ooc_name != nullptr) == (opt_ooc_handle != 0)) {
      taucs_printf((char*) "taucs_linsolve: ooc factorization requires exactly one of basename or iohandle\n");
      return TAUCS_ERROR_BADARGS;
    }
    taucs_printf((char*) "taucs_linsolve: taucs.ooc: the LL^T factor is kept in device memory; no out-of-core "
                         "file is written\n");
  }
  const bool mixed = opt_precision && !strcmp(opt_precision, "mixed");

  LinsolveFactor* f = nullptr;
  taucs_ccs_matrix* PAPT = nullptr;
  int retcode = TAUCS_SUCCESS;
  if (opt_factor) {
    if (!A) return TAUCS_ERROR_BADARGS;
    if (!opt_numeric && nrhs > 0) {
      taucs_printf((char*) "taucs_linsolve: WARNING, you can't solve without a numeric factorization\n");
      opt_numeric = 1;
    }
    f = new (std::nothrow) LinsolveFactor();
    if (!f) return TAUCS_ERROR_NOMEM;
    f->n = A->n;
    f->flags = A->flags;
    f->rowperm = f->colperm = nullptr;
    f->L = nullptr;
    // the reference's default for LL^T without METIS (src/taucs_linsolve.c:319-329)
    if (!opt_ordering) opt_ordering = "genmmd";
    taucs_ccs_order(A, &f->rowperm, &f->colperm, (char*) opt_ordering);
    if (!f->rowperm) {
      taucs_printf((char*) "taucs_factor: ordering failed\n");
      lf_free(f);
      return TAUCS_ERROR_NOMEM;
    }
    if (opt_llt) {
      PAPT = taucs_ccs_permute_symmetrically(A, f->rowperm, f->colperm);
      if (!PAPT) { lf_free(f); return TAUCS_ERROR_NOMEM; }
      if (!opt_numeric && opt_symbolic) {
        f->L = symbolic(PAPT, (int) opt_maxdepth);
      } else if (opt_numeric && !opt_symbolic) {
        LinsolveFactor* old = F ? (LinsolveFactor*) *F : nullptr;
        if (!old || !old->L) {
          taucs_printf((char*) "taucs_linsolve: ERROR, you need to provide a symbolic factorization for a numeric factorization\n");
          taucs_ccs_free(PAPT);
          lf_free(f);
          return TAUCS_ERROR_BADARGS;
        }
        // reuse the caller's symbolic factor (its ordering is recomputed
        // identically from the same matrix pattern)
        f->L = old->L;
        old->L = nullptr;
        taucs_supernodal_factor_free_numeric(f->L);
        if (mixed) taucs_b200_set_precision(f->L, 1);
        if (numeric_host(f->L, PAPT)) {
          taucs_supernodal_factor_free(f->L);
          f->L = nullptr;
        }
      } else {
        f->L = symbolic(PAPT, (int) opt_maxdepth);
        if (f->L) {
          if (mixed) taucs_b200_set_precision(f->L, 1);
          if (numeric_host(f->L, PAPT)) {
            taucs_supernodal_factor_free(f->L);
            f->L = nullptr;
          }
        }
      }
      if (!f->L) {
        taucs_printf((char*) "taucs_factor: factorization failed\n");
        taucs_ccs_free(PAPT);
        lf_free(f);
        return TAUCS_ERROR;
      }
    }
  }

  if (nrhs > 0) {
    if (!f) {
      if (!F || !*F) {
        taucs_printf((char*) "taucs_linsolve: can't solve, no factorization\n");
        taucs_ccs_free(PAPT);
        return TAUCS_ERROR;
      }
      f = (LinsolveFactor*) *F;
    }
    if (!f->L) {
      taucs_printf((char*) "taucs_linsolve: I don't know how to solve!\n");
      retcode = TAUCS_ERROR;
    } else {
      const int n = f->n;
      std::vector<double> PB((size_t) n * nrhs), PX((size_t) n * nrhs);
      for (int j = 0; j < nrhs; j++)
        taucs_vec_permute(n, TAUCS_DOUBLE, (double*) B + (size_t) j * n, PB.data() + (size_t) j * n, f->rowperm);
      int rc;
      if (opt_cg) {
        // conjugate gradients preconditioned by the factor, one column at a
        // time (src/taucs_linsolve.c:555-567)
        if (!PAPT) PAPT = taucs_ccs_permute_symmetrically(A, f->rowperm, f->colperm);
        rc = PAPT ? 0 : -1;
        for (int j = 0; j < nrhs && !rc; j++)
          rc = taucs_conjugate_gradients(PAPT, taucs_supernodal_solve_llt, f->L, PX.data() + (size_t) j * n,
                                         PB.data() + (size_t) j * n, (int) opt_cg_maxits, opt_convergetol);
      } else if (f->L->precision == 1 || mixed) {
        if (!PAPT) PAPT = taucs_ccs_permute_symmetrically(A, f->rowperm, f->colperm);
        rc = PAPT ? taucs_b200_solve_refine(f->L, PAPT, nrhs, PX.data(), PB.data(), opt_tol, (int) opt_maxits, nullptr) : -1;
        rc = rc < 0 ? -1 : 0;
      } else {
        rc = solve_host(f->L, nrhs, PX.data(), PB.data());
      }
      if (rc) retcode = TAUCS_ERROR;
      for (int j = 0; j < nrhs; j++)
        taucs_vec_ipermute(n, TAUCS_DOUBLE, PX.data() + (size_t) j * n, (double*) X + (size_t) j * n, f->rowperm);
    }
  }

  taucs_ccs_free(PAPT);
  if (opt_factor) {
    if (F) {
      if (*F && *F != f && ((LinsolveFactor*) *F)->L == nullptr) lf_free((LinsolveFactor*) *F);
      *F = f;
    } else {
      lf_free(f);
    }
  }
  return retcode;
}

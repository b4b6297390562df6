/*
 * ref_driver.c -- test-infrastructure shim linked into oracle/_ref/libtaucs_ref.so
 * next to the UNMODIFIED reference objects.  It only reads what the reference
 * computed; it performs no factorization arithmetic of its own.
 *
 * The reference keeps its supernodal factor type private to
 * src/taucs_sn_llt.c:603-623 (supernodal_factor_matrix), so this file mirrors
 * that layout field for field in order to dump the symbolic structure
 * (sn_size, sn_up_size, sn_struct, first_child/next_child) and the numeric
 * blocks (sn_blocks: s x s column-major ld=s; up_blocks: m x s column-major
 * ld=m) for parity checks.  The layout has to be identical or the dump would
 * read the wrong fields.
 *
 * Used only by tests/, smoke() and bench.py's CPU-baseline leg.
 */
#include <stdlib.h>
#include <string.h>
#include "taucs.h"

/* taucs.h redirects the libc allocator names; this shim frees arrays the
 * reference allocated through its malloc stubs, which are plain libc calls */
#undef malloc
#undef calloc
#undef realloc
#undef free

typedef struct {
  int     flags;
  char    uplo;
  int     n;
  int     n_sn;
  int*    parent;
  int*    first_child;
  int*    next_child;
  int*    sn_size;
  int*    sn_up_size;
  int**   sn_struct;
  int*    sn_blocks_ld;
  double** sn_blocks;
  int*    up_blocks_ld;
  double** up_blocks;
} ref_sn_factor; /* mirror of supernodal_factor_matrix, src/taucs_sn_llt.c:603-623 */

extern int taucs_ccs_etree(taucs_ccs_matrix* A, int* parent, int* l_colcount,
                           int* l_rowcount, int* l_nnz);

/* number of supernode slots (n_sn, including slots emptied by amalgamation)
 * and the matrix order */
int ref_factor_dims(void* vL, int* n, int* n_sn)
{
  ref_sn_factor* L = (ref_sn_factor*) vL;
  if (!L) return -1;
  *n = L->n;
  *n_sn = L->n_sn;
  return 0;
}

/* total length of all sn_struct arrays (sum of sn_up_size) */
long ref_factor_struct_len(void* vL)
{
  ref_sn_factor* L = (ref_sn_factor*) vL;
  long t = 0;
  int sn;
  for (sn = 0; sn < L->n_sn; sn++) t += L->sn_up_size[sn];
  return t;
}

/* Copies the supernodal tree and structure.  first_child/next_child have
 * n_sn+1 entries (index n_sn is the virtual root).  struct_ptr has n_sn+1
 * entries; struct_idx holds the concatenated sn_struct rows. */
int ref_factor_symbolic(void* vL, int* sn_size, int* sn_up_size,
                        int* first_child, int* next_child,
                        long* struct_ptr, int* struct_idx)
{
  ref_sn_factor* L = (ref_sn_factor*) vL;
  int sn;
  long p = 0;
  for (sn = 0; sn < L->n_sn; sn++) {
    sn_size[sn] = L->sn_size[sn];
    sn_up_size[sn] = L->sn_up_size[sn];
  }
  for (sn = 0; sn <= L->n_sn; sn++) {
    first_child[sn] = L->first_child[sn];
    next_child[sn] = L->next_child[sn];
  }
  for (sn = 0; sn < L->n_sn; sn++) {
    struct_ptr[sn] = p;
    if (L->sn_up_size[sn] > 0) {
      memcpy(struct_idx + p, L->sn_struct[sn], sizeof(int) * L->sn_up_size[sn]);
      p += L->sn_up_size[sn];
    }
  }
  struct_ptr[L->n_sn] = p;
  return 0;
}

/* Copies the numeric panel of every supernode into one array laid out as
 * f x s column-major (ld = f = sn_up_size) per supernode, rows in sn_struct
 * order: rows 0..s-1 from sn_blocks (lower triangle valid), rows s..f-1 from
 * up_blocks.  val_ptr (n_sn+1) gets the offsets. */
int ref_factor_values(void* vL, long* val_ptr, double* vals)
{
  ref_sn_factor* L = (ref_sn_factor*) vL;
  int sn, i, j;
  long p = 0;
  for (sn = 0; sn < L->n_sn; sn++) {
    int s = L->sn_size[sn], f = L->sn_up_size[sn], m = f - s;
    val_ptr[sn] = p;
    if (s == 0) continue;
    if (!L->sn_blocks || !L->sn_blocks[sn]) return -1;
    for (j = 0; j < s; j++) {
      for (i = 0; i < s; i++)
        vals[p + (long) j * f + i] = (i >= j) ? L->sn_blocks[sn][(long) j * L->sn_blocks_ld[sn] + i] : 0.0;
      for (i = 0; i < m; i++)
        vals[p + (long) j * f + s + i] = L->up_blocks[sn][(long) j * L->up_blocks_ld[sn] + i];
    }
    p += (long) f * s;
  }
  val_ptr[L->n_sn] = p;
  return 0;
}

/* total number of doubles ref_factor_values writes */
long ref_factor_values_len(void* vL)
{
  ref_sn_factor* L = (ref_sn_factor*) vL;
  long t = 0;
  int sn;
  for (sn = 0; sn < L->n_sn; sn++) t += (long) L->sn_size[sn] * L->sn_up_size[sn];
  return t;
}

/* elimination tree of an (already permuted) lower CCS matrix; parent[n] */
int ref_etree(taucs_ccs_matrix* A, int* parent)
{
  return taucs_ccs_etree(A, parent, NULL, NULL, NULL);
}

/* build a taucs_ccs_matrix view around caller-owned arrays (not freed) */
taucs_ccs_matrix* ref_ccs_wrap(int n, int flags, int* colptr, int* rowind, double* values)
{
  taucs_ccs_matrix* A = (taucs_ccs_matrix*) malloc(sizeof(taucs_ccs_matrix));
  if (!A) return NULL;
  A->n = n; A->m = n; A->flags = flags;
  A->colptr = colptr; A->rowind = rowind; A->values.d = values;
  return A;
}

void ref_ccs_unwrap(taucs_ccs_matrix* A) { free(A); }

/* copy out a reference-allocated CCS matrix (generators, permute) */
int ref_ccs_dims(taucs_ccs_matrix* A, int* n, int* nnz, int* flags)
{
  *n = A->n; *nnz = A->colptr[A->n]; *flags = A->flags;
  return 0;
}

int ref_ccs_copy(taucs_ccs_matrix* A, int* colptr, int* rowind, double* values)
{
  int n = A->n, nnz = A->colptr[n];
  memcpy(colptr, A->colptr, sizeof(int) * (n + 1));
  memcpy(rowind, A->rowind, sizeof(int) * nnz);
  memcpy(values, A->values.d, sizeof(double) * nnz);
  return 0;
}

/* ordering: copies perm/invperm out and frees the reference's arrays */
int ref_order(taucs_ccs_matrix* A, const char* which, int* perm, int* invperm)
{
  int *p = NULL, *ip = NULL;
  taucs_ccs_order(A, &p, &ip, (char*) which);
  if (!p || !ip) return -1;
  memcpy(perm, p, sizeof(int) * A->n);
  memcpy(invperm, ip, sizeof(int) * A->n);
  free(p); free(ip);
  return 0;
}

/* src/taucs_ccs_io.c's Harwell-Boeing reader calls the f2c'd readhb routines
   (external/src/readhb.c), which need libf2c's formatted I/O; the image has
   no libf2c and the oracle reads no HB files.  These stand-ins let the
   reference's binary readers (same file) link; they report failure. */
int ireadhb_(char* f, char* t, int* m, int* n, int* nz) { (void) f; (void) t; (void) m; (void) n; (void) nz; return -1; }
int dreadhb_(char* f, int* m, int* n, int* nz, int* cp, int* ri, taucs_double* v)
{ (void) f; (void) m; (void) n; (void) nz; (void) cp; (void) ri; (void) v; return -1; }

/* the reference's vector reader allocates with taucs_malloc (plain malloc in
   this build) */
void ref_free(void* p) { free(p); }

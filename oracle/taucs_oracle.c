/*
 * taucs_oracle.c -- ORACLE (test infrastructure, not product code).
 *
 * A plain-C, single-threaded restatement of the reference's multifrontal
 * supernodal Cholesky path, used only as the checker by tests/, smoke() and
 * the CPU-baseline leg of bench.py.  Nothing in the product links or calls it.
 * It is pinned against the reference itself (oracle/_ref/libtaucs_ref.so,
 * built from the unmodified sources by oracle/Makefile): symbolic structure
 * must match bit for bit, numeric values to rounding.
 *
 * Algorithms restated (reference file:line):
 *   etree ............ taucs_ccs_etree                    src/taucs_sn_llt.c:3243-3340
 *                      (the etree of a pattern is unique; Liu's ancestor
 *                      algorithm is used here and yields the same parent[])
 *   child lists ...... taucs_ccs_symbolic_elimination     src/taucs_sn_llt.c:3771-3776
 *   depth guard ...... same                               src/taucs_sn_llt.c:3781-3834
 *   fundamental sn ... recursive_symbolic_elimination     src/taucs_sn_llt.c:1377-1517
 *   amalgamation ..... recursive_amalgamate_supernodes    src/taucs_sn_llt.c:1527-1786
 *   numeric .......... recursive_multifrontal_supernodal_factor_llt
 *                                                         src/taucs_sn_llt.c:1829-1977
 *                      extend_add_wrapper                 src/taucs_sn_llt.c:1797-1827
 *                      multifrontal_supernodal_front_factor :1084-1194
 *                      multifrontal_supernodal_front_extend_add :1200-1240
 *   dense kernels .... POTRF/TRSM/SYRK written here as plain loops (the
 *                      reference calls LAPACK/BLAS at :1131, :1150, :1180)
 *   solve ............ recursive_supernodal_solve_l/_lt   src/taucs_sn_llt.c:2596-2841
 *                      taucs_dsupernodal_solve_llt        src/taucs_sn_llt.c:2844-2885
 *   SpMV ............. taucs_dccs_times_vec (symmetric)   src/taucs_ccs_ops.c:299-344
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int n;
  int n_sn;             /* number of supernode slots; the virtual root is n_sn */
  int* sn_size;         /* [n]  columns of each supernode                      */
  int* sn_up_size;      /* [n]  columns + update rows                          */
  int** sn_struct;      /* [n]  row structure, first sn_size entries = columns */
  int* first_child;     /* [n+1]                                               */
  int* next_child;      /* [n+1]                                               */
  double** f1;          /* per supernode: s x s, ld s (lower)                  */
  double** f2;          /* per supernode: m x s, ld m                          */
} orc_factor;

/* ---------------------------------------------------------------- etree */

int orc_etree(int n, const int* colptr, const int* rowind, int* parent)
{
  /* row lists of the strict lower triangle: for each row i, columns j < i */
  int* cnt = (int*) calloc((size_t) n + 1, sizeof(int));
  int* rp = (int*) malloc(sizeof(int) * ((size_t) n + 1));
  int nnz = colptr[n];
  int* ci = (int*) malloc(sizeof(int) * (size_t) (nnz > 0 ? nnz : 1));
  int* anc = (int*) malloc(sizeof(int) * (size_t) (n > 0 ? n : 1));
  int i, j, ip;
  if (!cnt || !rp || !ci || !anc) { free(cnt); free(rp); free(ci); free(anc); return -1; }
  for (j = 0; j < n; j++)
    for (ip = colptr[j]; ip < colptr[j + 1]; ip++)
      if (rowind[ip] > j) cnt[rowind[ip]]++;
  rp[0] = 0;
  for (i = 0; i < n; i++) rp[i + 1] = rp[i] + cnt[i];
  for (i = 0; i < n; i++) cnt[i] = rp[i];
  for (j = 0; j < n; j++)
    for (ip = colptr[j]; ip < colptr[j + 1]; ip++)
      if (rowind[ip] > j) ci[cnt[rowind[ip]]++] = j;
  /* Liu: walk from each k in row i up the partial tree, compressing paths */
  for (i = 0; i < n; i++) {
    parent[i] = n;
    anc[i] = n;
    for (ip = rp[i]; ip < rp[i + 1]; ip++) {
      int k = ci[ip];
      while (k != n && k < i) {
        int next = anc[k];
        anc[k] = i;
        if (next == n) { parent[k] = i; break; }
        k = next;
      }
    }
  }
  free(cnt); free(rp); free(ci); free(anc);
  return 0;
}

/* ------------------------------------------------------ fundamental sn */

typedef struct {
  int n;
  const int* colptr;
  const int* rowind;
  int* first_child;     /* etree children */
  int* next_child;
  int* col2sn;
  int* map;
  int* tmp;
  orc_factor* L;
} sym_ctx;

static int rse(sym_ctx* c, int j)
{
  orc_factor* L = c->L;
  int ch, ip, i, csn, in_prev, nnz = 0;
  for (ch = c->first_child[j]; ch != -1; ch = c->next_child[ch])
    if (rse(c, ch) == -1) return -1;

  in_prev = 1;
  if (j == c->n) in_prev = 0;
  else if (c->first_child[j] == -1) in_prev = 0;
  else if (c->next_child[c->first_child[j]] != -1) in_prev = 0;
  else {
    ch = c->first_child[j];
    for (ip = c->colptr[j]; ip < c->colptr[j + 1]; ip++)
      in_prev = in_prev && (c->map[c->rowind[ip]] == ch);
  }

  if (in_prev) {
    /* column j extends the single child's supernode (chain) */
    ch = c->first_child[j];
    csn = c->col2sn[ch];
    c->col2sn[j] = csn;
    for (ip = L->sn_size[csn]; ip < L->sn_up_size[csn]; ip++)
      if (L->sn_struct[csn][ip] == j) break;
    if (ip >= L->sn_up_size[csn]) return -1;
    L->sn_struct[csn][ip] = L->sn_struct[csn][L->sn_size[csn]];
    L->sn_struct[csn][L->sn_size[csn]] = j;
    for (ip = L->sn_size[csn]; ip < L->sn_up_size[csn]; ip++)
      c->map[L->sn_struct[csn][ip]] = j;
    L->sn_size[csn]++;
    return 0;
  }

  if (j < c->n) {
    nnz = 1;
    c->tmp[0] = j;
    c->map[j] = j;
    for (ch = c->first_child[j]; ch != -1; ch = c->next_child[ch]) {
      csn = c->col2sn[ch];
      for (ip = L->sn_size[csn]; ip < L->sn_up_size[csn]; ip++) {
        i = L->sn_struct[csn][ip];
        if (i > j && c->map[i] != j) { c->map[i] = j; c->tmp[nnz++] = i; }
      }
    }
    for (ip = c->colptr[j]; ip < c->colptr[j + 1]; ip++) {
      i = c->rowind[ip];
      if (c->map[i] != j) { c->map[i] = j; c->tmp[nnz++] = i; }
    }
  }

  /* supernodal children: first etree child first, later ones prepended */
  for (ch = c->first_child[j]; ch != -1; ch = c->next_child[ch]) {
    csn = c->col2sn[ch];
    if (ch == c->first_child[j]) L->first_child[L->n_sn] = csn;
    else { L->next_child[csn] = L->first_child[L->n_sn]; L->first_child[L->n_sn] = csn; }
  }

  if (j < c->n) {
    c->col2sn[j] = L->n_sn;
    L->sn_size[L->n_sn] = 1;
    L->sn_up_size[L->n_sn] = nnz;
    L->sn_struct[L->n_sn] = (int*) malloc(sizeof(int) * (size_t) nnz);
    if (!L->sn_struct[L->n_sn]) return -1;
    memcpy(L->sn_struct[L->n_sn], c->tmp, sizeof(int) * (size_t) nnz);
    L->n_sn++;
  }
  return 0;
}

/* ------------------------------------------------------- amalgamation */

typedef struct { double zeros, nonzeros; } znz;

static znz amalg(sym_ctx* c, int sn)
{
  orc_factor* L = c->L;
  int* ssz = L->sn_size;
  int* sup = L->sn_up_size;
  int i, ip, csn, gsn, nnz, nch, k, new_s, new_f, zn;
  znz me, merged, cz;
  double* zcount;

  me.zeros = 0.0;
  me.nonzeros = (double) (((sup[sn] - ssz[sn]) * ssz[sn]) + (ssz[sn] * (ssz[sn] + 1)) / 2);
  if (L->first_child[sn] == -1) return me;

  merged = me;
  for (csn = L->first_child[sn]; csn != -1; csn = L->next_child[csn]) {
    cz = amalg(c, csn);
    merged.nonzeros += cz.nonzeros;
    merged.zeros += cz.zeros;
  }

  /* merged row list: children's columns, own columns, then new update rows */
  nnz = 0;
  for (csn = L->first_child[sn]; csn != -1; csn = L->next_child[csn])
    for (ip = 0; ip < ssz[csn]; ip++) {
      i = L->sn_struct[csn][ip]; c->map[i] = sn; c->tmp[nnz++] = i;
    }
  for (ip = 0; ip < ssz[sn]; ip++) {
    i = L->sn_struct[sn][ip]; c->map[i] = sn; c->tmp[nnz++] = i;
  }
  new_s = nnz;
  for (csn = L->first_child[sn]; csn != -1; csn = L->next_child[csn])
    for (ip = ssz[csn]; ip < sup[csn]; ip++) {
      i = L->sn_struct[csn][ip];
      if (c->map[i] != sn) { c->map[i] = sn; c->tmp[nnz++] = i; }
    }
  for (ip = ssz[sn]; ip < sup[sn]; ip++) {
    i = L->sn_struct[sn][ip];
    if (c->map[i] != sn) { c->map[i] = sn; c->tmp[nnz++] = i; }
  }
  new_f = nnz;

  /* explicit zeros the merge would introduce, per row */
  zn = 0;
  for (ip = 0; ip < nnz; ip++) if (c->tmp[ip] >= zn) zn = c->tmp[ip] + 1;
  zcount = (double*) malloc(sizeof(double) * (size_t) (zn > 0 ? zn : 1));
  for (ip = 0; ip < new_s; ip++) zcount[c->tmp[ip]] = (double) (ip + 1);
  for (ip = new_s; ip < new_f; ip++) zcount[c->tmp[ip]] = (double) new_s;
  for (csn = L->first_child[sn]; csn != -1; csn = L->next_child[csn]) {
    for (ip = 0; ip < ssz[csn]; ip++) zcount[L->sn_struct[csn][ip]] -= (double) (ip + 1);
    for (ip = ssz[csn]; ip < sup[csn]; ip++) zcount[L->sn_struct[csn][ip]] -= (double) ssz[csn];
  }
  for (ip = 0; ip < ssz[sn]; ip++) zcount[L->sn_struct[sn][ip]] -= (double) (ip + 1);
  for (ip = ssz[sn]; ip < sup[sn]; ip++) zcount[L->sn_struct[sn][ip]] -= (double) ssz[sn];
  for (ip = 0; ip < new_f; ip++) merged.zeros += zcount[c->tmp[ip]];
  free(zcount);

  /* the reference's relaxation thresholds, src/taucs_sn_llt.c:1715-1725 */
  if (!((new_s < 16)
        || ((ssz[sn] < 50) && (merged.zeros < 0.5 * merged.nonzeros))
        || ((ssz[sn] < 250) && (merged.zeros < 0.25 * merged.nonzeros))
        || ((ssz[sn] < 500) && (merged.zeros < 0.10 * merged.nonzeros))
        || (merged.zeros < 0.05 * merged.nonzeros)))
    return me;

  ssz[sn] = new_s;
  sup[sn] = new_f;
  L->sn_struct[sn] = (int*) realloc(L->sn_struct[sn], sizeof(int) * (size_t) new_f);
  memcpy(L->sn_struct[sn], c->tmp, sizeof(int) * (size_t) new_f);

  nch = 0;
  for (csn = L->first_child[sn]; csn != -1; csn = L->next_child[csn]) {
    for (ip = 0; ip < ssz[csn]; ip++) c->col2sn[L->sn_struct[csn][ip]] = sn;
    for (gsn = L->first_child[csn]; gsn != -1; gsn = L->next_child[gsn]) c->tmp[nch++] = gsn;
  }
  for (csn = L->first_child[sn]; csn != -1; csn = L->next_child[csn]) {
    free(L->sn_struct[csn]);
    L->sn_struct[csn] = NULL;
    ssz[csn] = 0;
    sup[csn] = 0;
  }
  L->first_child[sn] = -1;
  for (k = 0; k < nch; k++) {
    L->next_child[c->tmp[k]] = L->first_child[sn];
    L->first_child[sn] = c->tmp[k];
  }
  return merged;
}

void orc_free(void* vL)
{
  orc_factor* L = (orc_factor*) vL;
  int sn;
  if (!L) return;
  for (sn = 0; sn < L->n; sn++) {
    if (L->sn_struct) free(L->sn_struct[sn]);
    if (L->f1) free(L->f1[sn]);
    if (L->f2) free(L->f2[sn]);
  }
  free(L->sn_struct); free(L->f1); free(L->f2);
  free(L->sn_size); free(L->sn_up_size); free(L->first_child); free(L->next_child);
  free(L);
}

/* symbolic analysis of an already permuted lower CCS pattern; NULL on failure
 * or when max_depth > 0 and the etree is deeper (src/taucs_sn_llt.c:3817) */
void* orc_analyze(int n, const int* colptr, const int* rowind, int max_depth)
{
  orc_factor* L = (orc_factor*) calloc(1, sizeof(orc_factor));
  sym_ctx c;
  int* parent = (int*) malloc(sizeof(int) * ((size_t) n + 1));
  int j, depth, *lvl, *nxt, cnt, ncnt;
  if (!L || !parent) { free(L); free(parent); return NULL; }
  L->n = n;
  L->sn_size = (int*) malloc(sizeof(int) * ((size_t) n + 1));
  L->sn_up_size = (int*) malloc(sizeof(int) * ((size_t) n + 1));
  L->sn_struct = (int**) calloc((size_t) n + 1, sizeof(int*));
  L->first_child = (int*) malloc(sizeof(int) * ((size_t) n + 1));
  L->next_child = (int*) malloc(sizeof(int) * ((size_t) n + 1));
  c.n = n; c.colptr = colptr; c.rowind = rowind; c.L = L;
  c.first_child = (int*) malloc(sizeof(int) * ((size_t) n + 1));
  c.next_child = (int*) malloc(sizeof(int) * ((size_t) n + 1));
  c.col2sn = (int*) malloc(sizeof(int) * ((size_t) n + 1));
  c.map = (int*) malloc(sizeof(int) * ((size_t) n + 1));
  c.tmp = (int*) malloc(sizeof(int) * ((size_t) n + 1));
  if (orc_etree(n, colptr, rowind, parent)) { orc_free(L); free(parent); return NULL; }
  for (j = 0; j <= n; j++) c.first_child[j] = -1;
  for (j = n - 1; j >= 0; j--) { c.next_child[j] = c.first_child[parent[j]]; c.first_child[parent[j]] = j; }

  /* breadth-first depth of the etree below the virtual root */
  lvl = c.tmp; nxt = c.map;
  lvl[0] = n; cnt = 1; depth = -1;
  while (cnt) {
    int ch, k;
    ncnt = 0;
    for (k = 0; k < cnt; k++)
      for (ch = c.first_child[lvl[k]]; ch != -1; ch = c.next_child[ch]) nxt[ncnt++] = ch;
    { int* t = lvl; lvl = nxt; nxt = t; }
    cnt = ncnt;
    depth++;
  }
  if (max_depth && depth > max_depth) {
    free(c.first_child); free(c.next_child); free(c.col2sn); free(c.map); free(c.tmp);
    free(parent); orc_free(L); return NULL;
  }

  L->n_sn = 0;
  for (j = 0; j < n; j++) c.map[j] = -1;
  for (j = 0; j <= n; j++) L->first_child[j] = L->next_child[j] = -1;
  if (rse(&c, n) == -1) {
    free(c.first_child); free(c.next_child); free(c.col2sn); free(c.map); free(c.tmp);
    free(parent); orc_free(L); return NULL;
  }
  for (j = 0; j < n; j++) c.map[j] = -1;
  if (L->n_sn > 0) (void) amalg(&c, L->n_sn - 1);

  free(c.first_child); free(c.next_child); free(c.col2sn); free(c.map); free(c.tmp);
  free(parent);
  L->f1 = (double**) calloc((size_t) n + 1, sizeof(double*));
  L->f2 = (double**) calloc((size_t) n + 1, sizeof(double*));
  return L;
}

int orc_dims(void* vL, int* n, int* n_sn, long* struct_len, long* values_len)
{
  orc_factor* L = (orc_factor*) vL;
  long t = 0, v = 0;
  int sn;
  for (sn = 0; sn < L->n_sn; sn++) {
    t += L->sn_up_size[sn];
    v += (long) L->sn_size[sn] * L->sn_up_size[sn];
  }
  *n = L->n; *n_sn = L->n_sn; *struct_len = t; *values_len = v;
  return 0;
}

int orc_symbolic_copy(void* vL, int* sn_size, int* sn_up_size, int* first_child,
                      int* next_child, long* struct_ptr, int* struct_idx)
{
  orc_factor* L = (orc_factor*) vL;
  int sn;
  long p = 0;
  for (sn = 0; sn < L->n_sn; sn++) { sn_size[sn] = L->sn_size[sn]; sn_up_size[sn] = L->sn_up_size[sn]; }
  for (sn = 0; sn <= L->n_sn; sn++) { first_child[sn] = L->first_child[sn]; next_child[sn] = L->next_child[sn]; }
  for (sn = 0; sn < L->n_sn; sn++) {
    struct_ptr[sn] = p;
    if (L->sn_up_size[sn]) memcpy(struct_idx + p, L->sn_struct[sn], sizeof(int) * (size_t) L->sn_up_size[sn]);
    p += L->sn_up_size[sn];
  }
  struct_ptr[L->n_sn] = p;
  return 0;
}

/* ------------------------------------------------------------ numeric */

typedef struct { int s, m; double *f1, *f2, *u; } front;

typedef struct {
  orc_factor* L;
  const int* colptr;
  const int* rowind;
  const double* val;
  int* bitmap;
  int fail;
} num_ctx;

static void front_free(front* F)
{
  if (!F) return;
  free(F->f1); free(F->f2); free(F->u); free(F);
}

static front* front_create(int s, int f)
{
  front* F = (front*) calloc(1, sizeof(front));
  if (!F) return NULL;
  F->s = s; F->m = f - s;
  if (s) F->f1 = (double*) calloc((size_t) s * s, sizeof(double));
  if (s && F->m) F->f2 = (double*) calloc((size_t) F->m * s, sizeof(double));
  if (F->m) F->u = (double*) calloc((size_t) F->m * F->m, sizeof(double));
  if ((s && !F->f1) || (s && F->m && !F->f2) || (F->m && !F->u)) { front_free(F); return NULL; }
  return F;
}

static void extend_add(num_ctx* c, int psn, front* P, int csn, front* C)
{
  orc_factor* L = c->L;
  int* ps = L->sn_struct[psn];
  int* cu = L->sn_struct[csn] + C->s;
  int i, j, pi, pj;
  for (i = 0; i < P->s; i++) c->bitmap[ps[i]] = i;
  for (i = 0; i < P->m; i++) c->bitmap[ps[P->s + i]] = P->s + i;
  for (j = 0; j < C->m; j++)
    for (i = j; i < C->m; i++) {
      double v = C->u[(size_t) C->m * j + i];
      pj = c->bitmap[cu[j]];
      pi = c->bitmap[cu[i]];
      if (pj > pi) { int t = pj; pj = pi; pi = t; }
      if (pj < P->s) {
        if (pi < P->s) P->f1[(size_t) P->s * pj + pi] += v;
        else P->f2[(size_t) P->m * pj + (pi - P->s)] += v;
      } else {
        P->u[(size_t) P->m * (pj - P->s) + (pi - P->s)] += v;
      }
    }
}

/* lower Cholesky in place, s x s ld s; returns 0 or the 1-based failing column */
static int dense_potrf(int s, double* a)
{
  int i, j, k;
  for (j = 0; j < s; j++) {
    double* cj = a + (size_t) s * j;
    double d;
    for (k = 0; k < j; k++) {
      const double* ck = a + (size_t) s * k;
      double ajk = ck[j];
      for (i = j; i < s; i++) cj[i] -= ck[i] * ajk;
    }
    d = cj[j];
    if (!(d > 0.0)) return j + 1;
    d = sqrt(d);
    cj[j] = d;
    for (i = j + 1; i < s; i++) cj[i] /= d;
  }
  return 0;
}

/* X := X * L^-T, X m x s ld m, L s x s ld s lower */
static void dense_trsm_rlt(int m, int s, const double* l, double* x)
{
  int r, j, k;
  for (j = 0; j < s; j++) {
    double* xj = x + (size_t) m * j;
    double d;
    for (k = 0; k < j; k++) {
      const double* xk = x + (size_t) m * k;
      double ljk = l[(size_t) s * k + j];
      for (r = 0; r < m; r++) xj[r] -= xk[r] * ljk;
    }
    d = l[(size_t) s * j + j];
    for (r = 0; r < m; r++) xj[r] /= d;
  }
}

/* U := U - X X^T (lower), X m x s ld m, U m x m ld m */
static void dense_syrk_ln(int m, int s, const double* x, double* u)
{
  int i, j, k;
  for (j = 0; j < m; j++) {
    double* uj = u + (size_t) m * j;
    for (k = 0; k < s; k++) {
      const double* xk = x + (size_t) m * k;
      double a = xk[j];
      for (i = j; i < m; i++) uj[i] -= xk[i] * a;
    }
  }
}

static int front_factor(num_ctx* c, int sn, front* F)
{
  orc_factor* L = c->L;
  int* st = L->sn_struct[sn];
  int i, j, ip, info;
  for (i = 0; i < F->s; i++) c->bitmap[st[i]] = i;
  for (i = 0; i < F->m; i++) c->bitmap[st[F->s + i]] = F->s + i;
  for (j = 0; j < F->s; j++) {
    int col = st[j];
    for (ip = c->colptr[col]; ip < c->colptr[col + 1]; ip++) {
      int r = c->bitmap[c->rowind[ip]];
      if (r < F->s) F->f1[(size_t) F->s * j + r] += c->val[ip];
      else F->f2[(size_t) F->m * j + (r - F->s)] += c->val[ip];
    }
  }
  if (F->s) {
    info = dense_potrf(F->s, F->f1);
    if (info) return -1;
  }
  if (F->m && F->s) dense_trsm_rlt(F->m, F->s, F->f1, F->f2);
  L->f1[sn] = F->f1;
  L->f2[sn] = F->f2;
  if (F->m && F->s) dense_syrk_ln(F->m, F->s, F->f2, F->u);
  F->f1 = NULL;
  F->f2 = NULL;
  return 0;
}

static front* mf(num_ctx* c, int sn, int is_root)
{
  orc_factor* L = c->L;
  front* me = NULL;
  int ch;
  for (ch = L->first_child[sn]; ch != -1; ch = L->next_child[ch]) {
    front* cf = mf(c, ch, 0);
    if (c->fail) { front_free(cf); front_free(me); return NULL; }
    if (!is_root) {
      if (!me) {
        me = front_create(L->sn_size[sn], L->sn_up_size[sn]);
        if (!me) { c->fail = 1; front_free(cf); return NULL; }
      }
      extend_add(c, sn, me, ch, cf);
    }
    front_free(cf);
  }
  if (is_root) return NULL;
  if (!me) {
    me = front_create(L->sn_size[sn], L->sn_up_size[sn]);
    if (!me) { c->fail = 1; return NULL; }
  }
  if (front_factor(c, sn, me)) { c->fail = 1; front_free(me); return NULL; }
  return me;
}

/* numeric factorization of the permuted lower CCS matrix on the analyzed
 * pattern; 0 on success, -1 on a nonpositive pivot or out of memory */
int orc_numeric(void* vL, const int* colptr, const int* rowind, const double* val)
{
  orc_factor* L = (orc_factor*) vL;
  num_ctx c;
  int sn;
  for (sn = 0; sn < L->n; sn++) {
    free(L->f1[sn]); free(L->f2[sn]);
    L->f1[sn] = L->f2[sn] = NULL;
  }
  c.L = L; c.colptr = colptr; c.rowind = rowind; c.val = val; c.fail = 0;
  c.bitmap = (int*) malloc(sizeof(int) * ((size_t) L->n + 1));
  if (!c.bitmap) return -1;
  (void) mf(&c, L->n_sn, 1);
  free(c.bitmap);
  if (c.fail) {
    for (sn = 0; sn < L->n; sn++) {
      free(L->f1[sn]); free(L->f2[sn]);
      L->f1[sn] = L->f2[sn] = NULL;
    }
    return -1;
  }
  return 0;
}

/* panels as f x s column-major per supernode (rows in sn_struct order) */
int orc_values(void* vL, long* val_ptr, double* vals)
{
  orc_factor* L = (orc_factor*) vL;
  int sn, i, j;
  long p = 0;
  for (sn = 0; sn < L->n_sn; sn++) {
    int s = L->sn_size[sn], f = L->sn_up_size[sn], m = f - s;
    val_ptr[sn] = p;
    if (!s) continue;
    if (!L->f1[sn]) return -1;
    for (j = 0; j < s; j++) {
      for (i = 0; i < s; i++) vals[p + (long) j * f + i] = i >= j ? L->f1[sn][(size_t) s * j + i] : 0.0;
      for (i = 0; i < m; i++) vals[p + (long) j * f + s + i] = L->f2[sn][(size_t) m * j + i];
    }
    p += (long) f * s;
  }
  val_ptr[L->n_sn] = p;
  return 0;
}

/* -------------------------------------------------------------- solve */

static void solve_l(orc_factor* L, int sn, int is_root, double* x, double* b, double* t)
{
  int ch, i, j, k;
  for (ch = L->first_child[sn]; ch != -1; ch = L->next_child[ch]) solve_l(L, ch, 0, x, b, t);
  if (!is_root) {
    int s = L->sn_size[sn], m = L->sn_up_size[sn] - s;
    int* st = L->sn_struct[sn];
    double* xd = t;
    double* bd = t + s;
    for (i = 0; i < s; i++) xd[i] = b[st[i]];
    for (i = 0; i < m; i++) bd[i] = 0.0;
    for (j = 0; j < s; j++) {
      xd[j] /= L->f1[sn][(size_t) s * j + j];
      for (i = j + 1; i < s; i++) xd[i] -= L->f1[sn][(size_t) s * j + i] * xd[j];
    }
    for (k = 0; k < s; k++)
      for (i = 0; i < m; i++) bd[i] += L->f2[sn][(size_t) m * k + i] * xd[k];
    for (i = 0; i < s; i++) x[st[i]] = xd[i];
    for (i = 0; i < m; i++) b[st[s + i]] -= bd[i];
  }
}

static void solve_lt(orc_factor* L, int sn, int is_root, double* x, double* b, double* t)
{
  int ch, i, j;
  if (!is_root) {
    int s = L->sn_size[sn], m = L->sn_up_size[sn] - s;
    int* st = L->sn_struct[sn];
    double* bd = t;
    double* xd = t + s;
    for (i = 0; i < s; i++) bd[i] = b[st[i]];
    for (i = 0; i < m; i++) xd[i] = x[st[s + i]];
    for (j = 0; j < s; j++) {
      double acc = 0.0;
      for (i = 0; i < m; i++) acc += L->f2[sn][(size_t) m * j + i] * xd[i];
      bd[j] -= acc;
    }
    for (j = s - 1; j >= 0; j--) {
      double acc = bd[j];
      for (i = j + 1; i < s; i++) acc -= L->f1[sn][(size_t) s * j + i] * bd[i];
      bd[j] = acc / L->f1[sn][(size_t) s * j + j];
    }
    for (i = 0; i < s; i++) x[st[i]] = bd[i];
  }
  for (ch = L->first_child[sn]; ch != -1; ch = L->next_child[ch]) solve_lt(L, ch, 0, x, b, t);
}

/* x := L^-T L^-1 b (permuted order, one right-hand side) */
int orc_solve(void* vL, double* x, const double* b)
{
  orc_factor* L = (orc_factor*) vL;
  int n = L->n, i;
  double* y = (double*) malloc(sizeof(double) * ((size_t) n + 1));
  double* t = (double*) malloc(sizeof(double) * ((size_t) n + 1));
  if (!y || !t) { free(y); free(t); return -1; }
  for (i = 0; i < n; i++) x[i] = b[i];
  solve_l(L, L->n_sn, 1, y, x, t);
  solve_lt(L, L->n_sn, 1, x, y, t);
  free(y); free(t);
  return 0;
}

/* ---------------------------------------------------------------- SpMV */

/* y := A x with A symmetric, lower triangle stored (src/taucs_ccs_ops.c:313-323) */
void orc_spmv_sym_lower(int n, const int* colptr, const int* rowind, const double* val,
                        const double* x, double* y)
{
  int i, j, ip;
  for (i = 0; i < n; i++) y[i] = 0.0;
  for (j = 0; j < n; j++)
    for (ip = colptr[j]; ip < colptr[j + 1]; ip++) {
      i = rowind[ip];
      y[i] += x[j] * val[ip];
      if (i != j) y[j] += x[i] * val[ip];
    }
}

/* ----------------------------------------------- lognormal operator inputs */

/* The seeded lognormal-coefficient 7-point (or, Z == 0, 5-point) operator the
 * benchmarks factor.  The reference has no generator for it, so this is a
 * second, independent statement of the input generator of the product
 * library (taucs_b200_generate_lognormal), kept here so that a process that
 * times the reference can build its inputs without loading the product:
 * per-edge conductance scale * exp(sigma * N(0,1)), N(0,1) by Box-Muller on
 * two splitmix64-hashed uniforms of the edge's stream id; off-diagonal -c,
 * the diagonal accumulates c (and the Dirichlet boundary faces' conductances);
 * lower CCS in the row order of taucs_ccs_generate_mesh3d
 * (src/taucs_ccs_generators.c:197-261).  The arrays hold at least X*Y*Z + 1
 * column pointers and (Z == 0 ? 3 : 4) * X*Y*Z entries; returns the entry
 * count, or -1 for bad sizes. */
static unsigned long long orc_splitmix64(unsigned long long x)
{
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

static double orc_cond(unsigned long long seed, unsigned long long k, double sigma, double scale)
{
  unsigned long long a = orc_splitmix64(seed ^ (2 * k));
  unsigned long long b = orc_splitmix64(seed ^ (2 * k + 1) ^ 0xD1B54A32D192ED03ull);
  double u1 = ((double) (a >> 11) + 1.0) * (1.0 / 9007199254740992.0);
  double u2 = (double) (b >> 11) * (1.0 / 9007199254740992.0);
  double g = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
  return scale * exp(sigma * g);
}

long orc_generate_lognormal(int X, int Y, int Z, double sigma, double ax, double ay, double az,
                            unsigned long long seed, int* colptr, int* rowind, double* val)
{
  int two_d = (Z == 0), x, y, z, j, N, ip = 0;
  unsigned long long NN, fb;
  double* diag;
  if (two_d) Z = 1;
  if (X <= 0 || Y <= 0 || Z <= 0) return -1;
  N = X * Y * Z;
  NN = (unsigned long long) N;
  diag = (double*) calloc((size_t) N, sizeof(double));
  if (!diag) return -1;
  for (z = 0; z < Z; z++)
    for (y = 0; y < Y; y++)
      for (x = 0; x < X; x++) {
        double c;
        j = z * X * Y + y * X + x;
        colptr[j] = ip;
        if (x < X - 1) {
          c = orc_cond(seed, 3 * (unsigned long long) j + 0, sigma, ax);
          rowind[ip] = j + 1; val[ip] = -c; ip++;
          diag[j] += c; diag[j + 1] += c;
        }
        if (y < Y - 1) {
          c = orc_cond(seed, 3 * (unsigned long long) j + 1, sigma, ay);
          rowind[ip] = j + X; val[ip] = -c; ip++;
          diag[j] += c; diag[j + X] += c;
        }
        if (!two_d && z < Z - 1) {
          c = orc_cond(seed, 3 * (unsigned long long) j + 2, sigma, az);
          rowind[ip] = j + X * Y; val[ip] = -c; ip++;
          diag[j] += c; diag[j + X * Y] += c;
        }
        fb = 3 * NN + 6 * (unsigned long long) j;
        if (x == 0) diag[j] += orc_cond(seed, fb + 0, sigma, ax);
        if (x == X - 1) diag[j] += orc_cond(seed, fb + 1, sigma, ax);
        if (y == 0) diag[j] += orc_cond(seed, fb + 2, sigma, ay);
        if (y == Y - 1) diag[j] += orc_cond(seed, fb + 3, sigma, ay);
        if (!two_d) {
          if (z == 0) diag[j] += orc_cond(seed, fb + 4, sigma, az);
          if (z == Z - 1) diag[j] += orc_cond(seed, fb + 5, sigma, az);
        }
        rowind[ip] = j;
        val[ip] = 0.0;
        ip++;
      }
  colptr[N] = ip;
  for (j = 0; j < N; j++) val[colptr[j + 1] - 1] = diag[j];
  free(diag);
  return ip;
}

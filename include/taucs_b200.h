/*
 * taucs_b200.h -- C ABI of libtaucs_b200.so, a B200 (sm_100a) implementation
 * of TAUCS's multifrontal supernodal Cholesky factorization and supernodal
 * triangular solve.
 *
 * The first part of this header repeats the reference's public interface for
 * this path with the same names, argument meanings, ownership and error
 * returns, so that a C caller of TAUCS can relink against this library:
 *
 *   taucs_ccs_matrix ............ src/taucs.h:537-554
 *   error codes / flags ......... src/taucs.h:90-108
 *   factor / solve / free ....... src/taucs_private.h:222-257
 *   taucs_linsolve .............. src/taucs_private.h:16-22
 *   CCS helpers ................. src/taucs_private.h:44-73
 *   ordering .................... src/taucs_private.h:97-101
 *   generators .................. src/taucs_private.h:145-147
 *   vector permutes ............. src/taucs_private.h:270-273
 *   logging / timers ............ src/taucs_private.h:280-285
 *
 * The numeric factorization and the solve run on the current CUDA device; the
 * factor handle keeps its L factor in device memory.  Host arrays passed to
 * these functions are ordinary (pageable or pinned) host memory.  There is no
 * CPU fallback: when no usable sm_100 device is present the factor functions
 * return NULL / TAUCS_ERROR and report the CUDA error through taucs_printf.
 *
 * The second part (taucs_b200_*) adds what the reference does not have:
 * device-pointer entry points, multi-RHS solves, stream selection, mixed
 * precision with iterative refinement, batched factorization of many small
 * systems, and inspection hooks used by the parity tests.
 */
#ifndef TAUCS_B200_H
#define TAUCS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* reference interface                                                 */
/* ------------------------------------------------------------------ */

#define TAUCS_SUCCESS           0
#define TAUCS_ERROR            -1
#define TAUCS_ERROR_NOMEM      -2
#define TAUCS_ERROR_BADARGS    -3
#define TAUCS_ERROR_INDEFINITE -4
#define TAUCS_ERROR_MAXDEPTH   -5

#define TAUCS_INT       1024
#define TAUCS_DOUBLE    2048
#define TAUCS_SINGLE    4096
#define TAUCS_DCOMPLEX  8192
#define TAUCS_SCOMPLEX 16384

#define TAUCS_LOWER      1
#define TAUCS_UPPER      2
#define TAUCS_TRIANGULAR 4
#define TAUCS_SYMMETRIC  8
#define TAUCS_HERMITIAN  16
#define TAUCS_PATTERN    32

/* Sparse matrix in compressed column storage, 0-based (src/taucs.h:537-554).
 * Symmetric matrices store the lower triangle including the diagonal; row
 * indices within a column need not be sorted and duplicates are summed. */
typedef struct {
  int  n;       /* columns */
  int  m;       /* rows */
  int  flags;
  int* colptr;  /* n+1 */
  int* rowind;  /* colptr[n] */
  union {
    void*   v;
    double* d;
    float*  s;
  } values;
} taucs_ccs_matrix;

/* CCS helpers (src/taucs_ccs_base.c:72-132, src/taucs_ccs_ops.c:174-344) */
taucs_ccs_matrix* taucs_ccs_create(int m, int n, int nnz, int flags);
taucs_ccs_matrix* taucs_dccs_create(int m, int n, int nnz);
void              taucs_ccs_free(taucs_ccs_matrix* A);
void              taucs_dccs_free(taucs_ccs_matrix* A);
taucs_ccs_matrix* taucs_ccs_permute_symmetrically(taucs_ccs_matrix* A, int* perm, int* invperm);
taucs_ccs_matrix* taucs_dccs_permute_symmetrically(taucs_ccs_matrix* A, int* perm, int* invperm);
void              taucs_ccs_times_vec(taucs_ccs_matrix* A, void* X, void* B);
void              taucs_dccs_times_vec(taucs_ccs_matrix* A, double* X, double* B);

/* binary files (src/taucs_ccs_io.c:31-113, :966-1052; matrix writer after
 * matlab/taucs_ccs_write_binary.m): int nrows, ncols, flags; int
 * colptr[ncols+1]; int rowind[nnz]; values[nnz], native byte order; vectors
 * are n raw values.  Double and single values.  Unlike the reference, the
 * readers return NULL on a missing, short or malformed file (decreasing
 * colptr, row index out of range) instead of asserting or reading garbage. */
taucs_ccs_matrix* taucs_ccs_read_binary(char* filename);
int               taucs_b200_ccs_write_binary(taucs_ccs_matrix* A, char* filename);
void*             taucs_vec_read_binary(int n, int flags, char* filename);
int               taucs_vec_write_binary(int n, int flags, void* v, char* filename);

/* vector permutes (src/taucs_vec_base.c:194-206): pv[i] = v[p[i]];
 * v[invp[i]] = pv[i] */
void taucs_vec_permute(int n, int flags, void* v, void* pv, int p[]);
void taucs_vec_ipermute(int n, int flags, void* pv, void* v, int invp[]);
void taucs_dvec_permute(int n, double v[], double pv[], int p[]);
/* axpby = a x + b y, and the 2-norm (src/taucs_vec_base.c:29-92) */
void   taucs_vec_axpby(int n, int flags, double a, void* x, double b, void* y, void* axpby);
double taucs_vec_norm2(int n, int flags, void* x);
void taucs_dvec_ipermute(int n, double pv[], double v[], int invp[]);

/* generators (src/taucs_ccs_generators.c:89-261) */
taucs_ccs_matrix* taucs_ccs_generate_mesh2d(int n, char* which);
taucs_ccs_matrix* taucs_ccs_generate_mesh3d(int X, int Y, int Z);

/* fill-reducing ordering (src/taucs_ccs_order.c:843-880): "amd", "identity",
 * "random" (and "genmmd"/"metis"/"colamd" report failure).  perm and invperm
 * are allocated with malloc; *perm == NULL on failure. */
void taucs_ccs_order(taucs_ccs_matrix* A, int** perm, int** invperm, char* which);

/* multifrontal supernodal LL^T (src/taucs_private.h:245-257).  A is the
 * already permuted lower triangle.  The handle's first member is int flags
 * (TAUCS_DOUBLE), as in the reference.  NULL on a nonpositive pivot, out of
 * memory (host or device), or an elimination tree deeper than max_depth. */
void* taucs_ccs_factor_llt_mf(taucs_ccs_matrix* A);
void* taucs_ccs_factor_llt_mf_maxdepth(taucs_ccs_matrix* A, int max_depth);
void* taucs_ccs_factor_llt_symbolic(taucs_ccs_matrix* A);
void* taucs_ccs_factor_llt_symbolic_maxdepth(taucs_ccs_matrix* A, int max_depth);
/* 0, or -1 on a nonpositive pivot (numeric part freed) */
int   taucs_ccs_factor_llt_numeric(taucs_ccs_matrix* A, void* L);
void* taucs_dccs_factor_llt_mf(taucs_ccs_matrix* A);
void* taucs_dccs_factor_llt_mf_maxdepth(taucs_ccs_matrix* A, int max_depth);
void* taucs_dccs_factor_llt_symbolic(taucs_ccs_matrix* A);
void* taucs_dccs_factor_llt_symbolic_maxdepth(taucs_ccs_matrix* A, int max_depth);
int   taucs_dccs_factor_llt_numeric(taucs_ccs_matrix* A, void* L);

/* x := (L L^T)^-1 b, one right-hand side, host vectors in permuted order.
 * b is read only.  0, or -1 on failure. */
int   taucs_supernodal_solve_llt(void* L, void* x, void* b);
int   taucs_dsupernodal_solve_llt(void* L, void* x, void* b);

void  taucs_supernodal_factor_free(void* L);
void  taucs_supernodal_factor_free_numeric(void* L);
taucs_ccs_matrix* taucs_supernodal_factor_to_ccs(void* L);
void* taucs_supernodal_factor_get_diag(void* L);
void  taucs_dsupernodal_factor_free(void* L);
void  taucs_dsupernodal_factor_free_numeric(void* L);
taucs_ccs_matrix* taucs_dsupernodal_factor_to_ccs(void* L);
double* taucs_dsupernodal_factor_get_diag(void* L);

/* preconditioned conjugate gradients (src/taucs_iter.c:66-223): host
 * vectors, precond_fn(precond_args, z, r) computes z = M^-1 r (NULL: none),
 * e.g. taucs_supernodal_solve_llt with a factor; stops when the recursively
 * updated residual has shrunk by convergetol in the 2-norm, or after
 * itermax + 1 iterations.  X holds the starting guess on entry.  0, or an
 * error code when the preconditioner fails. */
int taucs_conjugate_gradients(taucs_ccs_matrix* A, int (*precond_fn)(void*, void* x, void* b), void* precond_args,
                              void* X, void* B, int itermax, double convergetol);

/* unified interface (src/taucs_linsolve.c:189-622).  Options understood:
 *   taucs.factor=bool taucs.factor.symbolic=bool taucs.factor.numeric=bool
 *   taucs.factor.LLT=bool taucs.factor.mf=bool taucs.factor.ll=bool
 *   taucs.factor.ordering=string taucs.maxdepth=number
 *   taucs.solve.cg=bool taucs.solve.maxits=number taucs.solve.convergetol=number
 *     (conjugate gradients preconditioned by the factor, one column at a
 *     time, defaults 300 and 1e-6 as in the reference; the starting guess is
 *     zero, where the reference passes uninitialised memory)
 * plus the additions
 *   taucs.gpu.precision=fp64|mixed   (mixed: FP32 fronts + FP64 refinement)
 *   taucs.gpu.refine.tol=number      (scaled residual target, default 1e-12)
 *   taucs.gpu.refine.maxits=number   (default 10)
 * Values may be written as "=#k" to take opt_arg[k].  Unknown options are
 * reported through taucs_printf and ignored, as in the reference.  The LLT
 * factor is always the multifrontal one here (taucs.factor.ll selects it too).
 * All nrhs columns are solved together. */
int taucs_linsolve(taucs_ccs_matrix* A, void** F, int nrhs, void* X, void* B,
                   char* options[], void* opt_arg[]);

/* logging and timers (src/taucs_logging.c:32-80, src/taucs_timer.c:250-290) */
void   taucs_logfile(char* file_prefix);
int    taucs_printf(char* fmt, ...);
double taucs_wtime(void);
double taucs_ctime(void);

/* ------------------------------------------------------------------ */
/* B200 additions (no counterpart in the reference)                    */
/* ------------------------------------------------------------------ */

/* Stream used by the calling thread's subsequent taucs_* / taucs_b200_*
 * calls (a cudaStream_t; NULL = the legacy default stream). */
int taucs_b200_set_stream(void* cuda_stream);

/* Numeric factorization from DEVICE values (nnz doubles in the order of the
 * matrix the handle was analysed with).  Asynchronous on the current stream
 * except for the final status read; returns 0 or -1 (nonpositive pivot). */
int taucs_b200_factor_numeric_device(void* L, const double* d_values);

/* Same as taucs_ccs_factor_llt_numeric but returns without the final status
 * read: the status is read by the next call to taucs_b200_factor_status. */
int taucs_b200_factor_numeric_device_async(void* L, const double* d_values);
int taucs_b200_factor_status(void* L);

/* nrhs right-hand sides, column-major n x nrhs with leading dimension ld, on
 * the DEVICE, permuted order.  X may alias B. */
int taucs_b200_solve_device(void* L, int nrhs, double* d_X, const double* d_B, int ld);

/* No counterpart in the reference.  The same device solve for callers that
 * must not allocate device memory: serving threads that live inside a fixed,
 * pre-reserved memory budget they may not grow, latency-critical threads
 * that may not call cudaMalloc/cudaFree (which can synchronise the device
 * and stall other streams), and hosts whose own caching allocator already
 * holds the rest of the GPU's memory.  Work vectors, handshake flags and the
 * status word live in one static device array of this library (32 MiB of
 * work vectors + 16384 flags; every GPU that loads the library holds it
 * until exit), so the call allocates nothing; factors needing more work
 * space are rejected with -1 and a message in taucs_b200_last_error(), and
 * so is a call made while another device than the factor's is current.
 * Right-hand sides are solved one per pass.  The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress) and sets the solve
 * kernels' shared-memory limits on that device, so make that first call
 * before any stream capture.  All calls share the array: calls whose work
 * overlaps on the GPU (different streams, or different host threads on one
 * device) race and must be serialised by the caller.  Asynchronous on the
 * current stream. */
int taucs_b200_solve_device_noalloc(void* L, int nrhs, double* d_X, const double* d_B, int ld);
/* Status of the no-alloc solves on the current device: waits for the current
 * stream, then returns 0, or -1 when a bounded wait between thread blocks
 * gave up in one of them (the solution is then not valid; the message is in
 * taucs_b200_last_error()).  Each no-alloc solve clears the status word when
 * it starts, so the status covers the last no-alloc solve issued on the
 * device: call this after each one whose result you need. */
int taucs_b200_solve_device_noalloc_status(void);

/* nrhs right-hand sides in HOST memory (column-major, leading dimension n) */
int taucs_b200_solve_many(void* L, int nrhs, double* X, const double* B);

/* Precision of the numeric factor: 0 = FP64 fronts (default), 1 = FP32 fronts
 * (diagonal scaling, FP32 POTRF, FP32-accumulated products) for use with
 * taucs_b200_solve_refine. */
int taucs_b200_set_precision(void* L, int precision);

/* Iterative refinement: solves A x = b to scaled residual
 * ||A x - b||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= tol with the factor
 * in L (any precision) and an FP64 residual on the device.  A is the permuted
 * matrix the factor was computed from.  Host vectors, nrhs columns.  Returns
 * the number of refinement steps taken (>= 0), or -1 when the target was not
 * reached within maxits; res_out (nrhs) receives the final scaled residuals. */
int taucs_b200_solve_refine(void* L, taucs_ccs_matrix* A, int nrhs, double* X,
                            const double* B, double tol, int maxits, double* res_out);

/* The same refinement on device vectors: d_X (written) and d_B are
 * n x nrhs, column-major with leading dimension ld >= n, permuted order. */
int taucs_b200_solve_refine_device(void* L, int nrhs, double* d_X, const double* d_B,
                                   int ld, double tol, int maxits, double* res_out);

/* Fallback of the refinement when the FP32 factor's steps stall (a scaled
 * residual that fails to halve twice in a row, or the step limit): first
 * preconditioned conjugate gradients (after src/taucs_iter.c:66-223) with the
 * FP32 factor as preconditioner, up to `maxits` iterations (default 100; 0
 * skips it), then an FP64 refactorization.  Batches (several systems in one
 * handle) go straight to FP64.  The report gives how the last refinement
 * finished: 0 FP32 steps only, 1 PCG, 2 FP64 refactorization; and the PCG
 * iterations it used. */
int taucs_b200_set_pcg(void* L, int maxits);
/* How taucs_b200_solve_refine[_device] refines with an FP32 factor: 0
 * (default) refinement steps x += (L32 L32^T)^-1 r, with PCG only when they
 * stall; 1 conjugate gradients preconditioned by the FP32 factor from the
 * first step (one system per handle; batches keep method 0).  Either falls
 * back to an FP64 refactorization when it does not reach the tolerance. */
int taucs_b200_set_refinement(void* L, int method);
/* Operand format of the FP32 fronts' tensor-core products (no counterpart
 * in the reference): 0 TF32 hi + lo parts, three TF32 MMAs per product;
 * 1 (default) FP16 hi + lo parts (lo scaled by 2^11), three FP16 MMAs at
 * twice the TF32 rate and half the operand bytes.  Both keep about 21 bits of every operand; the FP16
 * form relies on the diagonal scaling of the FP32 fronts, which bounds every
 * factor entry by 1 in magnitude. */
int taucs_b200_set_split_format(void* L, int fmt);
int taucs_b200_refine_report(void* L, int* fallback, int* pcg_iterations);

/* Inspection of the symbolic factor, in the reference's own arrays (slots
 * 0..n_sn-1, virtual root n_sn) -- used by the parity tests. */
typedef struct {
  int    n;
  int    n_sn;           /* supernode slots, including emptied ones */
  int    n_live;         /* supernodes with at least one column      */
  int    n_levels;       /* height of the supernodal tree            */
  long   struct_len;     /* sum of sn_up_size                        */
  long   l_values;       /* sum of sn_size * sn_up_size (L doubles)  */
  double flops;          /* the reference's relaxed flop count       */
  double l_bytes;        /* device bytes of L panels                 */
  double u_bytes;        /* device bytes of the update arena (peak)  */
  double ea_bytes;       /* algorithmic extend-add + assembly bytes  */
  double solve_bytes;    /* algorithmic bytes of one 1-RHS solve     */
  int    max_front;      /* largest sn_up_size                       */
  int    max_sn_size;    /* largest sn_size                          */
} taucs_b200_info;

int taucs_b200_factor_info(void* L, taucs_b200_info* info);
int taucs_b200_export_symbolic(void* L, int* sn_size, int* sn_up_size,
                               int* first_child, int* next_child,
                               long* struct_ptr, int* struct_idx);
/* numeric panels as f x s column-major per supernode, rows in sn_struct order
 * (the reference's order), val_ptr[n_sn+1] offsets.  The FP64 factor; a
 * handle that holds only an FP32 factor (taucs_b200_set_precision(L, 1))
 * exports that one, the factor of the scaled matrix D A D with
 * D = diag(A)^-1/2, widened to double. */
int taucs_b200_export_values(void* L, long* val_ptr, double* vals);
/* elimination tree of a permuted lower CCS matrix (parent[n], root = n) */
int taucs_b200_etree(taucs_ccs_matrix* A, int* parent);
/* device layout of the level plan, for checking it (host memory only): per
 * front in device order (info.n_live of them) 14 values: level, parent
 * (device order, -1 root), s, f, and the offsets in elements of its L panel,
 * update matrix (-1 if none), solve work vector, diagonal-block inverses (-1
 * if none), first handshake flag (-1 if none), backward partial sums (-1 if
 * none), its partial-sum row chunks, its reference slot, and the offsets of
 * its row list (f global rows, ascending) and of its map into its parent's
 * row list (f - s local indices); totals: L, U, work-vector, inverse and
 * partial-sum arena lengths, the flag count, and the lengths of the row-list
 * and map arrays that taucs_b200_export_rows_maps fills. */
int taucs_b200_export_layout(void* L, long long* fronts, long long* totals);
int taucs_b200_export_rows_maps(void* L, int* rows, int* maps);
/* the persistent set (small fronts with only small fronts below them, which
 * one launch factors and one launch per direction solves, from device-side
 * queues), host memory only: per task in queue order its front (device
 * order), its parent's task (-1 when the parent is outside the set) and its
 * number of children; returns the number of tasks (arrays may be NULL) */
int taucs_b200_export_persistent(void* L, int* tasks, int* parent_task, int* pending);
/* the solve's block lists of level h (host memory only): (front, 64-row
 * block) pairs in launch order, forward (*n_diag diagonal blocks first, then
 * update-row blocks) and backward; with NULL arrays only the counts are set. */
int taucs_b200_export_solve_blocks(void* L, int h, int* fwd, int* n_fwd, int* n_diag, int* bwd, int* n_bwd);

/* 3D 7-point operator with per-edge conductances exp(sigma*N(0,1)) scaled
 * by (ax, ay, az) on an X x Y x Z grid, Dirichlet boundary (boundary faces
 * drawn the same way and added to the diagonal), seeded; lower CCS in the
 * row order of taucs_ccs_generate_mesh3d.  Z == 0 gives the 2D 5-point
 * analogue on X x Y. */
taucs_ccs_matrix* taucs_b200_generate_lognormal(int X, int Y, int Z, double sigma,
                                                double ax, double ay, double az,
                                                unsigned long long seed);

/* Device timing per kernel class, for benchmarks (off by default).  When
 * enabled, every launch of the library's kernels is bracketed by CUDA events
 * on its stream, and the algorithmic flops and bytes of the launch are
 * recorded.  Enabling or disabling clears the totals. */
#define TAUCS_B200_KC_SMALL_FRONT 0
#define TAUCS_B200_KC_BUILD       1
#define TAUCS_B200_KC_POTRF       2
#define TAUCS_B200_KC_TRSM        3
#define TAUCS_B200_KC_GEMM_PANEL  4
#define TAUCS_B200_KC_GEMM_U      5
#define TAUCS_B200_KC_SOLVE_FWD   6
#define TAUCS_B200_KC_SOLVE_BWD   7
#define TAUCS_B200_KC_OTHER       8
int taucs_b200_profile(int enable);
int taucs_b200_profile_read(int kernel_class, double* ms, long* launches, double* flops, double* bytes);
/* every profiled launch in issue order: its class and device time (ms);
 * copies at most cap entries and returns the number recorded */
long taucs_b200_profile_log(int* kernel_class, float* ms, long cap);

/* Autotuner (no counterpart in the reference): times the numeric
 * factorization of L's pattern on the device values d_values with each GEMM
 * variant (FP64 fronts: 64x64 or 128x128 DMMA tiles; FP32 fronts: the two
 * tcgen05 pipeline shapes) and keeps, per level of the supernodal tree and
 * per product (panel updates, update matrix), the faster one for every
 * later factorization of this handle in its current precision.  Runs four
 * factorizations; uses the library's per-launch profiling, so no other
 * thread may profile at the same time.  choices (2 x levels, may be NULL)
 * receives the variant per level: [2h] panel, [2h + 1] update matrix.
 * Returns 0, or -1 when a factorization failed. */
int taucs_b200_autotune(void* L, const double* d_values, int* choices);

/* The autotuner's measurements also go into a process-wide table keyed by
 * precision, product and the shape class of each level's largest product
 * (rows and K in powers of two); every handle analysed afterwards (including
 * the request server's and batches) takes its per-level variants from the
 * table.  The table can be saved to and loaded from a text file, so a tuning
 * run carries over to later processes; load returns the entries read. */
int  taucs_b200_tuning_save(const char* path);
int  taucs_b200_tuning_load(const char* path);
int  taucs_b200_tuning_entries(void);
void taucs_b200_tuning_clear(void);

/* Sets the GEMM variant per level and product for `precision` (0 FP64
 * fronts, 1 FP32 fronts) -- e.g. choices an earlier taucs_b200_autotune
 * returned for the same pattern, kept by the caller.  count = 2 x levels
 * (layout as in taucs_b200_autotune), or 0 for the default variants. */
int taucs_b200_set_gemm_choices(void* L, int precision, int count, const int* choices);
/* the current variants (2 x levels values) */
int taucs_b200_get_gemm_choices(void* L, int precision, int* choices);

/* Device-memory allocation tracking, after the reference's host allocation
 * tracking (src/taucs_malloc.c:127-250).  Every device and pinned-host
 * allocation this library makes counts as one attempt.
 * taucs_b200_allocation_induce_failure(i) makes attempt i (counted from the
 * last mark) fail as if the device were out of memory;
 * taucs_b200_allocation_mark_clean() restarts the attempt count;
 * taucs_b200_allocation_live() returns the number of the library's live
 * allocations (and their bytes).  A call whose allocation fails returns NULL
 * or -1 and leaves nothing allocated once its handle is freed. */
void taucs_b200_allocation_induce_failure(int i);
int  taucs_b200_allocation_attempts(void);
void taucs_b200_allocation_mark_clean(void);
int  taucs_b200_allocation_live(double* bytes);

/* Testing aid for the failure paths (no counterpart in the reference): sets,
 * on the current device, the polling limit of the bounded waits between
 * thread blocks (default 4194304 polls) and an offset added to the value
 * they wait for (default 0).  A nonzero offset makes every such wait run
 * out: the call that launched it then returns -1 with a timeout message,
 * without a fault or a hang, and the device stays usable.  Restore with
 * (4194304, 0). */
int taucs_b200_debug_waits(int limit, int skew);

/* CUDA kernel launches issued by this library on the calling thread since
 * the last reset (for launch accounting in benchmarks). */
long taucs_b200_launch_count(int reset);

/* last CUDA or internal error message of the calling thread ("" if none) */
const char* taucs_b200_last_error(void);

/* ---- Batches (no counterpart in the reference, which factors one system
 * per call, src/taucs_sn_llt.c:2894-3006).  `count` independent SPD systems
 * (unpermuted lower triangles) are ordered by AMD one by one and analysed
 * as the diagonal blocks of one matrix, so every system keeps its own
 * supernodes and one level-scheduled launch sequence factors (and one
 * solves) all of them.  The handle is a factor handle: taucs_b200_set_precision,
 * taucs_b200_factor_numeric_device (values in the combined order of
 * taucs_b200_batch_values), taucs_b200_solve_device and
 * taucs_b200_solve_refine_device (right-hand sides in the combined order of
 * taucs_b200_batch_rhs; res_out then holds one scaled residual per system
 * and right-hand side, system-major) and taucs_supernodal_factor_free apply;
 * refinement meets the target for every system on its own. */
void* taucs_b200_batch_analyze(int count, taucs_ccs_matrix* const* A);
/* the systems' values (same patterns) gathered into the combined order */
int taucs_b200_batch_values(void* L, taucs_ccs_matrix* const* A, double* combined);
/* right-hand sides of the systems (B[s] of length n_s) into the combined
 * order, and combined solutions back to the systems' own order */
int taucs_b200_batch_rhs(void* L, const double* const* B, double* combined);
int taucs_b200_batch_split(void* L, const double* combined, double* const* X);
/* numeric factorization of all systems from host values, in the precision
 * set by taucs_b200_set_precision */
int taucs_b200_batch_factor(void* L, taucs_ccs_matrix* const* A);
/* one right-hand side per system, host arrays; every system is refined to
 * scaled residual <= tol (res: one value per system, may be NULL); returns
 * the refinement steps, -1 on failure */
int taucs_b200_batch_solve(void* L, double* const* X, const double* const* B, double tol, int maxits,
                           double* res);
int taucs_b200_batch_info(void* L, int* count, int* rows, long* nnz);

/* ---- Request server (no counterpart in the reference, which solves one
 * system per taucs_linsolve call on the calling thread,
 * src/taucs_linsolve.c:433-583).  A server owns `workers` threads, each with
 * its own CUDA stream on the device that is current at creation.  Submitted
 * requests are taken from one FIFO queue by the first free worker, so the
 * work of several requests overlaps on the GPU.  Per sparsity pattern the
 * AMD ordering and the symbolic factor are computed once; factor instances
 * of a pattern are reused and keep their last numeric factor, so a request
 * for a matrix already factored only solves.  Each system is factored with
 * FP32 fronts and refined in FP64 to the request's scaled residual `tol`.
 * Device memory held by factor instances stays under hbm_budget_bytes:
 * idle instances are evicted least recently used first, and a request whose
 * instance does not fit waits until running requests finish. */
typedef struct {
  int    patterns;          /* sparsity patterns analysed             */
  int    instances;         /* factor instances held on the device    */
  double bytes_in_use;      /* predicted device bytes of the instances */
  double budget_bytes;
  long   factorizations;    /* requests that ran a numeric factorization */
  long   resident_solves;   /* requests solved on a resident factor    */
  long   evictions;
  long   waits_for_memory;  /* requests that waited for device memory  */
  long   failed;
  long   queued;            /* requests not yet taken by a worker      */
} taucs_b200_server_info;

void* taucs_b200_server_create(int workers, double hbm_budget_bytes);
/* A: unpermuted lower triangle (TAUCS_DOUBLE | TAUCS_SYMMETRIC | TAUCS_LOWER);
 * B, X: n x nrhs column-major host arrays.  A's arrays, B and X must stay
 * valid until taucs_b200_server_wait returns for the request.  Returns the
 * request id (> 0) or -1. */
long taucs_b200_server_submit(void* server, const taucs_ccs_matrix* A, int nrhs, const double* B,
                              double* X, double tol);
/* Blocks until the request is done: 0 on success, -1 on failure, -2 for an
 * unknown id.  latency_s = completion time - submission time; steps =
 * refinement steps; residual = worst scaled residual of the request's
 * columns; factored = 1 if a numeric factorization ran, 0 if it was solved on
 * a resident factor.  Any output pointer may be NULL. */
int taucs_b200_server_wait(void* server, long id, double* latency_s, int* steps, double* residual,
                           int* factored);
int taucs_b200_server_stats(void* server, taucs_b200_server_info* out);
/* waits for the workers to finish the queued requests, then frees everything */
void taucs_b200_server_destroy(void* server);

#ifdef __cplusplus
}
#endif
#endif

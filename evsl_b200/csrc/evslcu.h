/*
 * evslcu.h -- the thin C ABI between the C host (the EVSL API in the host sources)
 * and the CUDA sm_100a back end (the .cu sources).
 *
 * Conventions
 *   - Every device pointer is plain device memory; vectors are contiguous
 *     doubles, blocks of vectors are column-major with a leading dimension.
 *   - All work is enqueued on the library's stream (evslcu_stream()) and is
 *     asynchronous unless the function says it returns a host value.
 *   - Scalars that one kernel produces and a later kernel consumes stay in
 *     device memory ("device scalars"); the host reads them only where the
 *     algorithm needs a host decision.
 *   - Functions return 0 on success and a negative EVSLCU_ERR_* code on
 *     failure; evslcu_errstr() describes the last failure.
 *   - The FP64 filter kernels reproduce the reference CPU build's arithmetic
 *     bit for bit: each row of y = A x is summed left to right without fused
 *     multiply-add, and the Chebyshev update applies the same sequence of
 *     rounded axpy/scal operations (SRC/chebpoly.c:575-582).
 */
#ifndef EVSL_B200_EVSLCU_H
#define EVSL_B200_EVSLCU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  EVSLCU_OK = 0,
  EVSLCU_ERR_CUDA = -100,
  EVSLCU_ERR_ARG = -101,
  EVSLCU_ERR_NOMEM = -102,
  EVSLCU_ERR_NODEV = -103,
  EVSLCU_ERR_STATE = -104,
  EVSLCU_ERR_TIMEOUT = -105
};

/* ---- context ------------------------------------------------------------ */
int evslcu_init(void);
int evslcu_finish(void);
int evslcu_initialized(void);
const char *evslcu_errstr(void);
void evslcu_set_error(int code, const char *msg);
int evslcu_sync(void);                 /* wait for the library stream */
int evslcu_device_count(void);
int evslcu_device_name(int dev, char *buf, int len, int *sm_count, size_t *mem_bytes);
int evslcu_last_cuda_error(char *buf, int len);
/* Number of kernels this library has launched since evslcu_init. */
uint64_t evslcu_launch_count(void);

/* ---- memory ------------------------------------------------------------- */
void *evslcu_malloc(size_t nbytes);
int evslcu_free(void *p);
int evslcu_h2d(void *dst, const void *src, size_t nbytes);  /* synchronous */
int evslcu_d2h(void *dst, const void *src, size_t nbytes);  /* synchronous */
int evslcu_d2d(void *dst, const void *src, size_t nbytes);  /* async */
int evslcu_memset(void *p, int v, size_t nbytes);           /* async */
int evslcu_h2d_async(void *dst, const void *src, size_t nbytes);

/* ---- timing (CUDA events on the library stream) ------------------------- */
typedef struct evslcu_timer evslcu_timer;
evslcu_timer *evslcu_timer_start(void);
double evslcu_timer_stop(evslcu_timer *t); /* seconds; synchronises on the stop event */
/* A reusable set of timing marks on the library stream: record mark i,
 * then, once the stream has passed both, read the device seconds between
 * two marks (0 when either has not completed). */
typedef struct evslcu_marks evslcu_marks;
evslcu_marks *evslcu_marks_create(int count);
void evslcu_marks_record(evslcu_marks *m, int i);
double evslcu_marks_elapsed(evslcu_marks *m, int i, int j);
void evslcu_marks_destroy(evslcu_marks *m);

/* ---- prepared sparse matrix --------------------------------------------- */
typedef struct evslcu_mat evslcu_mat;
/* Build the device operator from a CSR matrix (0-based, rows sorted).  When
 * on_device is non-zero the arrays are device pointers (borrowed); otherwise
 * host arrays that are uploaded.  The SELL-32 copy used by the filter is
 * built once here. */
evslcu_mat *evslcu_mat_create(int n, int nnz, const int *ia, const int *ja, const double *a,
                              int on_device);
void evslcu_mat_destroy(evslcu_mat *A);
int evslcu_mat_n(const evslcu_mat *A);
long long evslcu_mat_nnz(const evslcu_mat *A);
long long evslcu_mat_padded_nnz(const evslcu_mat *A);
/* Kernel choice for the filter: 0 = SELL-32 thread-per-row, 1 = CSR thread-per-row. */
int evslcu_mat_set_kernel(evslcu_mat *A, int which);
int evslcu_mat_get_kernel(const evslcu_mat *A);
/* y = A x, rows summed left to right. */
int evslcu_spmv(const evslcu_mat *A, const double *x, double *y);
/* Y(:,c) = A X(:,c) for the m columns of column-major X, Y (n rows each) in
 * one launch; each column bitwise evslcu_spmv's. */
int evslcu_spmv_cols(const evslcu_mat *A, const double *X, double *Y, int m);

/* User matvec callback (SetAMatvec): y = A x on device vectors. */
typedef void (*evslcu_mvfunc)(double *x, double *y, void *data);

/* Operator used by the filter: a prepared matrix, or a user callback. */
typedef struct {
  const evslcu_mat *A;
  evslcu_mvfunc func;
  void *data;
  int n;
} evslcu_op;

/* Optional fused epilogue of the last Chebyshev step used by Lanczos:
 *   y <- y + nbeta * zold        (when zold != NULL; SRC/cheblanNr.c:197-200)
 *   *dot_out <- v . y            (device scalar; SRC/cheblanNr.c:202) */
typedef struct {
  const double *zold;
  double nbeta;
  const double *dotv;
  double *dot_out;
} evslcu_cheb_epi;

/* y = p((A - cc I)/dd) v with p = sum_k mu[k] T_k (SRC/chebpoly.c:519-598).
 * mu is a HOST array of deg+1 coefficients.  work holds 3n doubles (only 2n
 * are touched when a prepared matrix is registered). */
int evslcu_chebav(const evslcu_op *op, const double *mu, int deg, double cc, double dd,
                  const double *v, double *y, double *work, const evslcu_cheb_epi *epi);

/* Y = p((A - cc I)/dd) V for the ncols columns of V (column-major n x ncols,
 * ld = n); work holds 2 n ncols doubles.  With a registered matrix every
 * degree is one kernel reading A once per group of 8 columns; each column of
 * Y equals evslcu_chebav of that column bit for bit. */
int evslcu_chebav_block(const evslcu_op *op, const double *mu, int deg, double cc, double dd, int ncols,
                        const double *V, double *Y, double *work);

/* One fused Chebyshev update on device vectors (SRC/evsl_cuda.cu:175-191):
 *   w = t*(vkp1 - cc*vk) - (k>1 ? vkm1 : 0); vkp1 = w; y += s*w. */
int evslcu_cheb_update(int n, int k, double t, double s, double cc, double *vkp1,
                       const double *vk, const double *vkm1, double *y);

/* ---- level-1 with device scalars ---------------------------------------- */
/* out = x . y  (device scalar, deterministic fixed-order reduction) */
int evslcu_dot(int n, const double *x, const double *y, double *out_dev);
/* out = ||x||_2 (device scalar) */
int evslcu_nrm2(int n, const double *x, double *out_dev);
/* y <- y + sign * (*coef_dev) * x */
int evslcu_axpy_ds(int n, const double *coef_dev, double sign, const double *x, double *y);
/* y <- y + a * x (host scalar) */
int evslcu_axpy(int n, double a, const double *x, double *y);
/* x <- (1 / *s_dev) * x */
int evslcu_scal_inv_ds(int n, const double *s_dev, double *x);
/* x <- a * x (host scalar) */
int evslcu_scal(int n, double a, double *x);
int evslcu_copy(int n, const double *x, double *y);
/* read back device scalars (synchronous) */
int evslcu_get_scalars(const double *dev, double *host, int count);

/* ---- Gram-Schmidt (SRC/misc_la.c:221-261) -------------------------------- */
/* Classical GS of v against the k columns of Q (ld = ldq) with the DGKS test,
 * at most imax passes; the pass decisions are taken on the device.  When
 * nrm_out_dev is not NULL the final norm of v is stored there.  work must
 * hold evslcu_cgs_work_size(n, k) doubles. */
size_t evslcu_cgs_work_size(int n, int k);
int evslcu_cgs_dgks(int n, int k, int imax, const double *Q, long long ldq, double *v,
                    double *nrm_out_dev, double *work);

/* ---- dense kernels -------------------------------------------------------- */
/* y = alpha * op(A) x + beta * y, column-major A (m x n); trans 'N' or 'T'. */
int evslcu_dgemv(char trans, int m, int n, double alpha, const double *A, long long lda,
                 const double *x, double beta, double *y);
/* C = alpha * op(A) op(B) + beta * C, column-major; op = 'N' or 'T'. */
/* Tall no-transpose products: 2 (default) use the 128 x 128 tile kernel on
 * the FP64 tensor instruction (mma.sync m8n8k4), 1 the same tiles on DFMA
 * (bitwise equal to 0), 0 always the 64 x 64 kernel.  Returns the previous
 * setting. */
int evslcu_set_dgemm_tiled(int on);
/* FP64 throughput of this GPU (TFLOP/s): FMA chains per thread and
 * mma.sync m8n8k4 f64 chains per warp, registers only (the FP64 roofline). */
int evslcu_fp64_probe(double *dfma_tflops, double *dmma_tflops);
int evslcu_dgemm(char ta, char tb, int m, int n, int k, double alpha, const double *A,
                 long long lda, const double *B, long long ldb, double beta, double *C,
                 long long ldc);

/* ---- Ritz pairs (SRC/cheblanNr.c:336-399, SRC/cheblanTr.c:545-632) -------- */
/* For the m columns of U (n x m, ld = n):
 *   norm_c = ||U_c||; U_c *= 1/norm_c; W_c = A U_c; lam_c = U_c . W_c;
 *   res_c = || W_c - lam_c U_c ||.
 * Host arrays norm, lam, res receive m values each (synchronous).  W needs
 * n*m doubles of scratch. */
int evslcu_ritz_eval(const evslcu_op *op, int n, int m, double *U, double *W, double *norm,
                     double *lam, double *res);
/* Chebyshev filter on many columns at once, each with its own polynomial:
 * y_c = sum_{k<=deg_c} mu_c[k] T_k((A - cc_c)/dd_c) x_c.  x, y: device FP64
 * columns; mu: host array of deg+1 coefficients.  fp32 = 0: each column
 * bitwise equal to evslcu_chebav; fp32 = 1: FP32 values and recurrence
 * (evslcu_mat_prepare_fp32 first when the values are not floats).  Needs the
 * SELL-32 storage.  work: evslcu_filter_columns_work bytes of device memory. */
typedef struct {
  const double *mu;
  int deg;
  double cc, dd;
  const double *x;
  double *y;
} evslcu_filter_col;
/* One column of a batched filter over many matrices (mmfilter.cu): y =
 * p(A) x with the polynomial's coefficients on the device (deg + 1) and a
 * device workspace w of 2 n doubles. */
typedef struct {
  const evslcu_mat *A;
  const double *mu;
  int deg;
  double cc, dd;
  const double *x;
  double *y;
  double *w;
} evslcu_batch_col;
/* Device bytes of the batch's column table (ncols columns, total_rows rows). */
size_t evslcu_filter_batch_table_bytes(int ncols, long long total_rows);
/* Filters ncols columns of possibly different matrices, one launch per
 * degree for all columns whose degree reaches it; each column's y equals
 * ChebAv of that column bit for bit.  table: device memory of at least
 * evslcu_filter_batch_table_bytes(...) bytes. */
int evslcu_filter_batch(int ncols, const evslcu_batch_col *cols, void *table, size_t table_bytes);
/* 1: the batched filter runs every degree of every column in one persistent
 * launch (work items handed out in degree order, each waiting -- bounded --
 * for its column's previous degree); 0 (default): one launch per degree.
 * Same results bit for bit. */
int evslcu_set_batch_persistent(int on);
size_t evslcu_filter_columns_work(int n, int fp32, int ncols);
int evslcu_filter_columns(const evslcu_mat *A, int fp32, int ncols, const evslcu_filter_col *cols, void *work,
                          size_t work_bytes);
int evslcu_mat_prepare_fp32(evslcu_mat *A);
/* The same filter captured once as a CUDA graph for a fixed set of
 * polynomials (cols[].x/.y ignored) and replayed on any columns:
 * plan_run(x[ncols], y[ncols]) (host arrays of device pointers). */
typedef struct evslcu_filter_plan evslcu_filter_plan;
evslcu_filter_plan *evslcu_filter_plan_create(const evslcu_mat *A, int fp32, int ncols,
                                              const evslcu_filter_col *cols);
int evslcu_filter_plan_run(evslcu_filter_plan *P, const double *const *x, double *const *y);
int evslcu_filter_plan_columns(const evslcu_filter_plan *P);
/* Multi-column kernel variant (0..3): bit 0 = 32-byte column parts per
 * thread (else 16), bit 1 = rows' stored entries loaded cooperatively;
 * 4, 5: row-pattern dictionary; 6: column panels (one column); 7: the
 * column-split copy (2-16 columns);
 * -1 (default): per matrix, precision and block width, the variant an
 * autotuner measured fastest (timed once, on first use). */
int evslcu_set_filter_variant(int v);
int evslcu_get_filter_variant(void);
/* Bytes of block rows one column range of the column-split filter
 * (variant 7) gathers from; 0: the default (40 MiB). */
int evslcu_set_xs_range_bytes(long long bytes);
/* Variant the autotuner chose for A (fp32, block width B), -1 if untuned. */
int evslcu_mat_filter_variant(const evslcu_mat *A, int fp32, int B);
/* Measured device time (µs) of one degree step of the multi-column filter on
 * A with B columns (rounded up to the block width), from the autotuner
 * (timed on first use); < 0 if unavailable. */
double evslcu_filter_step_cost(evslcu_mat *A, int fp32, int B);
void evslcu_filter_plan_destroy(evslcu_filter_plan *P);
/* COO (device arrays, indices base 0 or 1) -> CSR on the device: rows in
 * order, entries of a row sorted by column with ties in input order (the
 * reference's cooMat_to_csrMat + sortrow).  Outputs are new device arrays
 * (free with evslcu_free). */
int evslcu_coo_to_csr(int n, long long nnz, const int *ir, const int *jc, const double *vv, int base, int **ia,
                      int **ja, double **a);
/* norms[c] = ||U_c|| for the m columns of U (n x m, ld n); host output. */
int evslcu_colnorms(int n, int m, const double *U, double *norms);
/* Gather columns: dst[:, j] = src[:, idx[j]] for j < cnt (idx host array). */
int evslcu_gather_cols(int n, int cnt, const int *idx, const double *src, double *dst);

/* ---- KPM block moments (SRC/spslice.c:76-130) ----------------------------- */
/* Runs the damped-Chebyshev moment recurrence for nvec probe vectors at once.
 * probes: device, column-major n x nvec (each column is normalised inside, as
 * the reference does).  dots (HOST, Mdeg x nvec, row k = degree k+1): the raw
 * products (T_{k+1}(A~) v_m) . v_m.  ctr/wid map the spectrum to [-1,1]. */
int evslcu_kpm_dots(const evslcu_op *op, int n, int Mdeg, int nvec, const double *probes,
                    double ctr, double wid, double *dots);

/* ---- filter timing ---------------------------------------------------------- */
/* When enabled, every filter application with a prepared matrix is bracketed
 * by CUDA events on the library stream; stats return the summed device time,
 * the algorithmic bytes (A once per degree + vectors touched), the number of
 * degree kernels and of filter calls since the last enable. */
int evslcu_filter_profile(int enable);
int evslcu_filter_stats(double *seconds, double *bytes, uint64_t *launches, uint64_t *calls);
void *evslcu_stream_handle(void);
/* Non-zero (EVSLCU_ERR_TIMEOUT) if a bounded grid barrier of the filter
 * kernel gave up since the last check; clears the flag.  Synchronous. */
int evslcu_filter_error(void);
/* Polls a device-side wait makes before giving up with EVSLCU_ERR_TIMEOUT:
 * the grid barrier of the single-launch filter and the dependency waits of
 * the pipelined filter.  0 restores the defaults (2^26 and 2^22 polls). */
int evslcu_set_wait_limit(unsigned long long polls);
/* Lossless compression of the SELL copy (values as float when all are exactly
 * floats, columns as int16 offsets when they fit); applies to matrices
 * created afterwards.  Default on. */
int evslcu_set_compression(int on);
/* Row order of the SELL copy: -1 automatic (rows sorted by length inside
 * windows of 256 when that cuts the padded slots), 0 never, or a window (a
 * power of two from 32 to 4096) always.  Matrices registered afterwards. */
int evslcu_set_sell_sigma(int sigma);
/* The sort window in use (0: rows in their original order) and the stored
 * slots with and without the sort. */
int evslcu_mat_sell_layout(const evslcu_mat *A, int *sigma, long long *padded, long long *padded_plain);
int evslcu_mat_storage(const evslcu_mat *A, int *vfmt, int *ifmt);
/* Row-pattern dictionary: built at registration when the rows take at most
 * 1024 distinct (value, column - row) sequences (default on; applies to
 * matrices created afterwards).  When built and in use, the FP64
 * single-vector filter and the SpMV read a 2-byte pattern id per row and the
 * pattern table instead of the stored entries; results are identical. */
int evslcu_set_row_patterns(int on);
int evslcu_mat_set_patterns(evslcu_mat *A, int on);
int evslcu_mat_pattern_count(const evslcu_mat *A); /* 0: no dictionary */
int evslcu_mat_uses_patterns(const evslcu_mat *A);
/* Row products of the per-degree filter kernel: unrolled and predicated for
 * rows of at most 8 or 16 stored entries (1, default) or the loop form (0).
 * Same arithmetic either way. */
int evslcu_set_row_unroll(int on);
/* KPM dots (evslcu_kpm_dots) through the Chebyshev product identities, two
 * moments per block matrix product (1, default), or one dot with the probe
 * per degree as the reference (0).  The moments agree to rounding. */
int evslcu_set_kpm_doubling(int on);
/* KPM block step of the product-identity form on the column-split copy of
 * the matrix (8 probes at a time, one launch per column range): -1
 * (default) for large matrices whose columns reach far from the diagonal,
 * 0 never, 1 whenever the matrix can have a copy.  The moments agree to
 * rounding. */
int evslcu_set_kpm_split(int mode);
/* 1: the KPM block step loads each row's own v_k and v_k-1 before its
 * gathers and stores the new vector 16 bytes at a time; 0: after them.
 * Same arithmetic. */
int evslcu_set_kpm_prefetch(int on);
/* The request engine's Lanczos step for many slots in a dozen launches:
 * per slot, z = V(:,k+1) (the filtered vector) gets z -= beta V(:,k-1)
 * (k > 0), alpha = z.V(:,k) into ds[0], z -= alpha V(:,k), then classical
 * Gram-Schmidt with the DGKS test against V(:,0..k) (at most imax passes),
 * the final norm into ds[1] -- the arithmetic, reduction orders included,
 * of evslcu_axpy / evslcu_dot / evslcu_axpy_ds / evslcu_cgs_dgks on each
 * slot alone.  cgsw: evslcu_cgs_work_size(n, k + 1) doubles; npart:
 * evslcu_lz_scratch_doubles() doubles of device scratch per slot (distinct
 * slots, distinct scratch).  table: device memory of
 * evslcu_lanczos_batch_table_bytes(ns) bytes. */
typedef struct {
  int n, k;
  double beta;
  double *V;
  double *ds;
  double *cgsw;
  double *npart;
} evslcu_lz_col;
size_t evslcu_lz_scratch_doubles(void);
size_t evslcu_lanczos_batch_table_bytes(int ns);
int evslcu_lanczos_batch(int ns, const evslcu_lz_col *cols, int imax, void *table, size_t table_bytes);
/* Block Gram-Schmidt, twice, on the m columns of W (n x m, ld n), blocks of
 * b columns: GEMM projections against the earlier columns, then CGS with the
 * DGKS test and unit norms inside the block.  H: (m - b) x b device doubles;
 * norm_dev: 1 device double; cgsw: evslcu_cgs_work_size(n, b) doubles. */
int evslcu_block_cgs2(int n, int m, double *W, int b, double *H, double *norm_dev, double *cgsw);
/* x_i *= a_i (evslcu_scal) for ns vectors in one launch. */
size_t evslcu_scal_batch_table_bytes(int ns);
int evslcu_scal_batch(int ns, const int *n, double *const *x, const double *a, void *table, size_t table_bytes);
void evslcu_lz_release(void);
/* Free the cached split-K partial products of evslcu_dgemm. */
void evslcu_gemm_release(void);
/* Free the cached KPM and tridiagonal workspaces (evslcu_finish calls them). */
void evslcu_kpm_release(void);
void evslcu_trid_release(void);
/* All k eigenvalues (ascending) of the symmetric tridiagonal matrix with
 * diagonal d[0..k) and off-diagonal e[0..k-1), all host arrays, computed on
 * the GPU by multisection on Sturm counts (one warp per eigenvalue);
 * synchronous. */
int evslcu_trid_eigvals(int k, const double *d, const double *e, double *w);
/* The same, computing only the eigenvalues that may be >= xmin (bit for bit
 * those of evslcu_trid_eigvals); the entries of the eigenvalues well below
 * xmin hold a value below xmin instead.  Ascending. */
int evslcu_trid_eigvals_above(int k, const double *d, const double *e, double xmin, double *w);
/* The same computation started on a side stream (inputs copied at the call;
 * one test in flight at a time): _ready returns 1 once it has finished (or
 * when none is in flight), _wait blocks for it and writes w as
 * evslcu_trid_eigvals_above would (same values). */
int evslcu_trid_eigvals_async(int k, const double *d, const double *e, double xmin);
int evslcu_trid_eigvals_async_ready(void);
int evslcu_trid_eigvals_async_wait(double *w);
/* Pattern tables read from the constant-memory pool when they fit there (1,
 * default) or always from global memory (0).  Same arithmetic either way. */
int evslcu_set_pattern_const(int on);
/* Single-vector filter kernel variant: -1 (default) times the allowed
 * variants on a matrix's first filter call and keeps the fastest; 0..6 forces
 * one (0/1 SELL-32 loop/unrolled, 2/3 pattern table in global memory
 * unrolled/loop, 4/5 pattern table in constant memory loop/unrolled, 6 the
 * constant table addressed by a per-row descriptor).  All give identical
 * results. */
int evslcu_set_cheb_variant(int v);
/* At most this many blocks per degree step of the single-vector filter
 * (0, default: one row per thread); rows beyond go round a grid-stride loop. */
int evslcu_set_cheb_max_grid(int blocks);
/* A's chosen variant (-1: not chosen yet) and, in us[0..6], the measured
 * microseconds per degree step of each variant timed (0: not timed). */
int evslcu_mat_cheb_variant(const evslcu_mat *A, float *us);
/* Column-panel layout for large general matrices (panel.cu): on/off, the
 * fewest rows for which it is built (0 keeps the current minimum, 2^18) and
 * the widest panel tried (0 keeps the current width, 16384 columns). */
int evslcu_set_panels(int on, int min_rows, int max_width);
/* Rows per block, panel width and device bytes of the matrix's panel layout
 * for the FP64 (fp32 = 0) or FP32 kernels (zeros when not built). */
int evslcu_mat_panel_layout(const evslcu_mat *A, int fp32, int *rows_per_block, int *panel_width,
                            long long *bytes);
/* The block limit per degree step chosen with the variant (0: none). */
int evslcu_mat_cheb_grid(const evslcu_mat *A);
/* Measured microseconds per degree step of the single-vector FP64 filter
 * kernel chosen for A (times the variants on first use; -1 on failure). */
double evslcu_chebav_step_cost(evslcu_mat *A);
/* Keep A's stored matrix resident in L2 (persisting access-policy window on
 * the library stream, set-aside sized to it) or release that (on = 0). */
int evslcu_mat_l2_persist(const evslcu_mat *A, int on);
/* Threads per block of the single-launch filter (256, 512, 1024; default
 * 1024: fewer blocks meet at each grid barrier). */
int evslcu_set_filter_block(int threads);
/* Rows per thread of the per-degree SELL-32 filter kernel (1 or 2, default 1). */
int evslcu_set_rows_per_thread(int r);
/* Allow (1, default) or forbid (0) the single-launch filter kernel. */
int evslcu_mat_set_persistent(evslcu_mat *A, int on);
/* 1: the filter runs as one pipelined launch (tiles of rows, step s of a tile
 * waits only for step s-1 of the tiles its rows reach); bitwise the same. */
int evslcu_mat_set_wave(evslcu_mat *A, int on);

/* Allocation-free variant of the KPM moments: all scratch (block vectors,
 * dots, partial sums, counters) lives in a fixed 32 MiB __device__ array
 * of the library image; jac/sdiff are the host-computed damping factors and
 * sine differences; mu (Mdeg+1) and ecnt are host outputs.  Synchronous.
 * Calls no allocation routine; sizes whose scratch exceeds the array are
 * rejected with EVSLCU_ERR_ARG.  The first call on a device looks up the
 * array's address (cudaGetSymbolAddress). */
size_t evslcu_kpm_noalloc_capacity(void);
size_t evslcu_kpm_noalloc_need(int n, int Mdeg, int nvec);
int evslcu_kpm_noalloc(const evslcu_op *op, int n, int Mdeg, int nvec, const double *probes, double ctr, double wid,
                       const double *jac, const double *sdiff, double bdiff, double t, double *mu, double *ecnt);

/* ---- random vectors ------------------------------------------------------- */
/* Counter-based uniform [-1,1) generator: value i of draw d under seed s is
 * mix64(s*0x9E3779B97F4A7C15 + (d<<32) + i) mapped to [-1,1), where mix64 is
 * the SplitMix64 output function.  Writes `count` draws starting at `draw`
 * into columns of v (ld = n). */
int evslcu_rand_pm1(int n, int count, uint64_t seed, uint64_t draw, double *v);
int evslcu_randn(int n, uint64_t seed, uint64_t draw, double *v);

#ifdef __cplusplus
}
#endif

#endif

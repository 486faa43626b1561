/*
 * evslx.h -- extensions of libevsl_b200 beyond the reference EVSL API.
 *
 * None of these exist in the reference; each says which reference behaviour
 * it exposes or replaces.  All functions return 0 on success and a negative
 * code on failure (evslx_last_error() then describes it), instead of the
 * reference's assert()/exit() on library failures.
 */
#ifndef EVSL_B200_EVSLX_H
#define EVSL_B200_EVSLX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes (the reference returns 0 / -1 / 2 from the solvers and calls
 * assert or exit elsewhere; those paths return these codes here). */
#define EVSLX_ERR_CUDA (-100)
#define EVSLX_ERR_ARG (-101)
#define EVSLX_ERR_NOMEM (-102)
#define EVSLX_ERR_NODEV (-103)
#define EVSLX_ERR_STATE (-104)
#define EVSLX_ERR_TIMEOUT (-105) /* a bounded device-side wait gave up */
#define EVSLX_ERR_UNSUPPORTED (-106)
#define EVSLX_ERR_NUMERIC (-107)

/* Text of the last error raised by the library. */
const char *evslx_last_error(void);

/* Seed of the device random-vector generator used by rand_double_device and
 * therefore by kpmdos probes and lucky-breakdown restarts (the reference uses
 * unseeded libc rand(), SRC/vect.c:14-20).  Resets the draw counter. */
int evslx_set_seed(uint64_t seed);
/* Current draw counter (each rand_double_device call consumes one draw). */
uint64_t evslx_get_draw(void);

/* kpmdos (SRC/spslice.c:29) with caller-supplied probe vectors instead of
 * vectors drawn inside: probes is DEVICE memory, column-major n x nvec; each
 * column is normalised inside exactly as the reference normalises its draws.
 * All nvec probes run as one block recurrence (one pass over A per degree). */
int evslx_kpmdos_probes(int Mdeg, int damping, int nvec, double *intv, const double *probes,
                        double *mu, double *ecnt);

/* kpmdos with caller probes that allocates nothing -- no counterpart in the
 * reference.  For callers that must not allocate device memory while they
 * run: a serving process that reserves the GPU's memory up front (resident
 * matrices and Lanczos bases under a fixed HBM budget) cannot let a density-
 * of-states request call cudaMalloc/cudaFree, which would break the budget
 * and synchronise the device in the middle of other requests.  Results agree
 * with evslx_kpmdos_probes to rounding (within 1e-12 of max |mu|, normwise):
 * this entry point forms one dot product with the probes per degree, while
 * evslx_kpmdos_probes by default takes two moments per block step from the
 * Chebyshev product identities.
 *
 * All device scratch (block vectors, dot products, partial sums, counters)
 * lives in one fixed 32 MiB array inside the library's device image, which
 * every GPU that loads the library holds until the process exits.  Limits:
 * 1 <= nvec <= 128, 1 <= Mdeg <= EVSLX_NOALLOC_KPM_MAX_DEG, and
 * 3*n*nvec + Mdeg*nvec + (partial sums) must fit the array (about
 * n*nvec <= 1.3 million); larger sizes return EVSLX_ERR_ARG with a message.
 * The calling thread must have the library's device (the one current at
 * EVSLStart) current; another device is rejected with EVSLX_ERR_STATE.  The
 * first call on that device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * The damping factors and sine differences are formed on the calling
 * thread's stack: 16*Mdeg bytes, 64 KiB at the largest Mdeg, which a thread
 * with a small stack must allow for.
 * Every call uses the same array and keeps the previous call's contents
 * (the reduction counters are cleared at the start of each call), so calls
 * that overlap on the GPU -- from several host threads, or enqueued on
 * different streams -- race and must be serialised by the caller.  Probes
 * are DEVICE memory (column-major n x nvec); mu and ecnt are host outputs;
 * the call returns when they are written. */
#define EVSLX_NOALLOC_KPM_MAX_DEG 4096
int evslx_kpmdos_probes_noalloc(int Mdeg, int damping, int nvec, double *intv, const double *probes,
                                double *mu, double *ecnt);

/* The two halves of kpmdos, for callers that distribute the probes (e.g.
 * one shard of probes per GPU): evslx_kpm_dots returns the raw products
 * dots[k*nvec + m] = (T_{k+1}(A~) v_m) . v_m of the normalised device probes
 * (column-major n x nvec); evslx_kpm_accumulate (host only, no GPU needed)
 * turns the dots of all nvec probes into mu[0..Mdeg] and the eigenvalue
 * count exactly as kpmdos does (SRC/spslice.c:76-136).  Each probe's dots do
 * not depend on which other probes share its block, so gathering shards and
 * accumulating gives bit for bit the single-call result. */
int evslx_kpm_dots(int Mdeg, int nvec, double *intv, const double *probes, double *dots);
int evslx_kpm_accumulate(int Mdeg, int damping, int nvec, int n, double *intv, const double *dots, double *mu,
                         double *ecnt);

/* Device vectors for explicit draws first_draw .. first_draw+count-1 of the
 * library generator (the draws kpmdos would consume), without advancing the
 * draw counter; v is column-major n x count. */
int evslx_rand_device_draws(int n, int count, uint64_t first_draw, double *v);

/* Filter SpMV kernel for the registered matrix: 0 = SELL-32 (default),
 * 1 = CSR one thread per row.  Both give identical (bitwise) results. */
int evslx_set_spmv_kernel(int which);
int evslx_get_spmv_kernel(void);

/* Filter execution: 0 (default) launches one fused kernel per degree, each
 * launched with programmatic dependent launch so consecutive degrees overlap
 * their launch; 1 runs all degrees of a filter application in one
 * cooperative kernel (bounded grid barriers between degrees, per-row state in
 * shared memory).  Results are identical bit for bit. */
int evslx_set_filter_persistent(int on);

/* ChebLanNr's convergence tests (the eigenvalues of T_k every 20 steps):
 * 1 (default) runs each on a side stream while the next Lanczos steps
 * proceed and reads it at the next test point or when it finishes (steps
 * taken past a converged test are discarded); 0 waits for each test.  The
 * results are identical bit for bit. */
int evslx_set_async_tests(int on);
/* Rows each thread of the per-degree filter kernel handles (1 or 2, default
 * 1; 2 gives each thread two independent load chains, measured slower on
 * the 3-D Laplacian).  Results are identical. */
int evslx_set_filter_rows_per_thread(int r);
/* Threads per block of the single-launch filter: 256, 512 or 1024 (default). */
int evslx_set_filter_block(int threads);

/* Lossless compression of the stored matrix used by the filter: values kept
 * as float when every value is exactly a float, columns as 16-bit offsets
 * from the row when they fit.  Applies to matrices registered afterwards;
 * default on.  Results are identical either way. */
int evslx_set_matrix_compression(int on);
/* SELL-C-sigma row order of the stored matrix (C = 32).  sigma -1 (default):
 * when the chunks of 32 consecutive rows would carry more than 10% padding
 * (rows of unequal length, as in general sparse matrices), the rows of each
 * window of 256 consecutive rows are sorted by length before they are cut
 * into chunks, and the sorted order is kept when it stores at least 5% fewer
 * slots; 0: never sort; a power of two from 32 to 4096: always sort with that
 * window.  Vectors stay in the caller's row order and every row is summed in
 * its CSR order, so results are identical either way.  Applies to matrices
 * registered afterwards.  (Replaces the cuSPARSE CSR descriptor of
 * SRC/spmat.c:529-621; the CSR matvec SRC/spmat.c:257-298 is the arithmetic.) */
int evslx_set_sell_sigma(int sigma);
/* Layout of the registered matrix: the sort window in use (0: rows in their
 * original order), the stored slots (entries plus padding) and the slots the
 * unsorted layout would store. */
int evslx_matrix_sell_layout(int *sigma, long long *stored, long long *stored_unsorted);
/* Run each filter application as one pipelined launch: rows in tiles, work
 * items (degree, tile) handed out in order, a tile's degree k waiting only
 * for degree k-1 of the tiles its rows reach (bounded waits).  Results are
 * bitwise those of the per-degree launches. */
int evslx_set_filter_wave(int on);
/* Every device-side wait is bounded: a block of the single-launch filter
 * gives up at a grid barrier after 2^26 polls (about 2 s), a tile of the
 * pipelined filter after 2^22 polls on a dependency; the call then returns
 * EVSLX_ERR_TIMEOUT and the library stays usable.  This sets both limits
 * (0 restores the defaults); a very small limit makes the waits run out,
 * which tests of the failure path use. */
int evslx_set_wait_limit(unsigned long long polls);

/* Keep the registered matrix's stored arrays resident in L2 (a persisting
 * access-policy window on the library stream with this process's persisting
 * L2 set-aside sized to them, up to the device maximum; released when the
 * matrix is dropped or at EVSLFinish).  Default off (measured no gain for the
 * 3-D Laplacian 100^3, whose working set already stays in L2); results are
 * identical either way. */
int evslx_set_l2_resident(int on);
/* Row-pattern dictionary of the stored matrix: when the rows take at most
 * 1024 distinct sequences of (value, column - row) pairs, as on structured
 * grids, registration also builds one table entry per distinct sequence and
 * a 2-byte pattern id per row, and the FP64 single-vector filter and the
 * matvec read those (same products in the same order as the CSR row, so
 * results are identical).  on = 0 stops using the dictionary for the
 * registered matrix and skips building it for matrices registered
 * afterwards.  Default on. */
int evslx_set_row_patterns(int on);
/* Distinct row patterns of the registered matrix (0: no dictionary). */
int evslx_row_pattern_count(void);
/* Kernel of the FP64 single-vector filter.  variant -1 (default): the first
 * filter call on a matrix times each variant allowed for it and keeps the
 * fastest; 0..6 forces one: 0/1 SELL-32 with looped/unrolled row products,
 * 2/3 pattern table in global memory unrolled/looped, 4/5 pattern table in
 * constant memory looped/unrolled, 6 constant-memory table addressed by a
 * 4-byte descriptor per row, 7 the column-panel layout (2-6 need the
 * row-pattern dictionary, 4-6 its table in the constant pool, 7 the panel
 * layout; filtering fails with EVSLX_ERR_ARG when the forced variant is not
 * available).  Every variant gives the same result
 * bit for bit. */
int evslx_set_filter_kernel(int variant);
/* The registered matrix's chosen variant (-1: not chosen yet) and, when us is
 * not NULL, us[0..7] = measured microseconds per degree step of each variant
 * timed (0: not timed).  Variant 7 is the column-panel kernel (see
 * evslx_set_panel_filter). */
int evslx_filter_kernel(double *us);
/* Column-panel filter for large general sparse matrices (no counterpart in
 * the reference, whose SpMV is the CSR matvec SRC/spmat.c:257-298 or
 * cuSPARSE, :529-621).  On a matrix whose rows have unequal lengths (SELL-C-
 * sigma sorted) and at least min_rows rows (default 2^18), the first filter
 * call also builds a layout in which each thread block owns a block of rows
 * and walks the columns in panels: each panel of x and the block's entries in
 * it are copied into shared memory by TMA bulk copies through a multi-stage
 * ring (a producer warp runs ahead of the warps that multiply), so the random
 * gathers read shared memory instead of one cache line each.
 * Every row is still summed left to right in CSR order: results are
 * bitwise those of the other FP64 kernels.  The timing-based kernel choice
 * (single vector: variant 7; multi-column filter at one column: variant 6)
 * uses it where it is faster.  on = 0 stops building it; min_rows <= 0 keeps
 * the current minimum; max_width > 0 caps the panel width (columns, at least
 * 512; default 16384), max_width <= 0 keeps the current cap.  Applies to
 * layouts built afterwards. */
int evslx_set_panel_filter(int on, int min_rows, int max_width);
/* The registered matrix's panel layout for the FP64 (fp32 = 0) or FP32
 * kernels: rows per block, panel width and device bytes (zeros if none). */
int evslx_matrix_panel_layout(int fp32, int *rows_per_block, int *panel_width, long long *bytes);
/* Blocks per degree step chosen with that variant (0: one row per thread;
 * otherwise rows go round a grid-stride loop of that many blocks). */
int evslx_filter_kernel_grid(void);
/* Bytes per stored value (4 or 8) and per stored column index (2 or 4). */
int evslx_matrix_storage(int *value_bytes, int *index_bytes);

/* y = A x for the registered matrix on device vectors (rows summed left to
 * right, like the reference CPU matvec SRC/spmat.c:257-298). */
int evslx_matvec(const double *x, double *y);
/* Y(:,c) = A X(:,c) for the m columns of the column-major device blocks X,
 * Y (n x m) in one launch, each column bitwise evslx_matvec's (a registered
 * CSR matrix; with a SetAMatvec operator, the callback once per column).
 * The Ritz pairs of the solvers use it for their residuals. */
int evslx_matvec_cols(int m, const double *X, double *Y);

/* Y = p(A) V for ncols device vectors at once (V, Y: column-major n x ncols;
 * work: 2 n ncols doubles).  One pass over A per degree serves every group
 * of 8 columns; each column of Y equals ChebAv (SRC/chebpoly.c:519) of the
 * same column bit for bit.  No reference counterpart: the reference filters
 * a block column by column (SRC/chebsi.c:127-129). */
int evslx_chebav_block(polparams *pol, int ncols, const double *V, double *Y, double *work);

/* Matrix-Market coordinate reader with the semantics of the reference
 * drivers' read_coo_MM (TESTS/COMMON/io.c:115): real or integer, square;
 * symmetric files are expanded (transposed off-diagonal entries appended in
 * file order); indices shifted by idxout - idxin.  Returns 0, 1 (unsupported
 * or malformed header), -1 (fewer entries than announced) or EVSLX_ERR_ARG
 * (file cannot be opened).  Output arrays are malloc'd (free_coo).  No GPU
 * needed. */
int evslx_read_coo_MM(const char *matfile, int idxin, int idxout, cooMat *Acoo);

/* COO -> CSR on the GPU: the CSR of cooMat_to_csrMat (rows sorted by column,
 * ties in input order) built on the device, as device arrays (owndata = 2,
 * free with evsl_free_csr_gpu).  coo_on_device: the COO arrays are device
 * pointers (else host arrays, uploaded).  Ready for SetAMatrix_device_csr. */
int evslx_coo_to_csr_device(int cooidx, const cooMat *coo, int coo_on_device, csrMat *Agpu);

/* ---------------------------------------------------------------------------
 * Batched and served slicing (no reference counterpart: the reference solves
 * one slice per call, SRC/cheblanNr.c:57).
 *
 * Resident matrices: evslx_matrix_create uploads a host CSR (on_device = 0)
 * or borrows a device CSR (on_device = 1) and prepares its SELL-32 copy.
 *
 * Engine: a queue of requests -- slice solves (ChebLanNr's algorithm and
 * outputs) and DOS estimates (kpmdos) -- served with up to max_slots slice
 * solves in flight.  evslx_engine_step admits queued requests (FIFO) while a
 * slot is free and the request's device memory fits hbm_budget (0: no
 * limit), advances every active solve by one Lanczos step (the filters of
 * all solves on one matrix share one multi-column filter per degree) and
 * retires finished ones into the result queue; it returns the number of
 * requests queued or active, or a negative error code.  Results are the
 * same for a request alone and in any mix.
 *
 * precision: EVSLX_PREC_FP64 (filter in FP64) or EVSLX_PREC_MIXED (filter in
 * FP32; Lanczos, orthogonalisation, Ritz step in FP64; Ritz pairs refined by
 * FP64 filtered Rayleigh-Ritz sweeps over the candidates plus half as many
 * guard vectors (at least 16), with a filter designed for the interval the
 * candidates span, until every pair inside [a, b] meets tol: at most 4
 * sweeps for filters of degree >= 128, up to 24 for low degrees).
 * ------------------------------------------------------------------------- */
#define EVSLX_PREC_FP64 0
#define EVSLX_PREC_MIXED 1
#define EVSLX_REQ_SLICE 1
#define EVSLX_REQ_KPM 2

typedef struct evslx_matrix evslx_matrix;
typedef struct evslx_engine evslx_engine;

typedef struct {
  uint64_t tag;        /* the submitter's tag */
  int kind;            /* EVSLX_REQ_SLICE or EVSLX_REQ_KPM */
  int rc;              /* 0 or an error code */
  int nev;             /* slice: eigenpairs found (in [a, b], residual < tol) */
  double *lam, *res;   /* slice: host arrays of nev (free with evslx_result_free) */
  double *Y;           /* slice: device n x nev when the engine keeps vectors */
  double *mu;          /* DOS: host array of Mdeg + 1 moments */
  double ecnt;         /* DOS: estimated eigenvalue count */
  int lanczos_steps;   /* slice: Lanczos dimension */
  int refine_sweeps;   /* slice, mixed precision: FP64 refinement sweeps */
  double t_submit, t_start, t_finish; /* evsl_timer() seconds */
} evslx_result;

evslx_matrix *evslx_matrix_create(csrMat *A, int on_device);
void evslx_matrix_free(evslx_matrix *M);
long long evslx_matrix_device_bytes(const evslx_matrix *M);

evslx_engine *evslx_engine_create(int max_slots, size_t hbm_budget, int precision, int keep_vectors);
void evslx_engine_free(evslx_engine *E);
/* vinit: n doubles, on the device when vinit_on_device (copied at submit). */
int evslx_engine_submit_slice(evslx_engine *E, evslx_matrix *M, const double *intv, const polparams *pol,
                              int maxit, double tol, const double *vinit, int vinit_on_device, uint64_t tag);
/* Probes: the generator's draws 0..nvec-1 of `seed` (kpmdos after
 * evslx_set_seed(seed) draws the same vectors). */
int evslx_engine_submit_kpm(evslx_engine *E, evslx_matrix *M, int Mdeg, int damping, int nvec, const double *intv,
                            uint64_t seed, uint64_t tag);
int evslx_engine_step(evslx_engine *E);
/* Mixed-precision engines created afterwards run the FP32 filter only on
 * matrices with at least `rows` rows (default 131072) and filter smaller ones
 * in FP64, where FP32 saves little and the refinement costs more. */
void evslx_set_mixed_min_rows(int rows);
/* Filters run as captured CUDA graphs, rebuilt when the set of requests on
 * a matrix changes (default on); plan_builds counts the captures. */
void evslx_engine_use_graphs(evslx_engine *E, int on);
/* Batched filter of the engine (default on, max_rows 2^18): every tick, the
 * lone FP64 columns of matrices with at most max_rows rows (independent
 * instances, small serving requests) are filtered together, one launch per
 * degree for all of them, instead of one launch per degree per matrix; each
 * column's result is bit for bit the single-vector filter's.  max_rows <= 0
 * keeps the current limit.  No counterpart in the reference, whose drivers
 * solve slices one after another (TESTS/PLanR/MMPLanR_omp.c:183-241 runs
 * them on OpenMP threads). */
void evslx_engine_use_batch(evslx_engine *E, int on, int max_rows);
/* 1 (default): the vector operations of the Lanczos steps of all slots run
 * together, one launch per operation for every slot (the same arithmetic,
 * reductions included, as each slot's own launches); 0: each slot's own
 * launches. */
void evslx_engine_use_batch_ops(evslx_engine *E, int on);
/* The batched filter's form, for every engine: 0 (default) one launch per
 * degree for all its columns; 1 one persistent launch for all degrees (work
 * items -- degree, block of a column -- handed out in degree order, each
 * waiting, with the bound of evslx_set_wait_limit, for its column's previous
 * degree; a wait that runs out makes the engine step return
 * EVSLX_ERR_TIMEOUT).  Results are the same bit for bit. */
int evslx_set_batch_persistent(int on);
/* Host wall-clock seconds the engine's steps spent so far in: [0] admission
 * and issuing the filters, [1] issuing the rest of the Lanczos steps, [2]
 * waiting for the step's scalars (the device's backlog), [3] the host part
 * (tridiagonal tests, restarts), [4] retiring finished requests.  No
 * synchronisation is added to measure them. */
void evslx_engine_phase_times(const evslx_engine *E, double out[5]);
/* Columns filtered through the batched filter so far. */
uint64_t evslx_engine_batched_columns(const evslx_engine *E);
uint64_t evslx_engine_plan_builds(const evslx_engine *E);
/* Filter groups launched so far, by block width 1, 2, 4, 8, 16 (a group of
 * one FP64 column runs the single-vector filter). */
void evslx_engine_group_widths(const evslx_engine *E, uint64_t counts[5]);
int evslx_engine_run(evslx_engine *E); /* step until nothing is queued or active */
int evslx_engine_pending(const evslx_engine *E);
size_t evslx_engine_bytes_in_use(const evslx_engine *E);
int evslx_engine_pop_result(evslx_engine *E, evslx_result *out); /* 1: a result was returned */
void evslx_result_free(evslx_result *r);

/* Y_c = p_c(A) X_c for ncols columns of the registered CSR matrix, each with
 * its own polynomial pols[c] (X, Y: device, column-major n x ncols).  FP64:
 * every column equal to ChebAv bit for bit; MIXED: the FP32 filter. */
int evslx_chebav_multi(int ncols, const polparams *pols, const double *X, double *Y, int precision);

/* Variant of the multi-column filter kernel (results are identical; the
 * SELL-32 forms add the zero padding of a chunk, which can only turn an
 * exactly zero row sum of -0 into +0):
 * 0..3 -- SELL-32; bit 0: each thread handles 32 bytes of a row's columns
 * (else 16), bit 1: a row's threads load its stored entries cooperatively;
 * 4, 5 -- the row-pattern dictionary (see evslx_set_row_patterns), 16- or
 * 32-byte column parts; filtering fails with EVSLX_ERR_ARG when the matrix
 * has none;
 * 6 -- one column on the column-panel layout (large general matrices);
 * 7 -- 2 to 16 columns on the column-split copy: the columns are cut into
 * ranges whose rows of the block fit in L2 (see
 * evslx_set_split_range_bytes), a degree step runs range by range and
 * carries each row's running sum between ranges (one range when the whole
 * block fits); streaming cache hints keep the gathered rows in L2.  Tried by
 * the autotuner on matrices of at least 2^18 rows (it costs another stored
 * copy of the matrix).
 * Rows are summed in their CSR order and padding is skipped, so FP64
 * columns equal ChebAv bit for bit.  Needs increasing column indices in
 * every row; filtering fails with EVSLX_ERR_ARG when the matrix or width
 * has no such copy;
 * -1 (default) -- autotuned: the first filter on a matrix with a given
 * precision and block width times the variants available for it on a few
 * degree steps and keeps the fastest for that matrix. */
int evslx_set_filter_variant(int v);
int evslx_get_filter_variant(void);
/* Bytes of the block's rows one column range of filter variant 7 may
 * gather from (default 40 MiB, about a third of the B200's L2; 0 restores
 * it).  Widths whose block fits in this many bytes run as one range.  Applies
 * to matrices whose filter is tuned afterwards. */
int evslx_set_split_range_bytes(long long bytes);
/* The variant tuned for the registered matrix (-1: not tuned yet). */
int evslx_tuned_filter_variant(int precision, int ncols);

/* nslices slices of the registered CSR matrix solved together in one engine
 * (intvs: 4 per slice; pols: one per slice; vinit: device start vector
 * shared by all).  Outputs per slice as ChebLanNr (lamo/reso host, Wo
 * device). */
int evslx_ChebLanNr_batch(int nslices, double *intvs, int maxit, double tol, double *vinit, polparams *pols,
                          int precision, int *nevOut, double **lamo, double **Wo, double **reso);

/* Size of the registered problem and of the stored matrix. */
int evslx_problem_info(int *n, long long *nnz, long long *stored_nnz);

/* Number of GPU kernels the library has launched since EVSLStart. */
uint64_t evslx_launch_count(void);

/* Device time (seconds, CUDA events) of the last kpmdos moment recurrence. */
double evslx_last_kpm_seconds(void);

/* Size of the last ChebLanNr solve: Lanczos dimension kdim and the number of
 * Ritz values >= bar examined (for ChebLanTr: total Lanczos steps). */
int evslx_last_solve_info(int *lanczos_steps, int *candidates);

/* The CUDA stream (cudaStream_t) all library work is queued on; callers can
 * record their own events on it. */
void *evslx_stream(void);

/* Filter instrumentation: when enabled, each filter application p(A)v with a
 * registered CSR matrix is bracketed by CUDA events.  evslx_filter_stats
 * returns the device seconds spent in the filter kernels, their algorithmic
 * bytes (12 bytes per nonzero + 4 per row for A at every degree, plus 8 bytes
 * per vector element read or written), the kernel count and the call count. */
int evslx_filter_profile(int enable);
int evslx_filter_stats(double *seconds, double *bytes, uint64_t *launches, uint64_t *calls);

#ifdef __cplusplus
}
#endif

#endif

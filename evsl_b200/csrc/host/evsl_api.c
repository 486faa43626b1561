/*
 * evsl_api.c -- library state, setters, CSR helpers, memory wrappers and the
 * device BLAS shims of the EVSL C API.
 *
 * Reference counterparts: SRC/evsl.c (state and setters), SRC/spmat.c (CSR
 * helpers, device CSR creation), SRC/evsl_memory.c (memory wrappers),
 * SRC/vect.c:212-284 (device BLAS shims).  The reference creates cuBLAS,
 * cuSPARSE and cuRAND handles in EVSLStart; this library starts its own CUDA
 * back end instead (evslcu_init) and uses none of those libraries.
 */
#include <stdarg.h>

#include "internal.h"

evslData evsldata;
evslStat evslstat;
evsl_host_state evslh;

static char g_errmsg[512] = "";

int evsl_seterr(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_errmsg, sizeof(g_errmsg), fmt, ap);
  va_end(ap);
  return code;
}

const char *evslx_last_error(void) {
  if (g_errmsg[0]) return g_errmsg;
  return evslcu_errstr();
}

static int from_cu(int rc) {
  if (rc) {
    const char *m = evslcu_errstr();
    snprintf(g_errmsg, sizeof(g_errmsg), "%s", m && m[0] ? m : "CUDA back end error");
  }
  return rc;
}

int evsl_require_started(void) {
  if (!evslh.started) return evsl_seterr(EVSLX_ERR_STATE, "EVSLStart has not been called");
  return 0;
}

int evsl_require_operator(void) {
  int rc = evsl_require_started();
  if (rc) return rc;
  if (!evslh.op.A && !evslh.op.func)
    return evsl_seterr(EVSLX_ERR_STATE, "no matrix registered (SetAMatrix / SetAMatrix_device_csr / SetAMatvec)");
  return 0;
}

const evslcu_op *evsl_op(void) { return &evslh.op; }

int evsl_check_intv(const double *intv, FILE *fstats) {
  double a = intv[0], b = intv[1], lmin = intv[2], lmax = intv[3];
  if (a >= b) {
    if (fstats) fprintf(fstats, " error: invalid interval (%e, %e)\n", a, b);
    return -1;
  }
  if (a >= lmax || b <= lmin) {
    if (fstats) fprintf(fstats, " error: interval (%e, %e) is outside (%e %e) \n", a, b, lmin, lmax);
    return -2;
  }
  return 0;
}

/* ---------------------------------------------------------------------------
 * Start / finish (SRC/evsl.c:24-87)
 * ------------------------------------------------------------------------- */
int EVSLStart(void) {
  memset(&evsldata, 0, sizeof(evsldata));
  StatsReset();
  evsl_timer();
  g_errmsg[0] = 0;
  int rc = evslcu_init();
  if (rc) return from_cu(rc);
  if (!evslh.started) {
    memset(&evslh, 0, sizeof(evslh));
    evslh.seed = 0x5EEDULL;
    evslh.kernel = -1;
    evslh.l2_resident = 0;
  }
  evslh.started = 1;
  return 0;
}

static void drop_matrix(void) {
  if (evslh.mat) evslcu_mat_destroy(evslh.mat);
  evslh.mat = NULL;
  evslh.mat_key = NULL;
  memset(&evslh.op, 0, sizeof(evslh.op));
}

int EVSLFinish(void) {
  drop_matrix();
  if (evsldata.Amv) free(evsldata.Amv);
  evsldata.Amv = NULL;
  evslh.started = 0;
  int rc = evslcu_finish();
  return from_cu(rc);
}

static int register_csr(csrMat *A, int on_device) {
  int rc = evsl_require_started();
  if (rc) return rc;
  if (!A || A->nrows != A->ncols || A->nrows <= 0)
    return evsl_seterr(EVSLX_ERR_ARG, "matrix must be square with n > 0");
  int nnz = 0;
  if (on_device) {
    if (evslcu_d2h(&nnz, A->ia + A->nrows, sizeof(int))) return from_cu(EVSLX_ERR_CUDA);
  } else {
    nnz = A->ia[A->nrows];
  }
  drop_matrix();
  evslh.mat = evslcu_mat_create(A->nrows, nnz, A->ia, A->ja, A->a, on_device);
  if (!evslh.mat) return from_cu(EVSLX_ERR_ARG);
  if (evslh.kernel >= 0) evslcu_mat_set_kernel(evslh.mat, evslh.kernel);
  evslcu_mat_set_persistent(evslh.mat, evslh.persistent);
  if (evslh.l2_resident) evslcu_mat_l2_persist(evslh.mat, 1);
  evslcu_mat_set_wave(evslh.mat, evslh.wave);
  evslh.mat_key = A;
  evslh.op.A = evslh.mat;
  evslh.op.func = NULL;
  evslh.op.data = NULL;
  evslh.op.n = A->nrows;
  evsldata.n = A->ncols;
  if (!evsldata.Amv) evsldata.Amv = (EVSLMatvec *)calloc(1, sizeof(EVSLMatvec));
  evsldata.Amv->func = NULL;
  evsldata.Amv->data = (void *)A;
  return 0;
}

/* SRC/evsl.c:95 -- host CSR: uploaded once to the device (the reference keeps
 * a borrowed host pointer and multiplies on the CPU). */
int SetAMatrix(csrMat *A) { return register_csr(A, 0); }

/* SRC/evsl.c:256 -- device CSR (borrowed; must outlive its use). */
int SetAMatrix_device_csr(csrMat *A) { return register_csr(A, 1); }

/* SRC/evsl.c:132 -- user matvec on device vectors. */
int SetAMatvec(int n, MVFunc func, void *data) {
  int rc = evsl_require_started();
  if (rc) return rc;
  if (n <= 0 || !func) return evsl_seterr(EVSLX_ERR_ARG, "SetAMatvec: need n > 0 and a function");
  drop_matrix();
  evslh.op.A = NULL;
  evslh.op.func = (evslcu_mvfunc)func;
  evslh.op.data = data;
  evslh.op.n = n;
  evsldata.n = n;
  if (!evsldata.Amv) evsldata.Amv = (EVSLMatvec *)calloc(1, sizeof(EVSLMatvec));
  evsldata.Amv->func = func;
  evsldata.Amv->data = data;
  return 0;
}

int SetStdEig(void) {
  evsldata.ifGenEv = 0;
  return 0;
}

/* The generalized problem A x = lambda B x is not part of this library. */
int SetGenEig(void) {
  return evsl_seterr(EVSLX_ERR_UNSUPPORTED, "generalized eigenproblems are not supported by this library");
}

void evsl_device_query(int dev) {
  char name[256];
  int sms = 0;
  size_t mem = 0;
  int cnt = evslcu_device_count();
  if (cnt <= 0) {
    printf("EVSL: no CUDA device\n");
    return;
  }
  if (evslcu_device_name(dev, name, sizeof(name), &sms, &mem) == 0)
    printf("EVSL: device %d of %d: %s, %d SMs, %.1f GB\n", dev, cnt, name, sms, mem / 1e9);
}

void evsl_last_device_err(void) {
  char buf[256];
  if (evslcu_last_cuda_error(buf, sizeof(buf))) printf(" EVSL CUDA error: %s\n", buf);
}

/* ---------------------------------------------------------------------------
 * CSR helpers (SRC/spmat.c)
 * ------------------------------------------------------------------------- */
/* Sort the entries of every row by column, ties in their current order --
 * the result of the reference's sortrow (SRC/spmat.c:67-85), a double
 * transposition, which is a stable sort by column. */
struct row_entry {
  int c, order;
  double v;
};

static int cmp_row_entry(const void *x, const void *y) {
  const struct row_entry *a = (const struct row_entry *)x, *b = (const struct row_entry *)y;
  if (a->c != b->c) return (a->c > b->c) - (a->c < b->c);
  return (a->order > b->order) - (a->order < b->order);
}

static int sort_rows(int n, const int *ia, int *ja, double *a) {
  int maxlen = 0;
  for (int r = 0; r < n; r++) maxlen = evsl_max(maxlen, ia[r + 1] - ia[r]);
  struct row_entry *buf = (struct row_entry *)malloc(sizeof(struct row_entry) * (size_t)(maxlen > 0 ? maxlen : 1));
  if (!buf) return evsl_seterr(EVSLX_ERR_NOMEM, "sorting CSR rows: out of memory");
  for (int r = 0; r < n; r++) {
    const int b = ia[r], len = ia[r + 1] - b;
    int sorted = 1;
    for (int j = 1; j < len && sorted; j++)
      if (ja[b + j] < ja[b + j - 1]) sorted = 0;
    if (sorted) continue;
    for (int j = 0; j < len; j++) {
      buf[j].c = ja[b + j];
      buf[j].order = j;
      buf[j].v = a[b + j];
    }
    qsort(buf, (size_t)len, sizeof(struct row_entry), cmp_row_entry);
    for (int j = 0; j < len; j++) {
      ja[b + j] = buf[j].c;
      a[b + j] = buf[j].v;
    }
  }
  free(buf);
  return 0;
}

int cooMat_to_csrMat(int cooidx, cooMat *coo, csrMat *csr) {
  const int n = coo->nrows, nnz = coo->nnz;
  csr->owndata = 1;
  csr->nrows = coo->nrows;
  csr->ncols = coo->ncols;
  csr->nnz = nnz;
  csr->descr = NULL;
  csr->dBuffer = NULL;
  csr->ia = (int *)calloc((size_t)n + 1, sizeof(int));
  csr->ja = (int *)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
  csr->a = (double *)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
  if (!csr->ia || !csr->ja || !csr->a) return evsl_seterr(EVSLX_ERR_NOMEM, "cooMat_to_csrMat: out of memory");
  for (int i = 0; i < nnz; i++) {
    const int r = coo->ir[i] - cooidx, c = coo->jc[i] - cooidx;
    if (r < 0 || r >= n || c < 0 || c >= coo->ncols) {
      free(csr->ia);
      free(csr->ja);
      free(csr->a);
      csr->ia = csr->ja = NULL;
      csr->a = NULL;
      return evsl_seterr(EVSLX_ERR_ARG, "cooMat_to_csrMat: entry %d has index (%d, %d) outside the %d x %d matrix", i,
                         r, c, n, coo->ncols);
    }
  }
  for (int i = 0; i < nnz; i++) csr->ia[coo->ir[i] - cooidx + 1]++;
  for (int i = 0; i < n; i++) csr->ia[i + 1] += csr->ia[i];
  int *pos = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  memcpy(pos, csr->ia, sizeof(int) * (size_t)n);
  for (int i = 0; i < nnz; i++) {
    const int r = coo->ir[i] - cooidx;
    const int k = pos[r]++;
    csr->ja[k] = coo->jc[i] - cooidx;
    csr->a[k] = coo->vv[i];
  }
  free(pos);
  return sort_rows(csr->nrows, csr->ia, csr->ja, csr->a);
}

void free_csr(csrMat *csr) {
  if (!csr || !csr->owndata) return;
  if (evslh.mat_key == (const void *)csr) drop_matrix();
  free(csr->ia);
  free(csr->ja);
  free(csr->a);
  csr->ia = NULL;
  csr->ja = NULL;
  csr->a = NULL;
}

void free_coo(cooMat *coo) {
  if (!coo) return;
  free(coo->ir);
  free(coo->jc);
  free(coo->vv);
  coo->ir = coo->jc = NULL;
  coo->vv = NULL;
}

void csr_copy(csrMat *A, csrMat *B, int allocB) {
  const int nrows = A->nrows, nnz = A->ia[nrows];
  if (allocB) {
    B->owndata = 1;
    B->ia = (int *)malloc(sizeof(int) * ((size_t)nrows + 1));
    B->ja = (int *)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    B->a = (double *)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
  }
  B->nrows = nrows;
  B->ncols = A->ncols;
  B->nnz = A->nnz;
  B->descr = NULL;
  B->dBuffer = NULL;
  memcpy(B->ia, A->ia, sizeof(int) * ((size_t)nrows + 1));
  memcpy(B->ja, A->ja, sizeof(int) * (size_t)nnz);
  memcpy(B->a, A->a, sizeof(double) * (size_t)nnz);
}

int arrays_copyto_csrMat(int nrow, int ncol, int *ia, int *ja, double *a, csrMat *A) {
  const int nnz = ia[nrow];
  A->owndata = 1;
  A->nrows = nrow;
  A->ncols = ncol;
  A->nnz = nnz;
  A->descr = NULL;
  A->dBuffer = NULL;
  A->ia = (int *)malloc(sizeof(int) * ((size_t)nrow + 1));
  A->ja = (int *)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
  A->a = (double *)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
  if (!A->ia || !A->ja || !A->a) return evsl_seterr(EVSLX_ERR_NOMEM, "arrays_copyto_csrMat: out of memory");
  memcpy(A->ia, ia, sizeof(int) * ((size_t)nrow + 1));
  memcpy(A->ja, ja, sizeof(int) * (size_t)nnz);
  memcpy(A->a, a, sizeof(double) * (size_t)nnz);
  return sort_rows(nrow, A->ia, A->ja, A->a);
}

/* SRC/spmat.c:626 -- device copy of a host CSR (owndata = 2 marks device data). */
void evsl_create_csr_gpu(csrMat *Acpu, csrMat *Agpu) {
  const int n = Acpu->nrows, nnz = Acpu->ia[n];
  Agpu->owndata = 2;
  Agpu->nrows = n;
  Agpu->ncols = Acpu->ncols;
  Agpu->nnz = nnz;
  Agpu->descr = NULL;
  Agpu->dBuffer = NULL;
  Agpu->ia = (int *)_evsl_Malloc_device(sizeof(int) * ((size_t)n + 1));
  Agpu->ja = (int *)_evsl_Malloc_device(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
  Agpu->a = (double *)_evsl_Malloc_device(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
  evsl_memcpy_host_to_device(Agpu->ia, Acpu->ia, sizeof(int) * ((size_t)n + 1));
  evsl_memcpy_host_to_device(Agpu->ja, Acpu->ja, sizeof(int) * (size_t)nnz);
  evsl_memcpy_host_to_device(Agpu->a, Acpu->a, sizeof(double) * (size_t)nnz);
}

void evsl_free_csr_gpu(csrMat *csr) {
  if (!csr) return;
  if (evslh.mat_key == (const void *)csr) drop_matrix();
  if (csr->owndata) {
    _evsl_Free_device(csr->ia);
    _evsl_Free_device(csr->ja);
    _evsl_Free_device(csr->a);
  }
  csr->ia = NULL;
  csr->ja = NULL;
  csr->a = NULL;
}

/* ---------------------------------------------------------------------------
 * Memory (SRC/evsl_memory.c).  Failures print a message and return NULL
 * instead of asserting.
 * ------------------------------------------------------------------------- */
void *_evsl_Malloc(size_t nbytes) {
  void *p = malloc(nbytes ? nbytes : 1);
  if (!p) evsl_seterr(EVSLX_ERR_NOMEM, "out of host memory [%zu bytes asked]", nbytes);
  return p;
}

void *_evsl_Calloc(size_t count, size_t nbytes) {
  void *p = calloc(count ? count : 1, nbytes ? nbytes : 1);
  if (!p) evsl_seterr(EVSLX_ERR_NOMEM, "out of host memory [%zu x %zu bytes asked]", count, nbytes);
  return p;
}

void *_evsl_Realloc(void *ptr, size_t nbytes) {
  void *p = realloc(ptr, nbytes ? nbytes : 1);
  if (!p) evsl_seterr(EVSLX_ERR_NOMEM, "out of host memory [%zu bytes asked]", nbytes);
  return p;
}

void _evsl_Free(void *ptr) { free(ptr); }

void *_evsl_Malloc_device(size_t nbytes) {
  void *p = evslcu_malloc(nbytes);
  if (!p) {
    from_cu(EVSLX_ERR_NOMEM);
    fprintf(stdout, "EVSL Error: out of device memory [%zu bytes asked]\n", nbytes);
  }
  return p;
}

void *_evsl_Calloc_device(size_t count, size_t nbytes) {
  void *p = _evsl_Malloc_device(count * nbytes);
  if (p && evslcu_memset(p, 0, count * nbytes) == 0) evslcu_sync();
  return p;
}

void *_evsl_Realloc_device(void *old_ptr, size_t old_nbytes, size_t new_nbytes) {
  void *p = _evsl_Malloc_device(new_nbytes);
  if (!p) return NULL;
  if (old_ptr) {
    evslcu_d2d(p, old_ptr, old_nbytes < new_nbytes ? old_nbytes : new_nbytes);
    evslcu_free(old_ptr);
  }
  return p;
}

void _evsl_Free_device(void *ptr) {
  if (ptr) evslcu_free(ptr);
}

void evsl_memcpy_device_to_host(void *dst, void *src, size_t nbytes) { from_cu(evslcu_d2h(dst, src, nbytes)); }

void evsl_memcpy_device_to_device(void *dst, void *src, size_t nbytes) {
  if (!from_cu(evslcu_d2d(dst, src, nbytes))) evslcu_sync();
}

void evsl_memcpy_host_to_device(void *dst, void *src, size_t nbytes) { from_cu(evslcu_h2d(dst, src, nbytes)); }

void evsl_memset_device(void *ptr, int value, size_t nbytes) {
  if (!from_cu(evslcu_memset(ptr, value, nbytes))) evslcu_sync();
}

/* ---------------------------------------------------------------------------
 * Device BLAS shims (SRC/vect.c:212-284).  Scalars returned to the host are
 * read back synchronously, as with cuBLAS in host pointer mode.
 * ------------------------------------------------------------------------- */
static double *shim_scalar(void) {
  static double *d = NULL;
  if (!d) d = (double *)evslcu_malloc(sizeof(double) * 2);
  return d;
}

double evsl_dnrm2_device(int *n, double *x, int *incr) {
  double h = 0.0;
  if (*incr != 1) {
    evsl_seterr(EVSLX_ERR_UNSUPPORTED, "evsl_dnrm2_device: only unit stride");
    return 0.0;
  }
  double *d = shim_scalar();
  if (d && !evslcu_nrm2(*n, x, d)) evslcu_get_scalars(d, &h, 1);
  return h;
}

void evsl_dscal_device(int *n, double *a, double *x, int *incr) {
  if (*incr == 1) evslcu_scal(*n, *a, x);
}

double evsl_ddot_device(int *n, double *x, int *incx, double *y, int *incy) {
  double h = 0.0;
  if (*incx != 1 || *incy != 1) {
    evsl_seterr(EVSLX_ERR_UNSUPPORTED, "evsl_ddot_device: only unit stride");
    return 0.0;
  }
  double *d = shim_scalar();
  if (d && !evslcu_dot(*n, x, y, d)) evslcu_get_scalars(d, &h, 1);
  return h;
}

void evsl_daxpy_device(int *n, double *a, double *x, int *incx, double *y, int *incy) {
  if (*incx == 1 && *incy == 1) evslcu_axpy(*n, *a, x, y);
}

void evsl_dcopy_device(int *n, double *x, int *incx, double *y, int *incy) {
  if (*incx == 1 && *incy == 1) evslcu_copy(*n, x, y);
}

void evsl_dgemv_device(const char *trans, int *m, int *n, double *alpha, double *a, int *lda, double *x, int *incx,
                       double *beta, double *y, int *incy) {
  if (*incx != 1 || *incy != 1) return;
  evslcu_dgemv(*trans, *m, *n, *alpha, a, *lda, x, *beta, y);
}

void evsl_dgemm_device(const char *transa, const char *transb, int *m, int *n, int *k, double *alpha, double *a,
                       int *lda, double *b, int *ldb, double *beta, double *c, int *ldc) {
  evslcu_dgemm(*transa, *transb, *m, *n, *k, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);
}

/* ---------------------------------------------------------------------------
 * Extensions (include/evslx.h)
 * ------------------------------------------------------------------------- */
int evslx_set_filter_wave(int on) {
  evslh.wave = on ? 1 : 0;
  if (evslh.mat) return from_cu(evslcu_mat_set_wave(evslh.mat, evslh.wave));
  return 0;
}

int evslx_set_row_patterns(int on) {
  evslcu_set_row_patterns(on);
  if (evslh.mat) return from_cu(evslcu_mat_set_patterns(evslh.mat, on));
  return 0;
}

int evslx_row_pattern_count(void) { return evslh.mat ? evslcu_mat_pattern_count(evslh.mat) : 0; }

int evslx_set_filter_kernel(int variant) { return from_cu(evslcu_set_cheb_variant(variant)); }

int evslx_filter_kernel_grid(void) { return evslh.mat ? evslcu_mat_cheb_grid(evslh.mat) : 0; }

int evslx_filter_kernel(double *us) {
  float f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int v = evslh.mat ? evslcu_mat_cheb_variant(evslh.mat, f) : -1;
  if (us)
    for (int i = 0; i < 8; ++i) us[i] = f[i];
  return v;
}

int evslx_set_panel_filter(int on, int min_rows, int max_width) {
  return from_cu(evslcu_set_panels(on, min_rows, max_width));
}

int evslx_matrix_panel_layout(int fp32, int *rows_per_block, int *panel_width, long long *bytes) {
  if (!evslh.mat) return evsl_seterr(EVSLX_ERR_STATE, "no registered CSR matrix");
  return from_cu(evslcu_mat_panel_layout(evslh.mat, fp32, rows_per_block, panel_width, bytes));
}

int evslx_set_l2_resident(int on) {
  evslh.l2_resident = on ? 1 : 0;
  if (evslh.mat) return from_cu(evslcu_mat_l2_persist(evslh.mat, evslh.l2_resident));
  return 0;
}

int evslx_set_seed(uint64_t seed) {
  evslh.seed = seed;
  evslh.draw = 0;
  return 0;
}

uint64_t evslx_get_draw(void) { return evslh.draw; }

int evslx_set_spmv_kernel(int which) {
  if (which < 0 || which > 1) return evsl_seterr(EVSLX_ERR_ARG, "kernel must be 0 (SELL-32) or 1 (CSR)");
  evslh.kernel = which;
  if (evslh.mat) return from_cu(evslcu_mat_set_kernel(evslh.mat, which));
  return 0;
}

int evslx_get_spmv_kernel(void) { return evslh.mat ? evslcu_mat_get_kernel(evslh.mat) : evslh.kernel; }

int evsl_apply_A(const double *x, double *y) {
  int rc = evsl_require_operator();
  if (rc) return rc;
  if (evslh.op.A) return from_cu(evslcu_spmv(evslh.op.A, x, y));
  if ((rc = evslcu_sync())) return from_cu(rc);
  evslh.op.func((double *)x, y, evslh.op.data);
  return 0;
}

int evslx_matvec(const double *x, double *y) {
  int rc = evsl_require_operator();
  if (rc) return rc;
  if (evslh.op.A) {
    rc = evslcu_spmv(evslh.op.A, x, y);
    if (!rc) rc = evslcu_sync();
    return from_cu(rc);
  }
  evslcu_sync();
  evslh.op.func((double *)x, y, evslh.op.data);
  return 0;
}

int evslx_matvec_cols(int m, const double *X, double *Y) {
  int rc = evsl_require_operator();
  if (rc) return rc;
  if (m < 0 || (m > 0 && (!X || !Y))) return evsl_seterr(EVSLX_ERR_ARG, "evslx_matvec_cols: bad arguments");
  if (evslh.op.A) {
    rc = evslcu_spmv_cols(evslh.op.A, X, Y, m);
    if (!rc) rc = evslcu_sync();
    return from_cu(rc);
  }
  evslcu_sync();
  const size_t n = (size_t)evslh.op.n;
  for (int c = 0; c < m; c++) evslh.op.func((double *)X + (size_t)c * n, Y + (size_t)c * n, evslh.op.data);
  return 0;
}

int evslx_problem_info(int *n, long long *nnz, long long *stored) {
  if (n) *n = evslh.op.n;
  if (nnz) *nnz = evslh.op.A ? evslcu_mat_nnz(evslh.op.A) : 0;
  if (stored) *stored = evslh.op.A ? evslcu_mat_padded_nnz(evslh.op.A) : 0;
  return 0;
}

uint64_t evslx_launch_count(void) { return evslcu_launch_count(); }

double evslx_last_kpm_seconds(void) { return evslh.last_kpm_seconds; }

int evsl_rand_device(int n, int count, double *v) {
  int rc = evslcu_rand_pm1(n, count, evslh.seed, evslh.draw, v);
  evslh.draw += (uint64_t)count;
  return from_cu(rc);
}

void *evslx_stream(void) { return evslcu_stream_handle(); }

int evslx_filter_profile(int enable) { return from_cu(evslcu_filter_profile(enable)); }

int evslx_filter_stats(double *seconds, double *bytes, uint64_t *launches, uint64_t *calls) {
  return from_cu(evslcu_filter_stats(seconds, bytes, launches, calls));
}

int evslx_last_solve_info(int *lanczos_steps, int *candidates) {
  if (lanczos_steps) *lanczos_steps = evslh.last_kdim;
  if (candidates) *candidates = evslh.last_candidates;
  return 0;
}

int evslx_set_filter_persistent(int on) {
  evslh.persistent = on ? 1 : 0;
  if (evslh.mat) return from_cu(evslcu_mat_set_persistent(evslh.mat, on));
  return 0;
}

int evslx_set_matrix_compression(int on) { return from_cu(evslcu_set_compression(on)); }

int evslx_set_async_tests(int on) {
  evslh.sync_tests = on ? 0 : 1;
  return 0;
}

int evslx_set_sell_sigma(int sigma) { return from_cu(evslcu_set_sell_sigma(sigma)); }

int evslx_set_wait_limit(unsigned long long polls) { return from_cu(evslcu_set_wait_limit(polls)); }

int evslx_matrix_sell_layout(int *sigma, long long *stored, long long *stored_unsorted) {
  if (!evslh.mat) return evsl_seterr(EVSLX_ERR_STATE, "no registered CSR matrix");
  return from_cu(evslcu_mat_sell_layout(evslh.mat, sigma, stored, stored_unsorted));
}

int evslx_matrix_storage(int *value_bytes, int *index_bytes) {
  int vf = 0, xf = 0;
  if (!evslh.mat) return evsl_seterr(EVSLX_ERR_STATE, "no registered CSR matrix");
  evslcu_mat_storage(evslh.mat, &vf, &xf);
  if (value_bytes) *value_bytes = vf ? 4 : 8;
  if (index_bytes) *index_bytes = xf ? 2 : 4;
  return 0;
}

int evslx_set_filter_block(int threads) { return from_cu(evslcu_set_filter_block(threads)); }

int evslx_rand_device_draws(int n, int count, uint64_t first_draw, double *v) {
  int rc = evsl_require_started();
  if (rc) return rc;
  if (n < 1 || count < 1 || !v) return evsl_seterr(EVSLX_ERR_ARG, "rand draws: bad arguments");
  rc = evslcu_rand_pm1(n, count, evslh.seed, first_draw, v);
  if (!rc) rc = evslcu_sync();
  return from_cu(rc);
}

int evslx_set_filter_rows_per_thread(int r) { return from_cu(evslcu_set_rows_per_thread(r)); }

/*
 * engine.c -- batched and served spectrum-slicing requests.
 *
 * A request is either a slice solve (the algorithm of ChebLanNr,
 * SRC/cheblanNr.c:57-434) or a DOS estimate (kpmdos, SRC/spslice.c:29-148)
 * on a resident matrix.  The engine keeps up to max_slots slice solves in
 * flight and advances all of them by one Lanczos step per tick:
 *
 *   1. admit queued requests (FIFO) while a slot is free and the request's
 *      device memory (Lanczos basis + workspaces) fits the HBM budget; a DOS
 *      request is run to completion when admitted;
 *   2. apply every active slot's filter p_s(A) to its current Lanczos vector
 *      -- one multi-column filter per matrix, each column with its own
 *      polynomial, so A is read once per degree for all slots on it;
 *   3. the rest of the Lanczos step of each slot on the GPU (beta and alpha
 *      updates, classical Gram-Schmidt with DGKS against the slot's basis);
 *   4. one device-to-host copy of every slot's alpha and beta, then the host
 *      part of each step (tridiagonal matrix, breakdown restart, the
 *      restricted-trace convergence test every 20 steps after step 30);
 *   5. finished slots form their Ritz pairs (selected tridiagonal
 *      eigenvectors, one GEMM, Rayleigh quotients and residuals with A) and
 *      retire; their result joins the output queue.
 *
 * Precision: EVSLX_PREC_FP64 runs the filter in FP64 (each filtered vector
 * equal bit for bit to ChebAv).  EVSLX_PREC_MIXED runs the filter with FP32
 * values, vectors and accumulation; the Lanczos basis, reorthogonalisation,
 * tridiagonal solve and Ritz step stay FP64, and the Ritz pairs are then
 * refined in FP64: the candidate block -- the Ritz vectors of the m Ritz
 * values above bar plus max(16, m/2) guard vectors from the next Ritz values
 * below it -- is filtered with an FP64 filter designed (find_pol, same
 * settings) for the interval spanned by the candidates' Rayleigh quotients,
 * orthonormalised, and a Rayleigh-Ritz step with A gives the new pairs,
 * repeated while a pair inside [a, b] misses tol (at most 4 sweeps for
 * filters of degree >= 128, up to 24 for low degrees, whose sweeps are cheap
 * but damp little).  The
 * guards put the eigenvectors next to [a, b], which a filter damps weakly,
 * inside the Rayleigh-Ritz subspace; the wider interval then needs a filter
 * of lower degree (about 0.6 of the slice's) and usually one sweep.
 *
 * Every per-slot computation depends only on that slot's data (the filter
 * treats columns independently and the reductions are per slot), so a
 * request's result is the same alone and in any mix of requests.
 */
#define _POSIX_C_SOURCE 199309L
#include <time.h>

#include "internal.h"

#define ENG_NTEST 30
#define ENG_NCYCLE 20
#define ENG_MAX_SWEEPS 4
#define ENG_NSCAL 4
#define ENG_MIN_GUARDS 16
#define ENG_CGS_BLOCK 32 /* columns per block of the refinement's Gram-Schmidt */

enum { PH_START = 0, PH_LANCZOS = 1, PH_RESTART = 2 };

struct evslx_matrix {
  evslcu_mat *mat;
  evslcu_op op;
  int owned;
};

typedef struct req_s {
  int kind;
  uint64_t tag;
  evslx_matrix *M;
  double intv[4];
  polparams pol;
  int maxit;
  double tol;
  double *vinit; /* device copy */
  double *mu_dev; /* device copy of pol.mu (batched filters) */
  uint64_t seed;
  int Mdeg, damping, nvec;
  double t_submit;
  size_t bytes;
  uint64_t uid; /* unique for the engine's lifetime */
  struct req_s *next;
} req_t;

/* A captured filter (CUDA graph) for the slots of one matrix, valid while
 * the same requests occupy them in the same order. */
typedef struct {
  evslx_matrix *M;
  int ncols, used;
  uint64_t *uids;
  evslcu_filter_plan *plan;
} plan_cache_t;

typedef struct {
  req_t *req;
  double *V, *cgsw, *vrand;
  double *bw; /* 2n recurrence workspace of the batched filter */
  double *dT, *eT, *EvalT;
  int k, phase, nwn, restarts;
  double beta, wn, tr0;
  double t_start;
} slot_t;

struct evslx_engine {
  int max_slots, precision, keep_vectors;
  int mixed_min_rows; /* mixed precision only for matrices with at least this many rows */
  size_t budget, in_use;
  slot_t *slots;
  int nactive;
  req_t *qhead, *qtail;
  int nqueued;
  evslx_result *res;
  int nres, capres, reshead;
  double *ds, *hs;
  void *fwork;
  size_t fwork_bytes;
  evslcu_filter_col *cols;
  int *colslot;
  const double **xs;
  double **ys;
  uint64_t *uidbuf;
  double *gbest;
  int *gcut, *gstart;
  plan_cache_t *plans;
  int nplans;
  uint64_t next_uid;
  int use_graphs;
  uint64_t ticks, plan_builds;
  uint64_t width_hist[5]; /* filter groups launched, by block width 1, 2, 4, 8, 16 */
  /* batched filter: one-column FP64 groups of matrices with at most
   * batch_max_rows rows, filtered together (one launch per degree) */
  int use_batch, batch_max_rows;
  evslcu_batch_col *bcols;
  void *btab;
  size_t btab_bytes;
  uint64_t batched_columns;
  /* batched Lanczos step: the vector operations of all slots in the Lanczos
   * phase as one launch per operation (evslcu_lanczos_batch), and the
   * normalisations of all continuing slots as one launch */
  int use_batch_ops;
  evslcu_lz_col *lzcols;
  double *lz_npart; /* max_slots x evslcu_lz_scratch_doubles() */
  void *lztab;
  size_t lztab_bytes;
  int *sc_n;
  double **sc_x;
  double *sc_a;
  void *sctab;
  size_t sctab_bytes;
  /* host wall-clock seconds per phase of engine_step (no device syncs added):
   * [0] admission and filter issue, [1] Lanczos-step issue, [2] the wait for
   * the scalars' copy (device backlog), [3] host part, [4] retirement */
  double phase_s[5];
};

/* ---------------------------------------------------------------------------
 * resident matrices
 * ------------------------------------------------------------------------- */
evslx_matrix *evslx_matrix_create(csrMat *A, int on_device) {
  if (evsl_require_started()) return NULL;
  if (!A || A->nrows <= 0 || A->nrows != A->ncols) {
    evsl_seterr(EVSLX_ERR_ARG, "evslx_matrix_create: need a square CSR matrix");
    return NULL;
  }
  evslx_matrix *M = (evslx_matrix *)calloc(1, sizeof(evslx_matrix));
  if (!M) {
    evsl_seterr(EVSLX_ERR_NOMEM, "evslx_matrix_create: out of memory");
    return NULL;
  }
  const int n = A->nrows;
  const int nnz = on_device ? 0 : A->ia[n];
  M->mat = evslcu_mat_create(n, nnz, A->ia, A->ja, A->a, on_device);
  if (!M->mat) {
    evsl_seterr(EVSLX_ERR_ARG, "%s", evslcu_errstr());
    free(M);
    return NULL;
  }
  M->op.A = M->mat;
  M->op.func = NULL;
  M->op.data = NULL;
  M->op.n = n;
  M->owned = 1;
  return M;
}

void evslx_matrix_free(evslx_matrix *M) {
  if (!M) return;
  if (M->owned) evslcu_mat_destroy(M->mat);
  free(M);
}

long long evslx_matrix_device_bytes(const evslx_matrix *M) {
  if (!M || !M->mat) return 0;
  int vf = 0, jf = 0;
  evslcu_mat_storage(M->mat, &vf, &jf);
  const long long padded = evslcu_mat_padded_nnz(M->mat);
  return padded * ((vf ? 4 : 8) + (jf ? 2 : 4)) + 12LL * evslcu_mat_nnz(M->mat) + 4LL * (M->op.n + 1);
}

/* ---------------------------------------------------------------------------
 * engine
 * ------------------------------------------------------------------------- */
/* Below this many rows the FP32 filter saves little (the launches are latency
 * bound) and the FP64 refinement costs more than it saves, so mixed-precision
 * engines filter small matrices in FP64. */
static int g_mixed_min_rows = 131072;

void evslx_set_mixed_min_rows(int rows) { g_mixed_min_rows = rows < 0 ? 0 : rows; }

static int slot_fp32(const evslx_engine *E, const evslx_matrix *M) {
  return E->precision == EVSLX_PREC_MIXED && M->op.n >= E->mixed_min_rows;
}

evslx_engine *evslx_engine_create(int max_slots, size_t hbm_budget, int precision, int keep_vectors) {
  if (evsl_require_started()) return NULL;
  if (max_slots < 1 || (precision != EVSLX_PREC_FP64 && precision != EVSLX_PREC_MIXED)) {
    evsl_seterr(EVSLX_ERR_ARG, "evslx_engine_create: bad arguments");
    return NULL;
  }
  evslx_engine *E = (evslx_engine *)calloc(1, sizeof(evslx_engine));
  if (!E) return NULL;
  E->max_slots = max_slots;
  E->precision = precision;
  E->keep_vectors = keep_vectors;
  E->budget = hbm_budget ? hbm_budget : (size_t)-1;
  E->mixed_min_rows = g_mixed_min_rows;
  E->slots = (slot_t *)calloc((size_t)max_slots, sizeof(slot_t));
  E->ds = (double *)evslcu_malloc(sizeof(double) * ENG_NSCAL * (size_t)max_slots);
  E->hs = (double *)malloc(sizeof(double) * ENG_NSCAL * (size_t)max_slots);
  E->cols = (evslcu_filter_col *)malloc(sizeof(evslcu_filter_col) * (size_t)max_slots);
  E->colslot = (int *)malloc(sizeof(int) * (size_t)max_slots);
  E->xs = (const double **)malloc(sizeof(double *) * (size_t)max_slots);
  E->ys = (double **)malloc(sizeof(double *) * (size_t)max_slots);
  E->uidbuf = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)max_slots);
  E->gbest = (double *)malloc(sizeof(double) * ((size_t)max_slots + 1));
  E->gcut = (int *)malloc(sizeof(int) * ((size_t)max_slots + 1));
  E->gstart = (int *)malloc(sizeof(int) * ((size_t)max_slots + 1));
  E->plans = (plan_cache_t *)calloc((size_t)max_slots, sizeof(plan_cache_t));
  E->use_graphs = 1;
  E->use_batch = 1;
  E->batch_max_rows = 1 << 18;
  E->bcols = (evslcu_batch_col *)malloc(sizeof(evslcu_batch_col) * (size_t)max_slots);
  E->use_batch_ops = 1;
  E->lzcols = (evslcu_lz_col *)malloc(sizeof(evslcu_lz_col) * (size_t)max_slots);
  E->sc_n = (int *)malloc(sizeof(int) * (size_t)max_slots);
  E->sc_x = (double **)malloc(sizeof(double *) * (size_t)max_slots);
  E->sc_a = (double *)malloc(sizeof(double) * (size_t)max_slots);
  E->lztab_bytes = evslcu_lanczos_batch_table_bytes(max_slots);
  E->sctab_bytes = evslcu_scal_batch_table_bytes(max_slots);
  E->lztab = evslcu_malloc(E->lztab_bytes);
  E->sctab = evslcu_malloc(E->sctab_bytes);
  E->lz_npart = (double *)evslcu_malloc(sizeof(double) * evslcu_lz_scratch_doubles() * (size_t)max_slots);
  if (!E->slots || !E->ds || !E->hs || !E->cols || !E->colslot || !E->xs || !E->ys || !E->uidbuf || !E->plans ||
      !E->gbest || !E->gcut || !E->gstart || !E->bcols || !E->lzcols || !E->sc_n || !E->sc_x || !E->sc_a ||
      !E->lztab || !E->sctab || !E->lz_npart) {
    evsl_seterr(EVSLX_ERR_NOMEM, "evslx_engine_create: out of memory");
    evslx_engine_free(E);
    return NULL;
  }
  return E;
}

static void req_free(req_t *r) {
  if (!r) return;
  free(r->pol.mu);
  evslcu_free(r->vinit);
  evslcu_free(r->mu_dev);
  free(r);
}

static void slot_release(evslx_engine *E, slot_t *s) {
  evslcu_free(s->V);
  evslcu_free(s->cgsw);
  evslcu_free(s->vrand);
  evslcu_free(s->bw);
  free(s->dT);
  free(s->eT);
  free(s->EvalT);
  if (s->req) {
    E->in_use -= s->req->bytes;
    req_free(s->req);
  }
  memset(s, 0, sizeof(*s));
  E->nactive--;
}

void evslx_result_free(evslx_result *r) {
  if (!r) return;
  free(r->lam);
  free(r->res);
  free(r->mu);
  evslcu_free(r->Y);
  memset(r, 0, sizeof(*r));
}

void evslx_engine_free(evslx_engine *E) {
  if (!E) return;
  for (int i = 0; i < E->max_slots && E->slots; i++)
    if (E->slots[i].req) slot_release(E, &E->slots[i]);
  while (E->qhead) {
    req_t *r = E->qhead;
    E->qhead = r->next;
    req_free(r);
  }
  for (int i = 0; i < E->nres; i++) evslx_result_free(&E->res[(E->reshead + i) % E->capres]);
  free(E->res);
  free(E->slots);
  evslcu_free(E->ds);
  free(E->hs);
  evslcu_free(E->fwork);
  evslcu_free(E->btab);
  free(E->bcols);
  free(E->lzcols);
  free(E->sc_n);
  free(E->sc_x);
  free(E->sc_a);
  evslcu_free(E->lztab);
  evslcu_free(E->sctab);
  evslcu_free(E->lz_npart);
  for (int i = 0; i < E->nplans; i++) {
    evslcu_filter_plan_destroy(E->plans[i].plan);
    free(E->plans[i].uids);
  }
  free(E->plans);
  free(E->cols);
  free(E->colslot);
  free(E->xs);
  free(E->ys);
  free(E->uidbuf);
  free(E->gbest);
  free(E->gcut);
  free(E->gstart);
  free(E);
}

void evslx_engine_use_graphs(evslx_engine *E, int on) {
  if (E) E->use_graphs = on ? 1 : 0;
}

int evslx_set_batch_persistent(int on) { return evslcu_set_batch_persistent(on); }

void evslx_engine_use_batch_ops(evslx_engine *E, int on) {
  if (E) E->use_batch_ops = on ? 1 : 0;
}

void evslx_engine_use_batch(evslx_engine *E, int on, int max_rows) {
  if (!E) return;
  E->use_batch = on ? 1 : 0;
  if (max_rows > 0) E->batch_max_rows = max_rows;
}

uint64_t evslx_engine_batched_columns(const evslx_engine *E) { return E ? E->batched_columns : 0; }

uint64_t evslx_engine_plan_builds(const evslx_engine *E) { return E ? E->plan_builds : 0; }

void evslx_engine_group_widths(const evslx_engine *E, uint64_t counts[5]) {
  for (int i = 0; i < 5; i++) counts[i] = E ? E->width_hist[i] : 0;
}

/* Runs the filters of the nc columns cols (all on M, request ids uids)
 * through a cached graph when the same requests were filtered together
 * before, else captures one (or, with graphs off, launches directly). */
static int run_group_filter(evslx_engine *E, evslx_matrix *M, int nc, const evslcu_filter_col *cols,
                            const uint64_t *uids, int fp32) {
  int wb = 0;
  while ((1 << wb) < nc && wb < 4) wb++;
  E->width_hist[wb]++;
  if (nc == 1 && !fp32) {
    /* one FP64 column: the single-vector filter (per-degree launches with
     * programmatic dependent launch), bitwise the same as the block kernel */
    const size_t need = 2 * sizeof(double) * (size_t)M->op.n;
    if (need > E->fwork_bytes) {
      evslcu_free(E->fwork);
      E->fwork = evslcu_malloc(need);
      E->fwork_bytes = E->fwork ? need : 0;
      if (!E->fwork) return evsl_seterr(EVSLX_ERR_NOMEM, "engine: out of device memory (filter work)");
    }
    int rc = evslcu_chebav(&M->op, cols[0].mu, cols[0].deg, cols[0].cc, cols[0].dd, cols[0].x, cols[0].y,
                           (double *)E->fwork, NULL);
    return rc ? evsl_seterr(rc, "%s", evslcu_errstr()) : 0;
  }
  if (E->use_graphs) {
    plan_cache_t *pc = NULL;
    for (int i = 0; i < E->nplans && !pc; i++)
      if (E->plans[i].M == M && E->plans[i].ncols == nc && !memcmp(E->plans[i].uids, uids, sizeof(uint64_t) * nc))
        pc = &E->plans[i];
    if (!pc && E->nplans < E->max_slots) {
      pc = &E->plans[E->nplans];
      pc->uids = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)E->max_slots);
      if (!pc->uids) return evsl_seterr(EVSLX_ERR_NOMEM, "engine: out of memory");
      pc->plan = evslcu_filter_plan_create(M->mat, fp32, nc, cols);
      E->plan_builds++;
      if (!pc->plan) {
        free(pc->uids);
        pc->uids = NULL;
        pc = NULL;
      } else {
        pc->M = M;
        pc->ncols = nc;
        memcpy(pc->uids, uids, sizeof(uint64_t) * (size_t)nc);
        E->nplans++;
      }
    }
    if (pc) {
      pc->used = 1;
      for (int c = 0; c < nc; c++) {
        E->xs[c] = cols[c].x;
        E->ys[c] = cols[c].y;
      }
      int rc = evslcu_filter_plan_run(pc->plan, E->xs, E->ys);
      return rc ? evsl_seterr(rc, "%s", evslcu_errstr()) : 0;
    }
  }
  const size_t need = evslcu_filter_columns_work(M->op.n, fp32, nc);
  if (need > E->fwork_bytes) {
    evslcu_free(E->fwork);
    E->fwork = evslcu_malloc(need);
    E->fwork_bytes = E->fwork ? need : 0;
    if (!E->fwork) return evsl_seterr(EVSLX_ERR_NOMEM, "engine: out of device memory (filter work)");
  }
  int rc = evslcu_filter_columns(M->mat, fp32, nc, cols, E->fwork, E->fwork_bytes);
  return rc ? evsl_seterr(rc, "%s", evslcu_errstr()) : 0;
}

static int push_result(evslx_engine *E, evslx_result *r) {
  if (E->nres == E->capres) {
    const int cap = E->capres ? 2 * E->capres : 16;
    evslx_result *nr = (evslx_result *)malloc(sizeof(evslx_result) * (size_t)cap);
    if (!nr) return evsl_seterr(EVSLX_ERR_NOMEM, "engine: out of memory (results)");
    for (int i = 0; i < E->nres; i++) nr[i] = E->res[(E->reshead + i) % E->capres];
    free(E->res);
    E->res = nr;
    E->capres = cap;
    E->reshead = 0;
  }
  E->res[(E->reshead + E->nres) % E->capres] = *r;
  E->nres++;
  return 0;
}

int evslx_engine_pop_result(evslx_engine *E, evslx_result *out) {
  if (!E || !out || E->nres == 0) return 0;
  *out = E->res[E->reshead];
  E->reshead = (E->reshead + 1) % E->capres;
  E->nres--;
  return 1;
}

int evslx_engine_pending(const evslx_engine *E) { return E ? E->nqueued + E->nactive : 0; }

size_t evslx_engine_bytes_in_use(const evslx_engine *E) { return E ? E->in_use : 0; }

static void enqueue(evslx_engine *E, req_t *r) {
  r->next = NULL;
  if (E->qtail)
    E->qtail->next = r;
  else
    E->qhead = r;
  E->qtail = r;
  E->nqueued++;
}

int evslx_engine_submit_slice(evslx_engine *E, evslx_matrix *M, const double *intv, const polparams *pol, int maxit,
                              double tol, const double *vinit, int vinit_on_device, uint64_t tag) {
  if (!E || !M || !intv || !pol || !pol->mu || !vinit || maxit < 1)
    return evsl_seterr(EVSLX_ERR_ARG, "evslx_engine_submit_slice: bad arguments");
  const int n = M->op.n;
  req_t *r = (req_t *)calloc(1, sizeof(req_t));
  if (!r) return evsl_seterr(EVSLX_ERR_NOMEM, "engine: out of memory");
  r->kind = EVSLX_REQ_SLICE;
  r->tag = tag;
  r->M = M;
  memcpy(r->intv, intv, sizeof(r->intv));
  r->pol = *pol;
  r->pol.mu = (double *)malloc(sizeof(double) * (size_t)(pol->deg + 1));
  r->maxit = evsl_min(n, maxit);
  r->tol = tol;
  r->seed = tag * 0x9E3779B97F4A7C15ULL + 0x5851F42D4C957F2DULL;
  r->vinit = (double *)evslcu_malloc(sizeof(double) * (size_t)n);
  if (!r->pol.mu || !r->vinit) {
    req_free(r);
    return evsl_seterr(EVSLX_ERR_NOMEM, "engine: out of memory (request of n=%d)", n);
  }
  memcpy(r->pol.mu, pol->mu, sizeof(double) * (size_t)(pol->deg + 1));
  int rc = vinit_on_device ? evslcu_d2d(r->vinit, vinit, sizeof(double) * (size_t)n)
                           : evslcu_h2d(r->vinit, vinit, sizeof(double) * (size_t)n);
  if (rc) {
    req_free(r);
    return evsl_seterr(rc, "%s", evslcu_errstr());
  }
  r->bytes = sizeof(double) * ((size_t)n * ((size_t)r->maxit + 5) + evslcu_cgs_work_size(n, r->maxit + 1));
  r->t_submit = evsl_timer();
  r->uid = ++E->next_uid;
  enqueue(E, r);
  return 0;
}

int evslx_engine_submit_kpm(evslx_engine *E, evslx_matrix *M, int Mdeg, int damping, int nvec, const double *intv,
                            uint64_t seed, uint64_t tag) {
  if (!E || !M || !intv || Mdeg < 1 || nvec < 1)
    return evsl_seterr(EVSLX_ERR_ARG, "evslx_engine_submit_kpm: bad arguments");
  req_t *r = (req_t *)calloc(1, sizeof(req_t));
  if (!r) return evsl_seterr(EVSLX_ERR_NOMEM, "engine: out of memory");
  r->kind = EVSLX_REQ_KPM;
  r->tag = tag;
  r->M = M;
  memcpy(r->intv, intv, sizeof(r->intv));
  r->Mdeg = Mdeg;
  r->damping = damping;
  r->nvec = nvec;
  r->seed = seed;
  r->bytes = sizeof(double) * 4 * (size_t)M->op.n * (size_t)evsl_min(nvec, 64);
  r->t_submit = evsl_timer();
  r->uid = ++E->next_uid;
  enqueue(E, r);
  return 0;
}

/* ---- DOS request: kpmdos with the request's own generator stream ---- */
static int run_kpm(evslx_engine *E, req_t *r, evslx_result *out) {
  const int n = r->M->op.n;
  const int Mdeg = r->Mdeg, nvec = r->nvec;
  double *iv = r->intv;
  out->mu = (double *)calloc((size_t)Mdeg + 1, sizeof(double));
  double *dots = (double *)malloc(sizeof(double) * (size_t)Mdeg * nvec);
  double *gd = (double *)malloc(sizeof(double) * (size_t)Mdeg * evsl_min(nvec, 64));
  double *probes = (double *)evslcu_malloc(sizeof(double) * (size_t)n * evsl_min(nvec, 64));
  int rc = 0;
  if (!out->mu || !dots || !gd || !probes) rc = evsl_seterr(EVSLX_ERR_NOMEM, "engine: out of memory (DOS)");
  if (!rc && (iv[0] > iv[3] || iv[1] < iv[2])) rc = -1; /* interval outside the spectrum bounds */
  const double ctr = (iv[3] + iv[2]) / 2.0, wid = (iv[3] - iv[2]) / 2.0;
  for (int g0 = 0; !rc && g0 < nvec; g0 += 64) {
    const int cnt = evsl_min(64, nvec - g0);
    rc = evslcu_rand_pm1(n, cnt, r->seed, (uint64_t)g0, probes);
    if (!rc) rc = evslcu_kpm_dots(&r->M->op, n, Mdeg, cnt, probes, ctr, wid, gd);
    if (rc) rc = evsl_seterr(rc, "%s", evslcu_errstr());
    for (int k = 0; !rc && k < Mdeg; k++)
      for (int p = 0; p < cnt; p++) dots[(size_t)k * nvec + g0 + p] = gd[(size_t)k * cnt + p];
  }
  if (!rc) rc = evslx_kpm_accumulate(Mdeg, r->damping, nvec, n, iv, dots, out->mu, &out->ecnt);
  free(dots);
  free(gd);
  evslcu_free(probes);
  (void)E;
  return rc;
}

/* ---- admission ---- */
static int admit(evslx_engine *E) {
  while (E->qhead) {
    req_t *r = E->qhead;
    if (r->bytes > E->budget) {
      /* can never fit: fail the request instead of blocking the queue */
      E->qhead = r->next;
      if (!E->qhead) E->qtail = NULL;
      E->nqueued--;
      evslx_result out;
      memset(&out, 0, sizeof(out));
      out.tag = r->tag;
      out.kind = r->kind;
      out.rc = evsl_seterr(EVSLX_ERR_NOMEM, "engine: request needs %zu bytes, budget %zu", r->bytes, E->budget);
      out.t_submit = r->t_submit;
      out.t_start = out.t_finish = evsl_timer();
      req_free(r);
      int rc = push_result(E, &out);
      if (rc) return rc;
      continue;
    }
    if (E->in_use + r->bytes > E->budget) break;
    if (r->kind == EVSLX_REQ_SLICE && E->nactive >= E->max_slots) break;
    E->qhead = r->next;
    if (!E->qhead) E->qtail = NULL;
    E->nqueued--;
    if (r->kind == EVSLX_REQ_KPM) {
      evslx_result out;
      memset(&out, 0, sizeof(out));
      out.tag = r->tag;
      out.kind = r->kind;
      out.t_submit = r->t_submit;
      out.t_start = evsl_timer();
      E->in_use += r->bytes;
      out.rc = run_kpm(E, r, &out);
      E->in_use -= r->bytes;
      out.t_finish = evsl_timer();
      req_free(r);
      int rc = push_result(E, &out);
      if (rc) return rc;
      continue;
    }
    /* slice: an interval outside [lmin, lmax] has no eigenpairs */
    if (r->intv[0] > r->intv[3] || r->intv[1] < r->intv[2] || r->pol.gam > 1.0 || r->pol.gam < -1.0) {
      evslx_result out;
      memset(&out, 0, sizeof(out));
      out.tag = r->tag;
      out.kind = r->kind;
      out.rc = (r->pol.gam > 1.0 || r->pol.gam < -1.0) ? -1 : 0;
      out.t_submit = r->t_submit;
      out.t_start = out.t_finish = evsl_timer();
      req_free(r);
      int rc = push_result(E, &out);
      if (rc) return rc;
      continue;
    }
    slot_t *s = NULL;
    for (int i = 0; i < E->max_slots; i++)
      if (!E->slots[i].req) {
        s = &E->slots[i];
        break;
      }
    const int n = r->M->op.n;
    s->req = r;
    E->nactive++;
    E->in_use += r->bytes;
    s->V = (double *)evslcu_malloc(sizeof(double) * (size_t)n * ((size_t)r->maxit + 1));
    s->cgsw = (double *)evslcu_malloc(sizeof(double) * evslcu_cgs_work_size(n, r->maxit + 1));
    s->vrand = (double *)evslcu_malloc(sizeof(double) * (size_t)n);
    s->bw = (double *)evslcu_malloc(sizeof(double) * 2 * (size_t)n);
    r->mu_dev = (double *)evslcu_malloc(sizeof(double) * ((size_t)r->pol.deg + 1));
    if (r->mu_dev && evslcu_h2d(r->mu_dev, r->pol.mu, sizeof(double) * ((size_t)r->pol.deg + 1))) {
      evslcu_free(r->mu_dev);
      r->mu_dev = NULL;
    }
    s->dT = (double *)malloc(sizeof(double) * (size_t)r->maxit);
    s->eT = (double *)malloc(sizeof(double) * (size_t)r->maxit);
    s->EvalT = (double *)malloc(sizeof(double) * (size_t)r->maxit);
    s->phase = PH_START;
    s->t_start = evsl_timer();
    if (!s->V || !s->cgsw || !s->vrand || !s->bw || !r->mu_dev || !s->dT || !s->eT || !s->EvalT) {
      evslx_result out;
      memset(&out, 0, sizeof(out));
      out.tag = r->tag;
      out.kind = r->kind;
      out.rc = evsl_seterr(EVSLX_ERR_NOMEM, "engine: out of device memory for a basis of %d x %d", n, r->maxit + 1);
      out.t_submit = r->t_submit;
      out.t_start = out.t_finish = evsl_timer();
      slot_release(E, s);
      int rc = push_result(E, &out);
      if (rc) return rc;
    }
  }
  return 0;
}

/* ---- Ritz pairs (+ FP64 refinement in mixed precision) ---- */
static int refine_fp64(evslx_engine *E, slot_t *s, int m, double *U, double *W, double *rnorm, double *rlam,
                       double *rres, int *sweeps) {
  req_t *r = s->req;
  const int n = r->M->op.n;
  const size_t n_l = (size_t)n;
  const double aa = r->intv[0], bb = r->intv[1], tol = r->tol;
  const double slack = EVSL_DBL_EPS_MULT * DBL_EPSILON;
  double *H = (double *)malloc(sizeof(double) * (size_t)m * m);
  double *Q = (double *)malloc(sizeof(double) * (size_t)m * m);
  double *th = (double *)malloc(sizeof(double) * (size_t)m);
  double *dH = (double *)evslcu_malloc(sizeof(double) * (size_t)m * m);
  double *cgsw = (double *)evslcu_malloc(sizeof(double) * evslcu_cgs_work_size(n, m));
  evslcu_filter_col *cols = (evslcu_filter_col *)malloc(sizeof(evslcu_filter_col) * (size_t)m);
  const size_t need = evslcu_filter_columns_work(n, 0, m);
  void *fw = evslcu_malloc(need);
  int rc = 0;
  if (!H || !Q || !th || !dH || !cgsw || !cols || !fw) rc = evsl_seterr(EVSLX_ERR_NOMEM, "engine: out of memory");
  /* The refinement filter: the request's filter design over the interval
   * spanned by the candidates' Rayleigh quotients (wanted pairs and
   * guards).  The Rayleigh-Ritz step resolves every eigenvector in that
   * interval, so the filter only has to damp the rest of the spectrum, which
   * a wider interval does with a lower degree. */
  polparams pw = r->pol;
  pw.mu = NULL;
  pw.deg = 0;
  double wiv[4] = {aa, bb, r->intv[2], r->intv[3]};
  for (int j = 0; j < m; j++) {
    wiv[0] = evsl_min(wiv[0], rlam[j]);
    wiv[1] = evsl_max(wiv[1], rlam[j]);
  }
  wiv[0] = evsl_max(wiv[0], r->intv[2]);
  wiv[1] = evsl_min(wiv[1], r->intv[3]);
  if (!rc && find_pol(wiv, &pw)) rc = evsl_seterr(EVSLX_ERR_NUMERIC, "engine: refinement filter design failed");
#define CU(x)                                   \
  if ((rc = (x))) {                             \
    rc = evsl_seterr(rc, "%s", evslcu_errstr()); \
    break;                                      \
  }
  /* a sweep costs (m + guards) x degree column-degree steps; low-degree
   * filters damp little per sweep but are cheap, so they get more sweeps */
  const int max_sweeps = evsl_max(ENG_MAX_SWEEPS, evsl_min(24, (ENG_MAX_SWEEPS * 128 + pw.deg - 1) / evsl_max(pw.deg, 1)));
  for (*sweeps = 0; !rc && *sweeps < max_sweeps; (*sweeps)++) {
    int missing = 0;
    for (int j = 0; j < m; j++)
      if (rlam[j] >= aa - slack && rlam[j] <= bb + slack && !(rres[j] < tol)) missing++;
    if (!missing) break;
    /* W = p(A) U in FP64 */
    for (int j = 0; j < m; j++) {
      cols[j].mu = pw.mu;
      cols[j].deg = pw.deg;
      cols[j].cc = pw.cc;
      cols[j].dd = pw.dd;
      cols[j].x = U + (size_t)j * n_l;
      cols[j].y = W + (size_t)j * n_l;
    }
    CU(evslcu_filter_columns(r->M->mat, 0, m, cols, fw, need));
    /* orthonormalise W in place: block Gram-Schmidt twice (GEMM projections
     * against the earlier blocks), CGS + DGKS inside each block */
    double *ds = E->ds + ENG_NSCAL * (size_t)(s - E->slots);
    CU(evslcu_block_cgs2(n, m, W, ENG_CGS_BLOCK, dH, ds + 3, cgsw));
    /* U = A W; H = W' A W (symmetrised on the host); eigenpairs; U = W Q */
    CU(evslcu_spmv_cols(r->M->mat, W, U, m));
    CU(evslcu_dgemm('T', 'N', m, m, n, 1.0, W, n, U, n, 0.0, dH, m));
    CU(evslcu_d2h(H, dH, sizeof(double) * (size_t)m * m));
    for (int i = 0; i < m; i++)
      for (int j = 0; j < i; j++) {
        const double v = 0.5 * (H[i + (size_t)j * m] + H[j + (size_t)i * m]);
        H[i + (size_t)j * m] = H[j + (size_t)i * m] = v;
      }
    if ((rc = evsl_sym_eig(m, H, m, Q, m, th))) break;
    CU(evslcu_h2d(dH, Q, sizeof(double) * (size_t)m * m));
    CU(evslcu_dgemm('N', 'N', n, m, m, 1.0, W, n, dH, m, 0.0, U, n));
    CU(evslcu_ritz_eval(&r->M->op, n, m, U, W, rnorm, rlam, rres));
  }
#undef CU
  free_pol(&pw);
  free(H);
  free(Q);
  free(th);
  free(cols);
  evslcu_free(dH);
  evslcu_free(cgsw);
  evslcu_free(fw);
  return rc;
}

static int finalize(evslx_engine *E, slot_t *s, int kdim, evslx_result *out) {
  req_t *r = s->req;
  const int n = r->M->op.n;
  const size_t n_l = (size_t)n;
  const double aa = r->intv[0], bb = r->intv[1], bar = r->pol.bar;
  const double slack = EVSL_DBL_EPS_MULT * DBL_EPSILON;
  int rc = 0, msel = 0, nev = 0;
  int *sel = (int *)malloc(sizeof(int) * (size_t)(kdim > 0 ? kdim : 1));
  double *wsel = (double *)malloc(sizeof(double) * (size_t)(kdim > 0 ? kdim : 1));
  double *EvecT = NULL, *EvecT_dev = NULL, *Rvec = NULL, *W = NULL, *rnorm = NULL;
  int *keep = NULL;
  if (!sel || !wsel) {
    rc = evsl_seterr(EVSLX_ERR_NOMEM, "engine: out of memory");
    goto done;
  }
  /* s->EvalT holds the eigenvalues of T_kdim from the convergence test that
   * ended the solve, those below bar only where they may reach it; the
   * FP32 path's guard vectors need the ones below bar: all of them again */
  if (slot_fp32(E, r->M) && (rc = evsl_trid_eigvals(kdim, s->dT, s->eT, s->EvalT))) goto done;
  for (int i = 0; i < kdim; i++)
    if (s->EvalT[i] >= bar) {
      wsel[msel] = s->EvalT[i];
      sel[msel++] = i;
    }
  if (msel == 0) goto done;
  if (slot_fp32(E, r->M)) {
    /* guard vectors for the refinement: the Ritz vectors of the next largest
     * Ritz values below bar, so that the eigenvectors just outside [a, b]
     * are resolved by the Rayleigh-Ritz step instead of damped by the
     * filter (whose damping is weak next to the interval) */
    const int g = evsl_min(kdim - msel, evsl_max(ENG_MIN_GUARDS, (msel + 1) / 2));
    const int first = sel[0];
    for (int i = msel - 1; i >= 0; i--) {
      sel[g + i] = sel[i];
      wsel[g + i] = wsel[i];
    }
    for (int i = 0; i < g; i++) {
      sel[i] = first - g + i;
      wsel[i] = s->EvalT[first - g + i];
    }
    msel += g;
  }
  EvecT = (double *)malloc(sizeof(double) * (size_t)kdim * msel);
  EvecT_dev = (double *)evslcu_malloc(sizeof(double) * (size_t)kdim * msel);
  Rvec = (double *)evslcu_malloc(sizeof(double) * n_l * msel);
  W = (double *)evslcu_malloc(sizeof(double) * n_l * msel);
  rnorm = (double *)malloc(sizeof(double) * 3 * (size_t)msel);
  keep = (int *)malloc(sizeof(int) * (size_t)msel);
  out->lam = (double *)malloc(sizeof(double) * (size_t)msel);
  out->res = (double *)malloc(sizeof(double) * (size_t)msel);
  if (!EvecT || !EvecT_dev || !Rvec || !W || !rnorm || !keep || !out->lam || !out->res) {
    rc = evsl_seterr(EVSLX_ERR_NOMEM, "engine: out of memory for %d Ritz vectors", msel);
    goto done;
  }
  double *rlam = rnorm + msel, *rres = rlam + msel;
  if ((rc = evsl_trid_eigvecs(kdim, s->dT, s->eT, msel, wsel, EvecT, kdim))) goto done;
  if ((rc = evslcu_h2d(EvecT_dev, EvecT, sizeof(double) * (size_t)kdim * msel)) ||
      (rc = evslcu_dgemm('N', 'N', n, msel, kdim, 1.0, s->V, n, EvecT_dev, kdim, 0.0, Rvec, n)) ||
      (rc = evslcu_ritz_eval(&r->M->op, n, msel, Rvec, W, rnorm, rlam, rres))) {
    rc = evsl_seterr(rc, "%s", evslcu_errstr());
    goto done;
  }
  for (int j = 0; j < msel; j++)
    if (rnorm[j] == 0.0) {
      rc = 2; /* zero Ritz vector */
      goto done;
    }
  if (slot_fp32(E, r->M)) {
    evslcu_free(EvecT_dev);
    EvecT_dev = NULL;
    if ((rc = refine_fp64(E, s, msel, Rvec, W, rnorm, rlam, rres, &out->refine_sweeps))) goto done;
  }
  for (int j = 0; j < msel; j++) {
    const double lam = rlam[j];
    if (lam < aa - slack || lam > bb + slack) continue;
    if (rres[j] < r->tol) {
      out->lam[nev] = lam;
      out->res[nev] = rres[j];
      keep[nev++] = j;
    }
  }
  if (E->keep_vectors && nev > 0) {
    if ((rc = evslcu_gather_cols(n, nev, keep, Rvec, Rvec))) {
      rc = evsl_seterr(rc, "%s", evslcu_errstr());
      goto done;
    }
    out->Y = Rvec;
    Rvec = NULL;
  }
done:
  out->nev = nev;
  free(sel);
  free(wsel);
  free(EvecT);
  free(rnorm);
  free(keep);
  evslcu_free(EvecT_dev);
  evslcu_free(Rvec);
  evslcu_free(W);
  if (nev == 0) {
    free(out->lam);
    free(out->res);
    out->lam = out->res = NULL;
  }
  return rc;
}

static int retire(evslx_engine *E, slot_t *s, int kdim, int rc_in) {
  evslx_result out;
  memset(&out, 0, sizeof(out));
  req_t *r = s->req;
  out.tag = r->tag;
  out.kind = r->kind;
  out.t_submit = r->t_submit;
  out.t_start = s->t_start;
  out.lanczos_steps = kdim;
  out.rc = rc_in ? rc_in : finalize(E, s, kdim, &out);
  out.t_finish = evsl_timer();
  slot_release(E, s);
  return push_result(E, &out);
}

/* one tick: admit, filter every active slot, Lanczos step, tests, retire */
static double eng_clock(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

void evslx_engine_phase_times(const evslx_engine *E, double out[5]) {
  for (int i = 0; i < 5; i++) out[i] = E ? E->phase_s[i] : 0.0;
}

int evslx_engine_step(evslx_engine *E) {
  if (!E) return evsl_seterr(EVSLX_ERR_ARG, "evslx_engine_step: null engine");
  double tph = eng_clock();
  int rc = admit(E);
  if (rc) return rc;
  if (E->nactive == 0) return evslx_engine_pending(E);
  /* 1. filters: the active slots of each matrix, in order of decreasing
   * degree, are cut into groups of at most 16 columns (a group runs to its
   * largest degree) by the measured cost of each width; each group is one
   * captured multi-column filter. */
  for (int i = 0; i < E->nplans; i++) E->plans[i].used = 0;
  for (int i = 0; i < E->max_slots; i++) E->colslot[i] = -1;
  int nbatch = 0;
  long long batch_rows = 0;
  evslx_matrix *batch_M = NULL;
  evslcu_filter_col batch_col;
  uint64_t batch_uid = 0;
  for (int i = 0; i < E->max_slots; i++) {
    slot_t *s0 = &E->slots[i];
    if (!s0->req || E->colslot[i] >= 0) continue;
    evslx_matrix *M = s0->req->M;
    const int fp32 = slot_fp32(E, M);
    int nc = 0;
    for (int j = i; j < E->max_slots; j++) {
      slot_t *t = &E->slots[j];
      if (!t->req || t->req->M != M) continue;
      const size_t n_l = (size_t)M->op.n;
      const polparams *p = &t->req->pol;
      evslcu_filter_col *c = &E->cols[nc];
      c->mu = p->mu;
      c->deg = p->deg;
      c->cc = p->cc;
      c->dd = p->dd;
      if (t->phase == PH_START) {
        c->x = t->req->vinit;
        c->y = t->V;
      } else if (t->phase == PH_RESTART) {
        c->x = t->vrand;
        c->y = t->V + (size_t)(t->k + 1) * n_l;
      } else {
        c->x = t->V + (size_t)t->k * n_l;
        c->y = t->V + (size_t)(t->k + 1) * n_l;
      }
      E->uidbuf[nc] = t->req->uid;
      E->colslot[j] = nc++;
    }
    /* order by decreasing degree (stable, insertion sort on the small set) */
    for (int a2 = 1; a2 < nc; a2++) {
      evslcu_filter_col cv = E->cols[a2];
      const uint64_t uv = E->uidbuf[a2];
      int b2 = a2 - 1;
      while (b2 >= 0 && E->cols[b2].deg < cv.deg) {
        E->cols[b2 + 1] = E->cols[b2];
        E->uidbuf[b2 + 1] = E->uidbuf[b2];
        b2--;
      }
      E->cols[b2 + 1] = cv;
      E->uidbuf[b2 + 1] = uv;
    }
    if (fp32 && (rc = evslcu_mat_prepare_fp32(M->mat))) return evsl_seterr(rc, "%s", evslcu_errstr());
    /* a lone FP64 column of a small matrix joins the batched filter: the
     * columns of all such matrices advance one degree per launch together */
    if (E->use_batch && nc == 1 && !fp32 && M->op.n <= E->batch_max_rows) {
      slot_t *t = &E->slots[i];
      evslcu_batch_col *b = &E->bcols[nbatch++];
      b->A = M->mat;
      b->mu = t->req->mu_dev;
      b->deg = E->cols[0].deg;
      b->cc = E->cols[0].cc;
      b->dd = E->cols[0].dd;
      b->x = E->cols[0].x;
      b->y = E->cols[0].y;
      b->w = t->bw;
      batch_rows += M->op.n;
      batch_M = M;
      batch_col = E->cols[0];
      batch_uid = E->uidbuf[0];
      evslstat.n_polAv += nc;
      continue;
    }
    /* groups: contiguous runs of the degree-sorted columns chosen to minimise
     * sum over groups of (largest degree) x (measured time of one degree step
     * at that width) -- the autotuner's timings for this matrix */
    double cost[17];
    int have_cost = 1;
    for (int b = 1; b <= 16 && have_cost; b++) {
      cost[b] = evslcu_filter_step_cost(M->mat, fp32, b);
      if (cost[b] <= 0.0) have_cost = 0;
    }
    /* one-column FP64 groups run the single-vector filter (run_group_filter) */
    if (have_cost && !fp32) {
      const double c1 = evslcu_chebav_step_cost(M->mat);
      if (c1 > 0.0) cost[1] = c1;
    }
    int ng = 0;
    if (have_cost) {
      double *best = E->gbest;
      int *cut = E->gcut;
      best[0] = 0.0;
      for (int i2 = 1; i2 <= nc; i2++) {
        best[i2] = 1e300;
        for (int g = 1; g <= 16 && g <= i2; g++) {
          const int j2 = i2 - g;
          const double v = best[j2] + (double)E->cols[j2].deg * cost[g];
          if (v < best[i2]) {
            best[i2] = v;
            cut[i2] = j2;
          }
        }
      }
      for (int i2 = nc; i2 > 0; i2 = cut[i2]) E->gstart[ng++] = cut[i2];
    } else {
      for (int g0 = 0; g0 < nc;) {
        int g1 = g0 + 1;
        while (g1 < nc && g1 - g0 < 16 && 2 * E->cols[g1].deg >= E->cols[g0].deg) g1++;
        E->gstart[ng++] = g0;
        g0 = g1;
      }
      for (int a3 = 0, b3 = ng - 1; a3 < b3; a3++, b3--) {
        const int t3 = E->gstart[a3];
        E->gstart[a3] = E->gstart[b3];
        E->gstart[b3] = t3;
      }
    }
    /* gstart holds the group starts in decreasing order (DP) or increasing
     * order (fallback, reversed above to decreasing) */
    for (int gi = 0; gi < ng; gi++) {
      const int g0 = E->gstart[gi];
      const int g1 = (gi == 0) ? nc : E->gstart[gi - 1];
      if ((rc = run_group_filter(E, M, g1 - g0, E->cols + g0, E->uidbuf + g0, fp32))) return rc;
    }
    evslstat.n_polAv += nc;
  }
  if (nbatch == 1) {
    /* a batch of one: the single-vector filter (its kernel tuned for the matrix) */
    if ((rc = run_group_filter(E, batch_M, 1, &batch_col, &batch_uid, 0))) return rc;
  } else if (nbatch > 1) {
    const size_t need = evslcu_filter_batch_table_bytes(nbatch, batch_rows);
    if (need > E->btab_bytes) {
      evslcu_free(E->btab);
      E->btab = evslcu_malloc(need);
      E->btab_bytes = E->btab ? need : 0;
      if (!E->btab) return evsl_seterr(EVSLX_ERR_NOMEM, "engine: out of device memory (batch table)");
    }
    if ((rc = evslcu_filter_batch(nbatch, E->bcols, E->btab, E->btab_bytes))) return evsl_seterr(rc, "%s", evslcu_errstr());
    E->batched_columns += (uint64_t)nbatch;
  }
  /* drop the captured filters no group used in this tick */
  for (int i = 0; i < E->nplans;) {
    if (E->plans[i].used) {
      i++;
      continue;
    }
    evslcu_filter_plan_destroy(E->plans[i].plan);
    free(E->plans[i].uids);
    E->plans[i] = E->plans[--E->nplans];
    memset(&E->plans[E->nplans], 0, sizeof(plan_cache_t));
  }
  {
    const double t = eng_clock();
    E->phase_s[0] += t - tph;
    tph = t;
  }
  /* 2. device part of the Lanczos step */
  int nlz = 0;
  for (int i = 0; i < E->max_slots; i++) {
    slot_t *s = &E->slots[i];
    if (!s->req) continue;
    const int n = s->req->M->op.n;
    const size_t n_l = (size_t)n;
    double *ds = E->ds + ENG_NSCAL * (size_t)i;
    if (s->phase == PH_START) {
      if ((rc = evslcu_nrm2(n, s->V, ds + 1)) || (rc = evslcu_scal_inv_ds(n, ds + 1, s->V))) break;
    } else if (s->phase == PH_LANCZOS && E->use_batch_ops) {
      evslcu_lz_col *c = &E->lzcols[nlz++];
      c->n = n;
      c->k = s->k;
      c->beta = s->beta;
      c->V = s->V;
      c->ds = ds;
      c->cgsw = s->cgsw;
      c->npart = E->lz_npart + evslcu_lz_scratch_doubles() * (size_t)i;
    } else if (s->phase == PH_LANCZOS) {
      double *v = s->V + (size_t)s->k * n_l, *z = v + n_l;
      if (s->k > 0 && (rc = evslcu_axpy(n, -s->beta, v - n_l, z))) break;
      if ((rc = evslcu_dot(n, z, v, ds)) || (rc = evslcu_axpy_ds(n, ds, -1.0, v, z)) ||
          (rc = evslcu_cgs_dgks(n, s->k + 1, EVSL_NGS_MAX, s->V, (long long)n, z, ds + 1, s->cgsw)))
        break;
    } else {
      double *z = s->V + (size_t)(s->k + 1) * n_l;
      if ((rc = evslcu_cgs_dgks(n, s->k + 1, EVSL_NGS_MAX, s->V, (long long)n, z, ds + 1, s->cgsw)) ||
          (rc = evslcu_scal_inv_ds(n, ds + 1, z)))
        break;
    }
  }
  if (!rc && nlz > 0) rc = evslcu_lanczos_batch(nlz, E->lzcols, EVSL_NGS_MAX, E->lztab, E->lztab_bytes);
  if (rc) return evsl_seterr(rc, "%s", evslcu_errstr());
  {
    const double t = eng_clock();
    E->phase_s[1] += t - tph;
    tph = t;
  }
  /* 3. one copy of every slot's scalars */
  if ((rc = evslcu_d2h(E->hs, E->ds, sizeof(double) * ENG_NSCAL * (size_t)E->max_slots)))
    return evsl_seterr(rc, "%s", evslcu_errstr());
  {
    const double t = eng_clock();
    E->phase_s[2] += t - tph;
    tph = t;
  }
  /* 4. host part of the step */
  int nsc = 0;
  for (int i = 0; i < E->max_slots; i++) {
    slot_t *s = &E->slots[i];
    if (!s->req) continue;
    req_t *r = s->req;
    const int n = r->M->op.n;
    const double *h = E->hs + ENG_NSCAL * (size_t)i;
    int step_done = 0;
    if (s->phase == PH_START) {
      s->phase = PH_LANCZOS;
      s->k = 0;
      continue;
    } else if (s->phase == PH_LANCZOS) {
      const double alpha = h[0];
      const double beta = h[1];
      s->dT[s->k] = alpha;
      s->wn += fabs(alpha) + 2.0 * beta;
      s->nwn += 3;
      if (beta * s->nwn < EVSL_ORTH_TOL * s->wn) {
        /* lucky breakdown: restart from a new filtered random vector */
        if ((rc = evslcu_rand_pm1(n, 1, r->seed, (uint64_t)s->restarts++, s->vrand)))
          return evsl_seterr(rc, "%s", evslcu_errstr());
        s->phase = PH_RESTART;
        continue;
      }
      s->beta = beta;
      if (E->use_batch_ops) {
        E->sc_n[nsc] = n;
        E->sc_x[nsc] = s->V + (size_t)(s->k + 1) * (size_t)n;
        E->sc_a[nsc] = 1.0 / beta;
        nsc++;
      } else if ((rc = evslcu_scal(n, 1.0 / beta, s->V + (size_t)(s->k + 1) * (size_t)n))) {
        return evsl_seterr(rc, "%s", evslcu_errstr());
      }
      s->eT[s->k] = beta;
      step_done = 1;
    } else {
      s->beta = 0.0;
      s->eT[s->k] = 0.0;
      s->phase = PH_LANCZOS;
      step_done = 1;
    }
    if (!step_done) continue;
    const int k = s->k;
    int finished = 0, kdim = k + 1;
    if (!((k < ENG_NTEST || (k - ENG_NTEST) % ENG_NCYCLE != 0) && k != r->maxit - 1)) {
      if ((rc = evsl_trid_eigvals_test(kdim, s->dT, s->eT, r->pol.bar - EVSL_DBL_EPS_MULT * DBL_EPSILON,
                                        s->EvalT)))
        return rc;
      double tr1 = 0.0;
      for (int j = 0; j < kdim; j++)
        if (s->EvalT[j] + EVSL_DBL_EPS_MULT * DBL_EPSILON >= r->pol.bar) tr1 += s->EvalT[j];
      if ((fabs(tr1 - s->tr0) < 2e-12) || (fabs(tr1) + fabs(s->tr0) < 1e-10)) finished = 1;
      s->tr0 = tr1;
    }
    if (!finished && k + 1 >= r->maxit) finished = 1;
    if (finished) {
      const double tr = eng_clock();
      /* the queued normalisations first: retiring releases this slot's basis */
      if (nsc > 0 && (rc = evslcu_scal_batch(nsc, E->sc_n, E->sc_x, E->sc_a, E->sctab, E->sctab_bytes)))
        return evsl_seterr(rc, "%s", evslcu_errstr());
      nsc = 0;
      if ((rc = retire(E, s, kdim, 0))) return rc;
      E->phase_s[4] += eng_clock() - tr;
      tph += eng_clock() - tr;  /* keep retirement out of the host-part time */
    } else {
      s->k = k + 1;
    }
  }
  if (nsc > 0 && (rc = evslcu_scal_batch(nsc, E->sc_n, E->sc_x, E->sc_a, E->sctab, E->sctab_bytes)))
    return evsl_seterr(rc, "%s", evslcu_errstr());
  E->phase_s[3] += eng_clock() - tph;
  E->ticks++;
  return evslx_engine_pending(E);
}

int evslx_engine_run(evslx_engine *E) {
  int rc;
  while ((rc = evslx_engine_step(E)) > 0) {
  }
  return rc < 0 ? rc : 0;
}

/* ---------------------------------------------------------------------------
 * several slices of the registered matrix in one batch
 * ------------------------------------------------------------------------- */
int evslx_ChebLanNr_batch(int nslices, double *intvs, int maxit, double tol, double *vinit, polparams *pols,
                          int precision, int *nevOut, double **lamo, double **Wo, double **reso) {
  int rc = evsl_require_operator();
  if (rc) return rc;
  if (nslices < 1 || !intvs || !vinit || !pols || !nevOut || !lamo || !Wo || !reso)
    return evsl_seterr(EVSLX_ERR_ARG, "evslx_ChebLanNr_batch: bad arguments");
  if (!evsl_op()->A) return evsl_seterr(EVSLX_ERR_UNSUPPORTED, "evslx_ChebLanNr_batch needs a CSR matrix (SetAMatrix)");
  evslx_matrix M;
  memset(&M, 0, sizeof(M));
  M.mat = (evslcu_mat *)evsl_op()->A;
  M.op = *evsl_op();
  M.owned = 0;
  evslx_engine *E = evslx_engine_create(nslices, 0, precision, 1);
  if (!E) return EVSLX_ERR_NOMEM;
  for (int s = 0; s < nslices && !rc; s++) {
    nevOut[s] = 0;
    lamo[s] = Wo[s] = reso[s] = NULL;
    rc = evslx_engine_submit_slice(E, &M, intvs + 4 * s, &pols[s], maxit, tol, vinit, 1, (uint64_t)s);
  }
  if (!rc) rc = evslx_engine_run(E);
  evslx_result out;
  while (evslx_engine_pop_result(E, &out)) {
    const int s = (int)out.tag;
    if (out.rc && !rc) rc = out.rc;
    nevOut[s] = out.nev;
    lamo[s] = out.lam;
    reso[s] = out.res;
    Wo[s] = out.Y;
  }
  evslx_engine_free(E);
  return rc;
}

/* ---------------------------------------------------------------------------
 * multi-column filter on the registered matrix
 * ------------------------------------------------------------------------- */
int evslx_chebav_multi(int ncols, const polparams *pols, const double *X, double *Y, int precision) {
  int rc = evsl_require_operator();
  if (rc) return rc;
  if (ncols < 1 || !pols || !X || !Y || (precision != EVSLX_PREC_FP64 && precision != EVSLX_PREC_MIXED))
    return evsl_seterr(EVSLX_ERR_ARG, "evslx_chebav_multi: bad arguments");
  evslcu_mat *A = (evslcu_mat *)evsl_op()->A;
  if (!A) return evsl_seterr(EVSLX_ERR_UNSUPPORTED, "evslx_chebav_multi needs a CSR matrix (SetAMatrix)");
  const int n = evsl_op()->n, fp32 = (precision == EVSLX_PREC_MIXED);
  evslcu_filter_col *cols = (evslcu_filter_col *)malloc(sizeof(evslcu_filter_col) * (size_t)ncols);
  if (!cols) return evsl_seterr(EVSLX_ERR_NOMEM, "evslx_chebav_multi: out of memory");
  for (int c = 0; c < ncols; c++) {
    cols[c].mu = pols[c].mu;
    cols[c].deg = pols[c].deg;
    cols[c].cc = pols[c].cc;
    cols[c].dd = pols[c].dd;
    cols[c].x = X + (size_t)c * n;
    cols[c].y = Y + (size_t)c * n;
  }
  const size_t need = evslcu_filter_columns_work(n, fp32, ncols);
  void *w = evslcu_malloc(need);
  if (!w) rc = EVSLCU_ERR_NOMEM;
  if (!rc && fp32) rc = evslcu_mat_prepare_fp32(A);
  if (!rc) rc = evslcu_filter_columns(A, fp32, ncols, cols, w, need);
  if (!rc) rc = evslcu_sync();
  evslcu_free(w);
  free(cols);
  if (rc) return evsl_seterr(rc, "%s", evslcu_errstr());
  evslstat.n_polAv += ncols;
  return 0;
}

int evslx_set_filter_variant(int v) {
  int rc = evslcu_set_filter_variant(v);
  return rc ? evsl_seterr(rc, "%s", evslcu_errstr()) : 0;
}

int evslx_get_filter_variant(void) { return evslcu_get_filter_variant(); }

int evslx_set_split_range_bytes(long long bytes) {
  int rc = evslcu_set_xs_range_bytes(bytes);
  return rc ? evsl_seterr(rc, "%s", evslcu_errstr()) : 0;
}

int evslx_tuned_filter_variant(int precision, int ncols) {
  if (evsl_require_operator() || !evsl_op()->A) return -1;
  int B = 1;
  while (B < ncols && B < 16) B *= 2;
  return evslcu_mat_filter_variant(evsl_op()->A, precision == EVSLX_PREC_MIXED, B);
}

/*
 * chebpoly.c -- Chebyshev polynomial filter: design (host, FP64 scalar work)
 * and application (GPU).
 *
 * Design follows the reference's SRC/chebpoly.c:
 *   set_pol_def  :15-24    defaults
 *   dampcf       :39-66    Jackson / Lanczos-sigma damping coefficients
 *   dif_eval     :78-84    p(theta) difference used for balancing
 *   chebxPltd    :105-135  evaluation of a Chebyshev series at points
 *   chext        :170-259  end-interval filter (scaled Chebyshev polynomial)
 *   rootchb      :288-336  Newton balancing of the delta-function centre
 *   find_pol     :363-490  degree loop and acceptance test
 * The arithmetic is the same sequence of double operations, so the designed
 * filter (degree, coefficients, gam, bar) is identical to the reference's.
 *
 * Application ChebAv (:519-598) runs on the GPU through evslcu_chebav: one
 * fused kernel per degree (SpMV + three-term recurrence + accumulation).
 */
#include "internal.h"

#include <pthread.h>
#include <unistd.h>

void set_pol_def(polparams *pol) {
  pol->max_deg = 10000;
  pol->min_deg = 2;
  pol->damping = 2;
  pol->thresh_ext = 0.20;
  pol->thresh_int = 0.8;
  pol->mu = NULL;
  pol->deg = 0;
  pol->intvtol = 1e-9;
}

int dampcf(int m, int damping, double *jac) {
  const double dm = (double)m;
  double thetJ = 0.0, thetL = 0.0, a1 = 0.0, a2 = 0.0;
  if (damping == 1) {
    thetJ = EVSL_PI / (dm + 2);
    a1 = 1 / (dm + 2);
    a2 = sin(thetJ);
  }
  if (damping == 2) thetL = EVSL_PI / (dm + 1);
  /* jac[0] = 1/2 carries the factor of the zeroth Chebyshev term */
  jac[0] = 0.5;
  for (int k = 1; k <= m; k++) {
    if (damping == 0) {
      jac[k] = 1.0;
    } else if (damping == 1) {
      const int k1 = k + 1;
      jac[k] = a1 * sin(k1 * thetJ) / a2 + (1 - k1 * a1) * cos(k * thetJ);
    } else {
      jac[k] = sin(k * thetL) / (k * thetL);
    }
  }
  return 0;
}

static double dif_eval(const double *v, int m, double thc, const double *jac) {
  double f = 0.0;
  for (int j = 0; j <= m; j++) f += v[j] * cos(j * thc) * jac[j];
  return f;
}

/* y_i = sum_k mu_k T_k(x_i) by the three-term recurrence. */
static void cheb_series(int m, const double *mu, int npts, const double *x, double *y) {
  for (int i = 0; i < npts; i++) {
    double tkm1 = 0.0, tk = 1.0, acc = mu[0];
    for (int k = 0; k < m; k++) {
      const double scal = (k == 0) ? 1.0 : 2.0;
      const double tkp1 = scal * x[i] * tk - tkm1;
      tkm1 = tk;
      tk = tkp1;
      acc += mu[k + 1] * tk;
    }
    y[i] = acc;
  }
}

/* End-interval filter: a Chebyshev polynomial of [a,b] scaled to 1 at gam,
 * re-expanded in the Chebyshev basis of [-1,1] degree by degree. */
static int chext(polparams *pol, double aIn, double bIn) {
  int max_deg = pol->max_deg;
  double thresh = pol->thresh_ext;
  double *mu = pol->mu;
  const double del = 0.1 * sqrt((bIn - aIn) * 0.5);
  const double eps = 1e-13;
  double a, b, x, gam;
  if (pol->deg > 0) {
    thresh = -1.0;
    max_deg = pol->deg;
  }
  if (bIn >= (1.0 - eps)) {
    x = aIn;
    b = x - del;
    a = -1.0;
    gam = 1.0;
  } else {
    x = bIn;
    a = x + del;
    b = 1.0;
    gam = -1.0;
  }
  const double e = (b - a) * 0.5, c = (b + a) * 0.5;
  const double sigma1 = e / (gam - c);
  double sigma = sigma1;
  const int m1 = max_deg + 1;
  double *t0 = (double *)calloc(3 * (size_t)m1, sizeof(double));
  if (!t0) return evsl_seterr(EVSLX_ERR_NOMEM, "find_pol: out of memory");
  double *t1 = t0 + m1, *tnew = t1 + m1;
  t0[0] = 1.0;
  t1[0] = -c * (sigma1 / e);
  t1[1] = (sigma1 / e);
  double g0 = 1.0, g1 = (x - c) * sigma1 / e;
  int mbest = 0;
  if (g1 < thresh) {
    mbest = 1;
  } else {
    for (int k = 2; k <= max_deg; k++) {
      const double sigma_new = 1.0 / (2.0 / sigma1 - sigma);
      const double s1 = sigma_new / e, s2 = 2 * s1 * c, s3 = sigma * sigma_new;
      for (int j = 2; j <= k; j++) tnew[j - 1] = s1 * (t1[j] + t1[j - 2]);
      tnew[1] = tnew[1] + s1 * t1[0];
      tnew[0] = s1 * t1[1];
      tnew[k] = s1 * t1[k - 1];
      for (int j = 0; j <= k; j++) tnew[j] = tnew[j] - s2 * t1[j] - s3 * t0[j];
      for (int j = 0; j <= k; j++) {
        t0[j] = t1[j];
        t1[j] = tnew[j];
      }
      const double gnew = 2 * (x - c) * s1 * g1 - s3 * g0;
      g0 = g1;
      g1 = gnew;
      mbest = k;
      if (g1 < thresh) break;
      sigma = sigma_new;
    }
  }
  memcpy(mu, t1, sizeof(double) * (size_t)(mbest + 1));
  pol->deg = mbest;
  pol->bar = g1;
  pol->gam = gam;
  free(t0);
  return 0;
}

/* Newton iteration (with bisection safeguard) for the centre theta_c that
 * balances p(a) = p(b); returns 1 if the degree is too low to balance. */
static int rootchb(int m, const double *v, const double *jac, double tha, double thb, double *mu, double *thcOut) {
  const int max_iter = 30;
  const double tolBal = fabs(tha - thb) * 1.e-13;
  double thc = 0.5 * (tha + thb);
  const double fb = dif_eval(v, m, thb, jac);
  const double fa = dif_eval(v, m, tha, jac);
  if ((fa > 0) || (fb < 0)) return 1;
  for (int it = 0; it <= max_iter; it++) {
    const double fval = dif_eval(v, m, thc, jac);
    double d = 0.0;
    for (int j = 1; j <= m; j++) d += jac[j] * j * sin(j * (thc)) * v[j];
    double thN = thc + fval / d;
    if ((fabs(fval) < tolBal) || fabs(thc - thN) < DBL_EPSILON * fabs(thc)) break;
    if (fval > 0) {
      if ((thN < thb) || (thN > tha)) thN = 0.5 * (thc + tha);
      thb = thc;
      thc = thN;
    } else {
      if ((thN < thb) || (thN > tha)) thN = 0.5 * (thc + thb);
      tha = thc;
      thc = thN;
    }
  }
  for (int j = 0; j <= m; j++) mu[j] = cos(j * (thc)) * jac[j];
  *thcOut = thc;
  return 0;
}

/* One candidate degree m of the mid-interval design: damping, balance,
 * peak and end values (each candidate is independent of the others). */
typedef struct {
  int skip, pass;
} fp_result;

static fp_result fp_candidate(int m, int damping, const double *v, double tha, double thb, int nitv,
                              const double *itv, double thresh, double *jac, double *mu, double *gam, double *t,
                              double *vals) {
  fp_result r = {0, 0};
  double thc = 0.0;
  dampcf(m, damping, jac);
  if (rootchb(m, v, jac, tha, thb, mu, &thc)) {
    r.skip = 1;
    return r;
  }
  *gam = cos(thc);
  cheb_series(m, mu, 1, gam, t);
  cheb_series(m, mu, nitv, itv, vals);
  r.pass = (vals[0] <= *t * thresh && vals[1] <= *t * thresh);
  return r;
}

/* The degree search over host threads: candidates are taken in increasing
 * order from a shared counter; a worker stops taking them once a passing
 * degree below its next candidate is known.  Every degree below the
 * smallest passing one is evaluated, so the first passing degree (or, with
 * none, the last degree that balances) is the sequential search's. */
typedef struct {
  int next, best; /* next candidate; smallest passing degree so far */
  int min_deg, max_deg, damping, nitv;
  const double *v, *itv;
  double tha, thb, thresh;
  unsigned char *state; /* per candidate: 1 skipped, 2 balanced, 3 passed */
} fp_search;

typedef struct {
  fp_search *S;
  double *jac, *mu;
} fp_worker;

static void *fp_worker_run(void *arg) {
  fp_worker *w = (fp_worker *)arg;
  fp_search *S = w->S;
  for (;;) {
    const int m = __atomic_fetch_add(&S->next, 1, __ATOMIC_RELAXED);
    if (m >= S->max_deg || m > __atomic_load_n(&S->best, __ATOMIC_RELAXED)) break;
    double gam = 0.0, t = 0.0, vals[2] = {0.0, 0.0};
    const fp_result r = fp_candidate(m, S->damping, S->v, S->tha, S->thb, S->nitv, S->itv, S->thresh, w->jac, w->mu,
                                     &gam, &t, vals);
    __atomic_store_n(&S->state[m - S->min_deg], (unsigned char)(r.skip ? 1 : (r.pass ? 3 : 2)), __ATOMIC_RELAXED);
    if (r.pass) {
      int cur = __atomic_load_n(&S->best, __ATOMIC_RELAXED);
      while (m < cur && !__atomic_compare_exchange_n(&S->best, &cur, m, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
      }
    }
  }
  return NULL;
}

#define FP_MAX_THREADS 16
#define FP_THREAD_MIN_DEG 100 /* below this the candidates are too cheap to share out */

/* Runs the search on threads; returns the degree whose design the
 * sequential loop ends with (first passing, else the last balanced one, or
 * -1 when none balanced) and *mend, the loop's final counter. */
static int fp_search_threads(fp_search *S, int nth, int *mend) {
  const int ncand = S->max_deg - S->min_deg;
  fp_worker wk[FP_MAX_THREADS];
  pthread_t tid[FP_MAX_THREADS];
  double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)(S->max_deg + 1) * (size_t)nth);
  if (!buf || !S->state) {
    free(buf);
    return -2;
  }
  for (int i = 0; i < nth; i++) {
    wk[i].S = S;
    wk[i].jac = buf + (size_t)2 * i * (size_t)(S->max_deg + 1);
    wk[i].mu = wk[i].jac + (S->max_deg + 1);
  }
  int started = 0;
  for (int i = 1; i < nth; i++) {
    if (pthread_create(&tid[i], NULL, fp_worker_run, &wk[i]) != 0) break;
    started = i;
  }
  fp_worker_run(&wk[0]);
  for (int i = 1; i <= started; i++) pthread_join(tid[i], NULL);
  free(buf);
  if (S->best < S->max_deg) {
    *mend = S->best + 1;
    return S->best;
  }
  *mend = S->max_deg;
  for (int c = ncand - 1; c >= 0; c--)
    if (S->state[c] == 2) return S->min_deg + c;
  return -1;
}

int find_pol(double *intv, polparams *pol) {
  int max_deg = pol->max_deg, min_deg = pol->min_deg;
  const int damping = pol->damping;
  double tha = 0.0, thb = 0.0, thc = 0.0, gam = 0.0, thresh, t = 0.0;
  double itv[2] = {0.0, 0.0}, vals[2] = {0.0, 0.0};
  int nitv;
  if (evsl_check_intv(intv, stdout) < 0) return -1;
  if (max_deg < 1) return evsl_seterr(EVSLX_ERR_ARG, "find_pol: max_deg must be positive");
  double *mu = (double *)malloc(sizeof(double) * ((size_t)max_deg + 1));
  double *v = (double *)malloc(sizeof(double) * ((size_t)max_deg + 1));
  double *jac = (double *)malloc(sizeof(double) * ((size_t)max_deg + 1));
  if (!mu || !v || !jac) {
    free(mu);
    free(v);
    free(jac);
    return evsl_seterr(EVSLX_ERR_NOMEM, "find_pol: out of memory");
  }
  pol->mu = mu;
  const double IntTol = pol->intvtol;
  double aa = evsl_max(intv[0], intv[2]), bb = evsl_min(intv[1], intv[3]);
  if (intv[0] < intv[2] || intv[1] > intv[3])
    fprintf(stdout, " warning [%s (%d)]: interval (%e, %e) is adjusted to (%e, %e)\n", __FILE__, __LINE__, intv[0],
            intv[1], aa, bb);
  const double lmin = intv[2], lmax = intv[3];
  const double cc = 0.5 * (lmax + lmin), dd = 0.5 * (lmax - lmin);
  pol->cc = cc;
  pol->dd = dd;
  /* map [lmin, lmax] to [-1, 1] */
  aa = (aa - cc) / dd;
  bb = (bb - cc) / dd;
  aa = evsl_max(aa, -1.0);
  bb = evsl_min(bb, 1.0);
  thb = acos(bb);
  tha = acos(aa);
  if (aa - IntTol <= -1.0) {
    thc = tha;
    nitv = 1;
    aa = -1.0;
    gam = -1.0;
    pol->type = 1;
  } else if (bb + IntTol >= 1.0) {
    thc = thb;
    nitv = 1;
    bb = 1;
    gam = 1;
    pol->type = 2;
  } else {
    itv[0] = aa;
    itv[1] = bb;
    nitv = 2;
    pol->type = 0;
  }
  (void)thc;
  int rc = 0;
  if (nitv == 1) {
    rc = chext(pol, aa, bb);
  } else {
    /* starting degree around 1/(half gap) */
    min_deg = 2 + 0.5 / (bb - aa);
    min_deg = evsl_max(min_deg, 2);
    min_deg = evsl_min(min_deg, (max_deg + 1) / 2);
    thresh = pol->thresh_int;
    if (pol->deg > 0) {
      thresh = -1;
      max_deg = pol->deg;
    }
    for (int j = 0; j < min_deg; j++) v[j] = cos(j * thb) - cos(j * tha);
    int m = min_deg;
    long nth = (min_deg >= FP_THREAD_MIN_DEG && max_deg - min_deg >= 2) ? sysconf(_SC_NPROCESSORS_ONLN) : 1;
    nth = evsl_min(evsl_min(nth, (long)FP_MAX_THREADS), (long)(max_deg - min_deg));
    int done = 0;
    if (nth > 1) {
      /* v[j] for every candidate first (the same values the loop forms) */
      for (int j = min_deg; j < max_deg; j++) v[j] = cos(j * thb) - cos(j * tha);
      fp_search S = {min_deg, max_deg, min_deg, max_deg, damping, nitv, v, itv, tha, thb, thresh,
                     (unsigned char *)calloc((size_t)(max_deg - min_deg), 1)};
      int mend = max_deg;
      const int mres = fp_search_threads(&S, (int)nth, &mend);
      free(S.state);
      if (mres >= -1) {
        /* the chosen degree's design again, as the loop leaves it */
        if (mres >= 0) fp_candidate(mres, damping, v, tha, thb, nitv, itv, thresh, jac, mu, &gam, &t, vals);
        m = mend;
        done = 1;
      }
    }
    if (!done) {
      for (m = min_deg; m < max_deg; m++) {
        v[m] = cos(m * thb) - cos(m * tha);
        const fp_result r = fp_candidate(m, damping, v, tha, thb, nitv, itv, thresh, jac, mu, &gam, &t, vals);
        if (r.skip) continue;
        if (r.pass) {
          m++;
          break;
        }
      }
    }
    const int mbest = m - 1;
    for (int j = 0; j <= mbest; j++) mu[j] /= t;
    pol->bar = evsl_min(vals[0], vals[1]) / t;
    pol->gam = gam;
    pol->deg = mbest;
  }
  free(v);
  free(jac);
  return rc;
}

void free_pol(polparams *pol) {
  if (pol->mu) {
    free(pol->mu);
    pol->mu = NULL;
  }
}

/* y = p[(A - cc)/dd] v on device vectors; w is 3n device doubles. */
int ChebAv(polparams *pol, double *v, double *y, double *w) {
  int rc = evsl_require_operator();
  if (rc) return rc;
  const double tt = evsl_timer();
  rc = evslcu_chebav(evsl_op(), pol->mu, pol->deg, pol->cc, pol->dd, v, y, w, NULL);
  if (!rc) rc = evslcu_sync();
  if (rc) return evsl_seterr(rc, "%s", evslcu_errstr());
  evslstat.n_polAv++;
  evslstat.t_polAv += evsl_timer() - tt;
  return 0;
}

int evslx_chebav_block(polparams *pol, int ncols, const double *V, double *Y, double *work) {
  int rc = evsl_require_operator();
  if (rc) return rc;
  if (!pol || !pol->mu || ncols < 1) return evsl_seterr(EVSLX_ERR_ARG, "evslx_chebav_block: bad arguments");
  const double tt = evsl_timer();
  rc = evslcu_chebav_block(evsl_op(), pol->mu, pol->deg, pol->cc, pol->dd, ncols, V, Y, work);
  if (!rc) rc = evslcu_sync();
  if (rc) return evsl_seterr(rc, "%s", evslcu_errstr());
  evslstat.n_polAv += ncols;
  evslstat.t_polAv += evsl_timer() - tt;
  return 0;
}

void evsl_chebAv_device(int n, int k, double t, double s, double cc, double *vkp1, double *vk, double *vkm1,
                        double *y) {
  evslcu_cheb_update(n, k, t, s, cc, vkp1, vk, vkm1, y);
}

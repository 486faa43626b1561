/*
 * cheblanNr.c -- polynomial-filtered non-restarted Lanczos with full
 * reorthogonalisation (reference SRC/cheblanNr.c:57-434).
 *
 * Same algorithm, same stopping test and same outputs as the reference:
 *   - the start vector is filtered (FILTER_VINIT, :16,150) and normalised;
 *   - each step applies the filter p(A) on the GPU, subtracts beta*v_{k-1}
 *     (fused into the last filter kernel, which also forms alpha = v.znew),
 *     subtracts alpha*v, and reorthogonalises against the whole basis with
 *     classical Gram-Schmidt + DGKS (misc_la.c:221-261) on the GPU;
 *   - lucky breakdown restarts from a new filtered random vector (:225-256);
 *   - every 20 steps after step 30 the restricted trace of the Ritz values
 *     above `bar` is tested (:269-309);
 *   - Ritz vectors are formed for every Ritz value >= bar with one GEMM
 *     V(:,1:kdim) * Y, then normalised, their Rayleigh quotients and
 *     residual norms w.r.t. A computed in batched kernels, and a pair is
 *     kept if lambda is in [a,b] (with 10*DBL_EPSILON slack) and the
 *     residual is below tol (:336-399).
 * Outputs follow the reference CUDA build: lamo/reso host, Wo device.
 */
#include "internal.h"

#define NR_NTEST 30
#define NR_CYCLE 20

/* Restricted-trace convergence test on the eigenvalues of T_kdim
 * (SRC/cheblanNr.c:269-309): 1 when converged; *tr0 carries the previous
 * trace. */
static int trace_converged(int kdim, const double *EvalT, double bar, double *tr0, int do_print, FILE *fstats) {
  double tr1 = 0.0;
  int nconv = 0;
  for (int i = 0; i < kdim; i++) {
    const double flami = EvalT[i];
    if (flami + EVSL_DBL_EPS_MULT * DBL_EPSILON >= bar) {
      tr1 += flami;
      nconv++;
    }
  }
  if (do_print) fprintf(fstats, "k %4d: nconv %4d  tr1 %21.15e\n", kdim - 1, nconv, tr1);
  if ((fabs(tr1 - *tr0) < 2e-12) || (fabs(tr1) + fabs(*tr0) < 1e-10)) return 1;
  *tr0 = tr1;
  return 0;
}

/* Read the side-stream test of T_kd into EvalT and apply the trace test. */
static int read_pending(int kd, double *EvalT, double bar, double *tr0, int do_print, FILE *fstats, int *conv) {
  const double te = evsl_timer();
  const int rc = evsl_trid_test_wait(EvalT);
  evslstat.t_eig += evsl_timer() - te;
  if (rc) return rc;
  *conv = trace_converged(kd, EvalT, bar, tr0, do_print, fstats);
  return 0;
}

int ChebLanNr(double *intv, int maxit, double tol, double *vinit, polparams *pol, int *nevOut, double **lamo,
              double **Wo, double **reso, FILE *fstats) {
  const double tall = evsl_timer();
  int rc = evsl_require_operator();
  if (rc) return rc;
  const int do_print = (fstats != NULL);
  const int n = evsl_op()->n;
  maxit = evsl_min(n, maxit);
  const size_t n_l = (size_t)n;
  const double bar = pol->bar, gamB = pol->gam;
  *nevOut = 0;
  *lamo = NULL;
  *Wo = NULL;
  *reso = NULL;
  if (evsl_check_intv(intv, fstats) < 0) return 0;
  const double aa = intv[0], bb = intv[1];
  const int deg = pol->deg;
  if (do_print) fprintf(fstats, " ** Cheb Poly of deg = %d, gam = %.15e, bar: %.15e\n", deg, gamB, bar);
  if (gamB > 1.0 || gamB < -1.0) {
    fprintf(stdout, "gamB error %.15e\n", gamB);
    return -1;
  }
  if (maxit < 1) return evsl_seterr(EVSLX_ERR_ARG, "ChebLanNr: maxit must be positive");
  if (do_print) fprintf(fstats, " ** Cheb-LanNr \n");

  const evslcu_op *op = evsl_op();
  double *V = (double *)evslcu_malloc(sizeof(double) * n_l * ((size_t)maxit + 1));
  double *wk = (double *)evslcu_malloc(sizeof(double) * 3 * n_l);
  double *vrand = (double *)evslcu_malloc(sizeof(double) * n_l);
  const size_t cgs_sz = evslcu_cgs_work_size(n, maxit + 1);
  double *cgsw = (double *)evslcu_malloc(sizeof(double) * cgs_sz);
  double *ds = (double *)evslcu_malloc(sizeof(double) * 8); /* device scalars */
  double *dT = (double *)malloc(sizeof(double) * (size_t)maxit);
  double *eT = (double *)malloc(sizeof(double) * (size_t)maxit);
  double *EvalT = (double *)malloc(sizeof(double) * (size_t)maxit);
  double *Lam = NULL, *res = NULL, *Rvec = NULL, *W = NULL, *EvecT = NULL, *EvecT_dev = NULL;
  double *rnorm = NULL, *rlam = NULL, *rres = NULL;
  int *sel = NULL;
  int kdim = 0, count = 0, nev = 0;
  double tt_ritz = 0.0;
  evslcu_marks *marks = NULL;
  int pend_k = 0; /* Lanczos dimension of the test running on the side stream */
  if (!V || !wk || !vrand || !cgsw || !ds || !dT || !eT || !EvalT) {
    rc = evsl_seterr(EVSLX_ERR_NOMEM, "ChebLanNr: out of memory for a basis of %d x %d", n, maxit + 1);
    goto done;
  }
  double *d_alpha = ds, *d_beta = ds + 1, *d_nrm = ds + 2;

  /* filter and normalise the start vector */
  if ((rc = evslcu_chebav(op, pol->mu, deg, pol->cc, pol->dd, vinit, V, wk, NULL))) goto cuda_fail;
  evslstat.n_polAv++;
  if ((rc = evslcu_nrm2(n, V, d_nrm))) goto cuda_fail;
  double h[2];
  if ((rc = evslcu_get_scalars(d_nrm, h, 1))) goto cuda_fail;
  double t = 1.0 / h[0];
  if ((rc = evslcu_scal(n, t, V))) goto cuda_fail;

  /* with a stats stream, the filter and reorthogonalisation device times of
   * every step go to evslstat.t_polAv / t_reorth (events read after the
   * step's scalar read has synchronised) */
  marks = fstats ? evslcu_marks_create(3) : NULL;
  /* Convergence tests run on a side stream while the next steps proceed;
   * each is read at the next test point, at the last step, before a lucky
   * breakdown draws random numbers, or as soon as it has finished.  Steps
   * taken past a test that reports convergence are discarded, so the result
   * is that of waiting for every test. */
  const int async_tests = !evslh.sync_tests;
  const double xmin = bar - EVSL_DBL_EPS_MULT * DBL_EPSILON;
  double wn = 0.0, tr0 = 0.0, beta = 0.0;
  int nwn = 0, k;
  for (k = 0; k < maxit; k++) {
    const double *zold = (k > 0) ? V + (size_t)(k - 1) * n_l : NULL;
    double *v = V + (size_t)k * n_l;
    double *vnew = v + n_l;
    /* znew = p(A) v - beta zold; alpha = v . znew */
    evslcu_cheb_epi epi = {zold, -beta, v, d_alpha};
    evslcu_marks_record(marks, 0);
    if ((rc = evslcu_chebav(op, pol->mu, deg, pol->cc, pol->dd, v, vnew, wk, &epi))) goto cuda_fail;
    evslstat.n_polAv++;
    evslcu_marks_record(marks, 1);
    /* znew -= alpha v */
    if ((rc = evslcu_axpy_ds(n, d_alpha, -1.0, v, vnew))) goto cuda_fail;
    /* full reorthogonalisation, beta = ||vnew|| */
    if ((rc = evslcu_cgs_dgks(n, k + 1, EVSL_NGS_MAX, V, (long long)n, vnew, d_beta, cgsw))) goto cuda_fail;
    evslcu_marks_record(marks, 2);
    if ((rc = evslcu_get_scalars(ds, h, 2))) goto cuda_fail;
    if (marks) {
      evslstat.t_polAv += evslcu_marks_elapsed(marks, 0, 1);
      evslstat.t_reorth += evslcu_marks_elapsed(marks, 1, 2);
    }
    const double alpha = h[0];
    beta = h[1];
    dT[k] = alpha;
    wn += fabs(alpha);
    wn += 2.0 * beta;
    nwn += 3;
    if (beta * nwn < EVSL_ORTH_TOL * wn) {
      if (pend_k) {
        const int kd = pend_k;
        int conv = 0;
        pend_k = 0;
        if ((rc = read_pending(kd, EvalT, bar, &tr0, do_print, fstats, &conv))) goto done;
        if (conv) {
          kdim = count = kd;
          break;
        }
      }
      if (do_print) fprintf(fstats, "it %4d: Lucky breakdown, beta = %.15e\n", k, beta);
      /* restart from a new filtered random vector */
      if ((rc = evsl_rand_device(n, 1, vrand))) goto done;
      if ((rc = evslcu_chebav(op, pol->mu, deg, pol->cc, pol->dd, vrand, vnew, wk, NULL))) goto cuda_fail;
      if ((rc = evslcu_cgs_dgks(n, k + 1, EVSL_NGS_MAX, V, (long long)n, vnew, d_beta, cgsw))) goto cuda_fail;
      if ((rc = evslcu_get_scalars(d_beta, h, 1))) goto cuda_fail;
      t = 1.0 / h[0];
      if ((rc = evslcu_scal(n, t, vnew))) goto cuda_fail;
      beta = 0.0;
    } else {
      t = 1.0 / beta;
      if ((rc = evslcu_scal(n, t, vnew))) goto cuda_fail;
    }
    eT[k] = beta;
    const int test_here = !((k < NR_NTEST || (k - NR_NTEST) % NR_CYCLE != 0) && k != maxit - 1);
    if (pend_k && (test_here || evsl_trid_test_ready())) {
      const int kd = pend_k;
      int conv = 0;
      pend_k = 0;
      if ((rc = read_pending(kd, EvalT, bar, &tr0, do_print, fstats, &conv))) goto done;
      if (conv) {
        kdim = count = kd;
        break;
      }
    }
    if (!test_here) continue;
    kdim = k + 1;
    if (async_tests && k != maxit - 1) {
      const int st = evsl_trid_test_start(kdim, dT, eT, xmin);
      if (st < 0) {
        rc = st;
        goto done;
      }
      if (st == 1) {
        pend_k = kdim;
        continue;
      }
    }
    const double te = evsl_timer();
    if ((rc = evsl_trid_eigvals_test(kdim, dT, eT, xmin, EvalT))) goto done;
    evslstat.t_eig += evsl_timer() - te;
    count = kdim;
    if (trace_converged(kdim, EvalT, bar, &tr0, do_print, fstats)) break;
  }
  if (k >= maxit && do_print)
    fprintf(fstats,
            "The max number of iterations [%d] has been reached. The eigenvalues computed may not have converged\n",
            maxit);

  /* ---- Ritz pairs ---- */
  {
    const double te = evsl_timer();
    /* EvalT holds the eigenvalues of T_kdim from the last convergence test
     * (the loop ends right after one): the ones >= bar are selected */
    int msel = 0;
    sel = (int *)malloc(sizeof(int) * (size_t)(kdim > 0 ? kdim : 1));
    for (int i = 0; i < count; i++)
      if (EvalT[i] >= bar) sel[msel++] = i;
    evslh.last_candidates = msel;
    double *wsel = (double *)malloc(sizeof(double) * (size_t)(msel > 0 ? msel : 1));
    for (int j = 0; j < msel; j++) wsel[j] = EvalT[sel[j]];
    EvecT = (double *)malloc(sizeof(double) * (size_t)kdim * (size_t)(msel > 0 ? msel : 1));
    if (!EvecT) {
      free(wsel);
      rc = evsl_seterr(EVSLX_ERR_NOMEM, "ChebLanNr: out of memory (Ritz)");
      goto done;
    }
    rc = evsl_trid_eigvecs(kdim, dT, eT, msel, wsel, EvecT, kdim);
    free(wsel);
    if (rc) goto done;
    evslstat.t_eig += evsl_timer() - te;
    const double tr = evsl_timer();
    Lam = (double *)malloc(sizeof(double) * (size_t)(msel > 0 ? msel : 1));
    res = (double *)malloc(sizeof(double) * (size_t)(msel > 0 ? msel : 1));
    if (msel > 0) {
      EvecT_dev = (double *)evslcu_malloc(sizeof(double) * (size_t)kdim * msel);
      Rvec = (double *)evslcu_malloc(sizeof(double) * n_l * msel);
      W = (double *)evslcu_malloc(sizeof(double) * n_l * msel);
      rnorm = (double *)malloc(sizeof(double) * 3 * (size_t)msel);
      if (!EvecT_dev || !Rvec || !W || !rnorm || !Lam || !res) {
        rc = evsl_seterr(EVSLX_ERR_NOMEM, "ChebLanNr: out of memory for %d Ritz vectors", msel);
        goto done;
      }
      rlam = rnorm + msel;
      rres = rlam + msel;
      if ((rc = evslcu_h2d(EvecT_dev, EvecT, sizeof(double) * (size_t)kdim * msel))) goto cuda_fail;
      /* Rvec = V(:, 1:kdim) * EvecT(:, sel) */
      if ((rc = evslcu_dgemm('N', 'N', n, msel, kdim, 1.0, V, n, EvecT_dev, kdim, 0.0, Rvec, n))) goto cuda_fail;
      if ((rc = evslcu_ritz_eval(op, n, msel, Rvec, W, rnorm, rlam, rres))) goto cuda_fail;
      int *keep = (int *)malloc(sizeof(int) * (size_t)msel);
      for (int j = 0; j < msel; j++) {
        if (rnorm[j] == 0.0) {
          free(keep);
          rc = 2; /* zero Ritz vector (reference return code 2) */
          goto done;
        }
        const double lam = rlam[j];
        if (lam < aa - EVSL_DBL_EPS_MULT * DBL_EPSILON || lam > bb + EVSL_DBL_EPS_MULT * DBL_EPSILON) continue;
        if (rres[j] < tol) {
          Lam[nev] = lam;
          res[nev] = rres[j];
          keep[nev] = j;
          nev++;
        }
      }
      rc = evslcu_gather_cols(n, nev, keep, Rvec, Rvec);
      free(keep);
      if (rc) goto cuda_fail;
      if ((rc = evslcu_sync())) goto cuda_fail;
    }
    tt_ritz = evsl_timer() - tr;
  }
  evslh.last_kdim = kdim;
  *nevOut = nev;
  *lamo = Lam;
  *reso = res;
  *Wo = (nev > 0) ? Rvec : NULL;
  if (nev == 0) evslcu_free(Rvec);
  Lam = res = Rvec = NULL;
  evslstat.t_ritz = tt_ritz;
  evslstat.t_iter = evsl_timer() - tall;
  rc = 0;
  goto done;

cuda_fail:
  rc = evsl_seterr(rc, "%s", evslcu_errstr());
done:
  if (pend_k) evsl_trid_test_wait(EvalT); /* an error left a test in flight */
  evslcu_marks_destroy(marks);
  evslcu_free(V);
  evslcu_free(wk);
  evslcu_free(vrand);
  evslcu_free(cgsw);
  evslcu_free(ds);
  evslcu_free(EvecT_dev);
  evslcu_free(W);
  evslcu_free(Rvec);
  free(dT);
  free(eT);
  free(EvalT);
  free(EvecT);
  free(Lam);
  free(res);
  free(rnorm);
  free(sel);
  return rc;
}

/*
 * lanbounds.c -- Lanczos estimates of the spectrum bounds [lmin, lmax]
 * (reference SRC/lanbounds.c:21-144 and SRC/lanTrbounds.c:35-422).  These
 * give the interval (intv[2], intv[3]) that kpmdos and find_pol need when the
 * spectrum is not known analytically.
 *
 * Vectors live on the GPU; the tridiagonal / arrow-head eigenproblems are
 * solved on the host (tridiag.c).  `v` / `vinit` are DEVICE vectors, as for
 * the other solvers of the CUDA build.
 */
#include "internal.h"

#define TRB_MIN_INNER 5

/* SRC/lanbounds.c:21: msteps Lanczos steps with full reorthogonalisation
 * (one modified Gram-Schmidt pass, as the reference), then
 *   lmin = theta_1 - |beta_m s_{m,1}|,  lmax = theta_m + |beta_m s_{m,m}|. */
int LanBounds(int msteps, double *v, double *lmin, double *lmax) {
  int rc = evsl_require_operator();
  if (rc) return rc;
  const int n = evsl_op()->n;
  const size_t n_l = (size_t)n;
  msteps = evsl_min(n, msteps);
  if (msteps < 1 || !v || !lmin || !lmax) return evsl_seterr(EVSLX_ERR_ARG, "LanBounds: bad arguments");
  double *alp = (double *)malloc(sizeof(double) * (size_t)msteps);
  double *bet = (double *)malloc(sizeof(double) * (size_t)msteps);
  double *V = (double *)evslcu_malloc(sizeof(double) * n_l * ((size_t)msteps + 1));
  double *ds = (double *)evslcu_malloc(sizeof(double) * 4);
  double *w = (double *)malloc(sizeof(double) * (size_t)msteps);
  double *S = (double *)malloc(sizeof(double) * 2 * (size_t)msteps);
  double h[2];
  if (!alp || !bet || !V || !ds || !w || !S) {
    rc = evsl_seterr(EVSLX_ERR_NOMEM, "LanBounds: out of memory");
    goto done;
  }
  /* V(:,0) = v / ||v|| */
  if ((rc = evslcu_nrm2(n, v, ds)) || (rc = evslcu_get_scalars(ds, h, 1))) goto cuda_fail;
  if ((rc = evslcu_copy(n, v, V)) || (rc = evslcu_scal(n, 1.0 / h[0], V))) goto cuda_fail;
  double wn = 0.0;
  for (int j = 0; j < msteps; j++) {
    double *vj = V + (size_t)j * n_l, *znew = V + (size_t)(j + 1) * n_l;
    if ((rc = evsl_apply_A(vj, znew))) goto done;
    if (j && (rc = evslcu_axpy(n, -bet[j - 1], V + (size_t)(j - 1) * n_l, znew))) goto cuda_fail;
    if ((rc = evslcu_dot(n, znew, vj, ds))) goto cuda_fail;
    if ((rc = evslcu_axpy_ds(n, ds, -1.0, vj, znew))) goto cuda_fail;
    for (int i = 0; i <= j; i++) {
      const double *vi = V + (size_t)i * n_l;
      if ((rc = evslcu_dot(n, znew, vi, ds + 2)) || (rc = evslcu_axpy_ds(n, ds + 2, -1.0, vi, znew))) goto cuda_fail;
    }
    if ((rc = evslcu_dot(n, znew, znew, ds + 1)) || (rc = evslcu_get_scalars(ds, h, 2))) goto cuda_fail;
    alp[j] = h[0];
    wn += alp[j] * alp[j];
    bet[j] = h[1];
    if (bet[j] * (j + 1) < EVSL_ORTH_TOL * wn) {
      fprintf(stdout, "lanbounds: lucky break, j=%d, beta=%e, break\n", j, bet[j]);
      msteps = j + 1;
      break;
    }
    wn += 2.0 * bet[j];
    bet[j] = sqrt(bet[j]);
    if ((rc = evslcu_scal(n, 1.0 / bet[j], znew))) goto cuda_fail;
  }
  {
    const double bottom = bet[msteps - 1];
    if ((rc = evsl_trid_eigvals(msteps, alp, bet, w))) goto done;
    double ws[2] = {w[0], w[msteps - 1]};
    const int nsel = (msteps > 1) ? 2 : 1;
    if ((rc = evsl_trid_eigvecs(msteps, alp, bet, nsel, ws, S, msteps))) goto done;
    const double *s_last = S + (size_t)(nsel - 1) * msteps;
    *lmin = w[0] - fabs(bottom * S[msteps - 1]);
    *lmax = w[msteps - 1] + fabs(bottom * s_last[msteps - 1]);
  }
  rc = 0;
  goto done;
cuda_fail:
  rc = evsl_seterr(rc, "%s", evslcu_errstr());
done:
  free(alp);
  free(bet);
  free(w);
  free(S);
  evslcu_free(V);
  evslcu_free(ds);
  return rc;
}

/* SRC/lanTrbounds.c:35: thick-restart Lanczos on A keeping the two extreme
 * Ritz pairs; bounds simple (|beta s|) or Kato-Temple (bndtype > 1);
 * stops when t1 + t2 < tol (|lmin| + |lmax|). */
int LanTrbounds(int lanm, int maxit, double tol, double *vinit, int bndtype, double *lammin, double *lammax,
                FILE *fstats) {
  int rc = evsl_require_operator();
  if (rc) return rc;
  const int do_print = (fstats != NULL);
  const int n = evsl_op()->n;
  const size_t n_l = (size_t)n;
  double lmin = 0.0, lmax = 0.0, t1, t2;
  lanm = evsl_min(lanm, n);
  const int lanm1 = lanm + 1;
  const size_t lanm1_l = (size_t)lanm1;
  if (lanm == n) maxit = evsl_min(maxit, n);
  if (lanm < 2 || !vinit || !lammin || !lammax) return evsl_seterr(EVSLX_ERR_ARG, "LanTrbounds: bad arguments");
  if (do_print) fprintf(fstats, " LanTR for bounds: dim %d, maxits %d\n", lanm, maxit);
  int it = 0, trlen = 0;
  double *V = (double *)evslcu_malloc(sizeof(double) * n_l * lanm1_l);
  double *T = (double *)calloc(lanm1_l * lanm1_l, sizeof(double));
  double *Rval = (double *)malloc(sizeof(double) * (size_t)lanm1);
  double *Rvec = (double *)evslcu_malloc(sizeof(double) * n_l * 2);
  double *EvecT = (double *)calloc(lanm1_l * lanm1_l, sizeof(double));
  double *Ed = (double *)evslcu_malloc(sizeof(double) * lanm1_l * 2);
  double *vrand = NULL;
  double *cgsw = (double *)evslcu_malloc(sizeof(double) * evslcu_cgs_work_size(n, lanm1));
  double *ds = (double *)evslcu_malloc(sizeof(double) * 8);
  double s[3] = {0.0, 0.0, 0.0};
  double h[2];
  if (!V || !T || !Rval || !Rvec || !EvecT || !Ed || !cgsw || !ds) {
    rc = evsl_seterr(EVSLX_ERR_NOMEM, "LanTrbounds: out of memory");
    goto done;
  }
  double *d_alpha = ds, *d_beta = ds + 1;
  if ((rc = evslcu_copy(n, vinit, V)) || (rc = evslcu_nrm2(n, V, ds + 2)) || (rc = evslcu_get_scalars(ds + 2, h, 1)))
    goto cuda_fail;
  if ((rc = evslcu_scal(n, 1.0 / h[0], V))) goto cuda_fail;
  while (it < maxit) {
    double wn = 0.0, beta = 0.0;
    int nwn = 0;
    int k = trlen > 0 ? trlen + 1 : 0;
    if (k + TRB_MIN_INNER > lanm1) {
      rc = evsl_seterr(EVSLX_ERR_ARG, "LanTrbounds: Krylov dim too small for this problem");
      goto done;
    }
    if (trlen > 0) {
      const int k1 = k - 1;
      double *v = V + (size_t)k1 * n_l, *vnew = v + n_l;
      if ((rc = evsl_apply_A(v, vnew))) goto done;
      for (int i = 0; i < trlen; i++) {
        T[i * lanm1_l + i] = Rval[i];
        wn += fabs(Rval[i]);
      }
      if ((rc = evslcu_dot(n, v, vnew, ds + 3)) || (rc = evslcu_get_scalars(ds + 3, h, 1))) goto cuda_fail;
      s[k1] = h[0];
      for (int i = 0; i < k; i++)
        if ((rc = evslcu_axpy(n, -s[i], V + (size_t)i * n_l, vnew))) goto cuda_fail;
      for (int i = 0; i < k1; i++) {
        T[trlen * lanm1_l + i] = s[i];
        T[i * lanm1_l + trlen] = s[i];
        wn += 2.0 * fabs(s[i]);
      }
      T[trlen * lanm1_l + trlen] = s[k1];
      wn += fabs(s[k1]);
      if ((rc = evslcu_nrm2(n, vnew, d_beta)) || (rc = evslcu_get_scalars(d_beta, h, 1))) goto cuda_fail;
      beta = h[0];
      wn += 2.0 * beta;
      nwn += 3 * k;
      if (beta * nwn < EVSL_ORTH_TOL * wn) {
        if ((rc = evsl_rand_device(n, 1, vnew))) goto done;
        if ((rc = evslcu_cgs_dgks(n, k, EVSL_NGS_MAX, V, (long long)n, vnew, d_beta, cgsw)) ||
            (rc = evslcu_get_scalars(d_beta, h, 1)) || (rc = evslcu_scal(n, 1.0 / h[0], vnew)))
          goto cuda_fail;
        beta = 0.0;
      } else if ((rc = evslcu_scal(n, 1.0 / beta, vnew))) {
        goto cuda_fail;
      }
      T[k1 * lanm1_l + k] = beta;
      T[k * lanm1_l + k1] = beta;
    }
    const double *zold = k > 0 ? V + (size_t)(k - 1) * n_l : NULL;
    while (k < lanm && it < maxit) {
      k++;
      double *v = V + (size_t)(k - 1) * n_l, *vnew = v + n_l;
      if ((rc = evsl_apply_A(v, vnew))) goto done;
      it++;
      if (zold && (rc = evslcu_axpy(n, -beta, zold, vnew))) goto cuda_fail;
      if ((rc = evslcu_dot(n, v, vnew, d_alpha)) || (rc = evslcu_axpy_ds(n, d_alpha, -1.0, v, vnew))) goto cuda_fail;
      if ((rc = evslcu_cgs_dgks(n, k, EVSL_NGS_MAX, V, (long long)n, vnew, d_beta, cgsw))) goto cuda_fail;
      if ((rc = evslcu_get_scalars(ds, h, 2))) goto cuda_fail;
      const double alpha = h[0];
      beta = h[1];
      T[(k - 1) * lanm1_l + (k - 1)] = alpha;
      wn += fabs(alpha);
      wn += 2.0 * beta;
      nwn += 3;
      zold = v;
      if (beta * nwn < EVSL_ORTH_TOL * wn) {
        if (do_print) fprintf(fstats, "it %4d: Lucky breakdown, beta = %.15e\n", it, beta);
        if ((rc = evsl_rand_device(n, 1, vnew))) goto done;
        if ((rc = evslcu_cgs_dgks(n, k, EVSL_NGS_MAX, V, (long long)n, vnew, d_beta, cgsw)) ||
            (rc = evslcu_get_scalars(d_beta, h, 1)) || (rc = evslcu_scal(n, 1.0 / h[0], vnew)))
          goto cuda_fail;
        beta = 0.0;
      } else if ((rc = evslcu_scal(n, 1.0 / beta, vnew))) {
        goto cuda_fail;
      }
      T[k * lanm1_l + (k - 1)] = beta;
      T[(k - 1) * lanm1_l + k] = beta;
    }
    /* extreme Ritz pairs of T (ascending Rval) */
    if ((rc = evsl_tr_eig_sel(k, trlen, T, lanm1, 1, 0.0, Rval, EvecT, lanm1))) goto done;
    s[0] = beta * EvecT[k - 1];
    s[1] = beta * EvecT[(size_t)(k - 1) * lanm1_l + (k - 1)];
    if (bndtype <= 1) {
      t1 = fabs(s[0]);
      t2 = fabs(s[1]);
    } else {
      t1 = 2.0 * s[0] * s[0] / (Rval[1] - Rval[0]);
      t2 = 2.0 * s[1] * s[1] / (Rval[k - 1] - Rval[k - 2]);
    }
    lmin = Rval[0] - t1;
    lmax = Rval[k - 1] + t2;
    /* Rvec(:,0) = V(:,1:k) y_1, Rvec(:,1) = V(:,1:k) y_k */
    if ((rc = evslcu_h2d(Ed, EvecT, sizeof(double) * (size_t)k)) ||
        (rc = evslcu_h2d(Ed + lanm1_l, EvecT + (size_t)(k - 1) * lanm1_l, sizeof(double) * (size_t)k)))
      goto cuda_fail;
    if ((rc = evslcu_dgemv('N', n, k, 1.0, V, n, Ed, 0.0, Rvec)) ||
        (rc = evslcu_dgemv('N', n, k, 1.0, V, n, Ed + lanm1_l, 0.0, Rvec + n_l)))
      goto cuda_fail;
    trlen = 2;
    if ((rc = evslcu_d2d(V, Rvec, sizeof(double) * 2 * n_l))) goto cuda_fail;
    Rval[1] = Rval[k - 1];
    if (do_print)
      fprintf(fstats, "it %4d, k %3d: ritz %.15e %.15e, t1,t2 %e %e, res %.15e %.15e\n", it, k, Rval[0], Rval[1], t1,
              t2, fabs(s[0]), fabs(s[1]));
    if (t1 + t2 < tol * (fabs(lmin) + fabs(lmax))) break;
    memset(T, 0, sizeof(double) * lanm1_l * lanm1_l);
    if ((rc = evslcu_d2d(V + (size_t)trlen * n_l, V + (size_t)k * n_l, sizeof(double) * n_l))) goto cuda_fail;
  }
  if ((rc = evslcu_sync())) goto cuda_fail;
  *lammin = lmin;
  *lammax = lmax;
  rc = 0;
  goto done;
cuda_fail:
  rc = evsl_seterr(rc, "%s", evslcu_errstr());
done:
  evslcu_free(V);
  free(T);
  free(Rval);
  evslcu_free(Rvec);
  free(EvecT);
  evslcu_free(Ed);
  evslcu_free(vrand);
  evslcu_free(cgsw);
  evslcu_free(ds);
  return rc;
}

/*
 * cheblanTr.c -- polynomial-filtered thick-restart Lanczos with locking
 * (reference SRC/cheblanTr.c:59-707).
 *
 * Same algorithm and outputs as the reference:
 *   - after a restart, the arrow-head step (:224-319): filter the last
 *     vector, deflate against locked vectors, s = V(:,1:k)' znew applied as a
 *     GEMV, beta = ||znew||;
 *   - inner Lanczos loop (:331-503) with deflation against the locked set,
 *     full CGS+DGKS reorthogonalisation on the GPU, and every `cycle` steps a
 *     dense eigensolve of T whose count and trace of Ritz values above bar
 *     decide the restart;
 *   - pass 1 keeps Ritz values >= bar, pass 2 forms the Ritz vectors with one
 *     GEMM, evaluates Rayleigh quotients and residuals in batched kernels,
 *     locks converged pairs (growing the locked block by 1 + 20% when full,
 *     :598-610) and keeps the others as the thick-restart set (:620-629).
 * Outputs: vals/resW on the host, W on the device (n x nev2).
 * Where the reference calls exit(1) ("Krylov dim too small") this returns
 * EVSLX_ERR_ARG.
 */
#include "internal.h"

#define TR_CYCLE 50
#define TR_MIN_INNER 5

int ChebLanTr(int lanm, int nev, double *intv, int maxit, double tol, double *vinit, polparams *pol, int *nev2,
              double **vals, double **W, double **resW, FILE *fstats) {
  const double tall = evsl_timer();
  int rc = evsl_require_operator();
  if (rc) return rc;
  const int do_print = (fstats != NULL);
  const int n = evsl_op()->n;
  const size_t n_l = (size_t)n;
  *nev2 = 0;
  *vals = NULL;
  *W = NULL;
  *resW = NULL;
  lanm = evsl_min(lanm, n);
  const int lanm1 = lanm + 1;
  const size_t lanm1_l = (size_t)lanm1;
  if (lanm == n) maxit = evsl_min(maxit, n);
  const double nevInc = 0.2;
  int Ntest = evsl_min(lanm, nev + 50);
  if (evsl_check_intv(intv, fstats) < 0) return 0;
  const double aa = intv[0], bb = intv[1];
  const double gamB = pol->gam, bar = pol->bar;
  if (gamB > 1.0 || gamB < -1.0) {
    if (fstats) fprintf(fstats, "gamB error %.15e\n", gamB);
    return -1;
  }
  if (nev < 1) nev = 1;
  if (do_print) fprintf(fstats, " Cheb-LanTR, dim %d  cycle %d  \n", lanm, TR_CYCLE);
  const evslcu_op *op = evsl_op();
  const int deg = pol->deg;

  double *V = (double *)evslcu_malloc(sizeof(double) * n_l * lanm1_l);
  double *T = (double *)calloc(lanm1_l * lanm1_l, sizeof(double));
  double *Y = (double *)evslcu_malloc(sizeof(double) * n_l * (size_t)nev);
  double *Lam = (double *)malloc(sizeof(double) * (size_t)nev);
  double *res = (double *)malloc(sizeof(double) * (size_t)nev);
  double *Rval = (double *)malloc(sizeof(double) * (size_t)lanm);
  double *resi = (double *)malloc(sizeof(double) * (size_t)lanm);
  double *Rvec = (double *)evslcu_malloc(sizeof(double) * n_l * (size_t)lanm);
  double *Wt = (double *)evslcu_malloc(sizeof(double) * n_l * (size_t)lanm);
  double *EvecT = (double *)malloc(sizeof(double) * lanm1_l * lanm1_l);
  double *EvecT_dev = (double *)evslcu_malloc(sizeof(double) * lanm1_l * lanm1_l);
  double *s = (double *)malloc(sizeof(double) * (size_t)lanm1);
  double *s_dev = (double *)evslcu_malloc(sizeof(double) * (size_t)lanm1);
  double *work = (double *)evslcu_malloc(sizeof(double) * 3 * n_l);
  double *vrand = (double *)evslcu_malloc(sizeof(double) * n_l);
  const size_t cgs_sz = evslcu_cgs_work_size(n, evsl_max(lanm1, nev) + 64);
  double *cgsw = (double *)evslcu_malloc(sizeof(double) * cgs_sz);
  double *ds = (double *)evslcu_malloc(sizeof(double) * 8);
  double *rnorm = (double *)malloc(sizeof(double) * 3 * (size_t)lanm);
  int cgs_cap = evsl_max(lanm1, nev) + 64;
  int lock = 0, trlen = 0, prtrlen = -1, it = 0;
  if (!V || !T || !Y || !Lam || !res || !Rval || !resi || !Rvec || !Wt || !EvecT || !EvecT_dev || !s || !s_dev ||
      !work || !vrand || !cgsw || !ds || !rnorm) {
    rc = evsl_seterr(EVSLX_ERR_NOMEM, "ChebLanTr: out of memory (n=%d, lanm=%d)", n, lanm);
    goto done;
  }
  double *d_alpha = ds, *d_beta = ds + 1, *d_nrm = ds + 2, *d_s = ds + 3;
  double h[4];

  if ((rc = evslcu_chebav(op, pol->mu, deg, pol->cc, pol->dd, vinit, V, work, NULL))) goto cuda_fail;
  if ((rc = evslcu_nrm2(n, V, d_nrm)) || (rc = evslcu_get_scalars(d_nrm, h, 1))) goto cuda_fail;
  if ((rc = evslcu_scal(n, 1.0 / h[0], V))) goto cuda_fail;

  while (it < maxit) {
    double wn = 0.0, beta = 0.0;
    int nwn = 0;
    int k = trlen > 0 ? trlen + 1 : 0;
    if (k + TR_MIN_INNER > lanm1) {
      if (fstats) fprintf(fstats, "Krylov dim too small for this problem. Try a larger dim\n");
      rc = evsl_seterr(EVSLX_ERR_ARG, "ChebLanTr: Krylov dimension %d too small for %d restart vectors", lanm,
                       trlen);
      goto done;
    }
    /* grow the GS workspace if the locked set outgrew it */
    if (lock + 8 > cgs_cap) {
      evslcu_free(cgsw);
      cgs_cap = lock + 256;
      cgsw = (double *)evslcu_malloc(sizeof(double) * evslcu_cgs_work_size(n, cgs_cap));
      if (!cgsw) {
        rc = evsl_seterr(EVSLX_ERR_NOMEM, "ChebLanTr: out of device memory");
        goto done;
      }
    }
    if (trlen > 0) {
      /* thick-restart arrow-head step */
      const int k1 = k - 1;
      double *v = V + (size_t)k1 * n_l;
      double *vnew = v + n_l;
      if ((rc = evslcu_chebav(op, pol->mu, deg, pol->cc, pol->dd, v, vnew, work, NULL))) goto cuda_fail;
      if (lock > 0 && (rc = evslcu_cgs_dgks(n, lock, EVSL_NGS_MAX, Y, (long long)n, vnew, NULL, cgsw)))
        goto cuda_fail;
      for (int i = 0; i < trlen; i++) {
        T[i * lanm1_l + i] = Rval[i];
        wn += fabs(Rval[i]);
      }
      if ((rc = evslcu_dot(n, v, vnew, d_s)) || (rc = evslcu_get_scalars(d_s, h, 1))) goto cuda_fail;
      s[k1] = h[0];
      /* znew -= V(:,1:k) s(1:k) */
      if ((rc = evslcu_h2d(s_dev, s, sizeof(double) * (size_t)k))) goto cuda_fail;
      if ((rc = evslcu_dgemv('N', n, k, -1.0, V, n, s_dev, 1.0, vnew))) goto cuda_fail;
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
        if (do_print) fprintf(fstats, "it %4d: Lucky breakdown, beta = %.15e\n", k, beta);
        if ((rc = evsl_rand_device(n, 1, vrand))) goto done;
        if ((rc = evslcu_chebav(op, pol->mu, deg, pol->cc, pol->dd, vrand, vnew, work, NULL))) goto cuda_fail;
        if (lock > 0 && (rc = evslcu_cgs_dgks(n, lock, EVSL_NGS_MAX, Y, (long long)n, vnew, NULL, cgsw)))
          goto cuda_fail;
        if ((rc = evslcu_cgs_dgks(n, k, EVSL_NGS_MAX, V, (long long)n, vnew, d_beta, cgsw))) goto cuda_fail;
        if ((rc = evslcu_get_scalars(d_beta, h, 1))) goto cuda_fail;
        if ((rc = evslcu_scal(n, 1.0 / h[0], vnew))) goto cuda_fail;
        beta = 0.0;
      } else {
        if ((rc = evslcu_scal(n, 1.0 / beta, vnew))) goto cuda_fail;
      }
      T[k1 * lanm1_l + k] = beta;
      T[k * lanm1_l + k1] = beta;
    }
    Ntest = evsl_max(20, nev - lock + 10);
    int last_jl = 0, jl = 0;
    double last_tr = 0.0, tr = 0.0;
    const double *zold = k > 0 ? V + (size_t)(k - 1) * n_l : NULL;
    while (k < lanm && it < maxit) {
      k++;
      double *v = V + (size_t)(k - 1) * n_l;
      double *vnew = v + n_l;
      if (lock > 0) {
        /* filter, then deflate against the locked vectors, then -beta zold */
        if ((rc = evslcu_chebav(op, pol->mu, deg, pol->cc, pol->dd, v, vnew, work, NULL))) goto cuda_fail;
        if ((rc = evslcu_cgs_dgks(n, lock, EVSL_NGS_MAX, Y, (long long)n, vnew, NULL, cgsw))) goto cuda_fail;
        if (zold && (rc = evslcu_axpy(n, -beta, zold, vnew))) goto cuda_fail;
        if ((rc = evslcu_dot(n, v, vnew, d_alpha))) goto cuda_fail;
      } else {
        evslcu_cheb_epi epi = {zold, -beta, v, d_alpha};
        if ((rc = evslcu_chebav(op, pol->mu, deg, pol->cc, pol->dd, v, vnew, work, &epi))) goto cuda_fail;
      }
      it++;
      if ((rc = evslcu_axpy_ds(n, d_alpha, -1.0, v, vnew))) goto cuda_fail;
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
        if ((rc = evsl_rand_device(n, 1, vrand))) goto done;
        if ((rc = evslcu_chebav(op, pol->mu, deg, pol->cc, pol->dd, vrand, vnew, work, NULL))) goto cuda_fail;
        if (lock > 0 && (rc = evslcu_cgs_dgks(n, lock, EVSL_NGS_MAX, Y, (long long)n, vnew, NULL, cgsw)))
          goto cuda_fail;
        if ((rc = evslcu_cgs_dgks(n, k, EVSL_NGS_MAX, V, (long long)n, vnew, d_beta, cgsw))) goto cuda_fail;
        if ((rc = evslcu_get_scalars(d_beta, h, 1))) goto cuda_fail;
        if ((rc = evslcu_scal(n, 1.0 / h[0], vnew))) goto cuda_fail;
        beta = 0.0;
      } else {
        if ((rc = evslcu_scal(n, 1.0 / beta, vnew))) goto cuda_fail;
      }
      T[k * lanm1_l + (k - 1)] = beta;
      T[(k - 1) * lanm1_l + k] = beta;
      const int k1 = k - trlen - Ntest;
      if (((k1 >= 0) && (k1 % TR_CYCLE == 0)) || (k == lanm) || it == maxit) {
        /* eigenvalues only at a test; the wanted eigenvectors are formed
         * below once the inner loop stops */
        const double te = evsl_timer();
        rc = evsl_tr_eig(k, trlen, T, lanm1, 0.0, Rval, NULL, 0);
        evslstat.t_eig += evsl_timer() - te;
        if (rc) goto done;
        if (k == lanm || it == maxit) break;
        jl = 0;
        tr = 0.0;
        for (int i = 0; i < k; i++) {
          if (Rval[i] + EVSL_DBL_EPS_MULT * DBL_EPSILON >= bar) {
            jl++;
            tr += Rval[i];
          }
        }
        if (fabs(tr - last_tr) <= 2e-12 && jl == last_jl) {
          if (fstats)
            fprintf(fstats, "break: [it %d, k %d]: last_tr %.15e, tr %.15e, last_jl %d  jl %d\n", it, k, last_tr, tr,
                    last_jl, jl);
          break;
        }
        if (fstats)
          fprintf(fstats, "[it %d, k %d] testing: last_tr %.15e, tr %.15e, last_jl %d  jl %d\n", it, k, last_tr, tr,
                  last_jl, jl);
        last_tr = tr;
        last_jl = jl;
      }
    }
    /* eigenvectors of T for the Ritz values that pass 1 keeps */
    {
      const double te = evsl_timer();
      rc = evsl_tr_eig(k, trlen, T, lanm1, bar - 2 * EVSL_DBL_EPS_MULT * DBL_EPSILON, Rval, EvecT, lanm1);
      evslstat.t_eig += evsl_timer() - te;
      if (rc) goto done;
    }
    /* pass 1: Ritz values above bar, their vectors moved to the front */
    jl = 0;
    for (int i = 0; i < k; i++) {
      if (Rval[i] + EVSL_DBL_EPS_MULT * DBL_EPSILON >= bar) {
        if (i != jl) {
          memcpy(EvecT + (size_t)jl * lanm1_l, EvecT + (size_t)i * lanm1_l, sizeof(double) * (size_t)k);
          Rval[jl] = Rval[i];
        }
        resi[jl] = fabs(beta * EvecT[(size_t)jl * lanm1_l + (k - 1)]);
        jl++;
      }
    }
    int ll = 0;
    prtrlen = trlen;
    trlen = 0;
    if (jl > 0) {
      if ((rc = evslcu_h2d(EvecT_dev, EvecT, sizeof(double) * lanm1_l * (size_t)jl))) goto cuda_fail;
      const double trz = evsl_timer();
      if ((rc = evslcu_dgemm('N', 'N', n, jl, k, 1.0, V, n, EvecT_dev, lanm1, 0.0, Rvec, n))) goto cuda_fail;
      /* pass 2: Rayleigh quotients and residuals of all candidates at once */
      double *rn = rnorm, *rl = rnorm + jl, *rr = rnorm + 2 * jl;
      if ((rc = evslcu_ritz_eval(op, n, jl, Rvec, Wt, rn, rl, rr))) goto cuda_fail;
      for (int i = 0; i < jl; i++) {
        double *y = Rvec + (size_t)i * n_l;
        if (rn[i] == 0.0) {
          rc = 2;
          goto done;
        }
        const double t3 = rl[i];
        if (t3 >= aa - EVSL_DBL_EPS_MULT * DBL_EPSILON && t3 <= bb + EVSL_DBL_EPS_MULT * DBL_EPSILON) {
          ll++;
          const double r = rr[i];
          if (r < tol) {
            if (lock >= nev) {
              const int old_nev = nev;
              nev += 1 + (int)(nev * nevInc);
              if (do_print) fprintf(fstats, "-- More eigval found: realloc space for %d evs\n", nev);
              double *Y2 = (double *)evslcu_malloc(sizeof(double) * n_l * (size_t)nev);
              if (!Y2) {
                rc = evsl_seterr(EVSLX_ERR_NOMEM, "ChebLanTr: out of device memory growing the locked set");
                goto done;
              }
              if ((rc = evslcu_d2d(Y2, Y, sizeof(double) * n_l * (size_t)old_nev))) goto cuda_fail;
              evslcu_free(Y);
              Y = Y2;
              Lam = (double *)realloc(Lam, sizeof(double) * (size_t)nev);
              res = (double *)realloc(res, sizeof(double) * (size_t)nev);
            }
            if ((rc = evslcu_d2d(Y + (size_t)lock * n_l, y, sizeof(double) * n_l))) goto cuda_fail;
            Lam[lock] = t3;
            res[lock] = r;
            lock++;
          } else {
            Rval[trlen] = Rval[i];
            if ((rc = evslcu_d2d(V + (size_t)trlen * n_l, y, sizeof(double) * n_l))) goto cuda_fail;
            s[trlen] = beta * EvecT[(size_t)i * lanm1_l + (k - 1)];
            trlen++;
          }
        }
      }
      evslstat.t_ritz += evsl_timer() - trz;
    }
    if (do_print)
      fprintf(fstats, "it %4d:  k %3d, jl %3d, ll %3d, lock %3d, trlen %3d\n", it, k, jl, ll, lock, trlen);
    if ((prtrlen == 0) && (ll == 0)) {
      if (do_print) fprintf(fstats, "--------------------------------------------------\n --> No ev.s left to be computed\n");
      break;
    }
    if (it == maxit) {
      if (do_print) fprintf(fstats, "--------------------------------------------------\n --> Max its reached without convergence\n");
      break;
    }
    memset(T, 0, sizeof(double) * lanm1_l * lanm1_l);
    if ((rc = evslcu_d2d(V + (size_t)trlen * n_l, V + (size_t)k * n_l, sizeof(double) * n_l))) goto cuda_fail;
  }
  if ((rc = evslcu_sync())) goto cuda_fail;
  if (do_print) fprintf(fstats, "     Number of evals found = %d\n--------------------------------------------------\n", lock);
  evslh.last_kdim = it;
  *nev2 = lock;
  *vals = Lam;
  *resW = res;
  *W = Y;
  Lam = res = Y = NULL;
  evslstat.t_iter = evsl_timer() - tall;
  rc = 0;
  goto done;

cuda_fail:
  rc = evsl_seterr(rc, "%s", evslcu_errstr());
done:
  evslcu_free(V);
  free(T);
  evslcu_free(Y);
  free(Lam);
  free(res);
  free(Rval);
  free(resi);
  evslcu_free(Rvec);
  evslcu_free(Wt);
  free(EvecT);
  evslcu_free(EvecT_dev);
  free(s);
  evslcu_free(s_dev);
  evslcu_free(work);
  evslcu_free(vrand);
  evslcu_free(cgsw);
  evslcu_free(ds);
  free(rnorm);
  return rc;
}

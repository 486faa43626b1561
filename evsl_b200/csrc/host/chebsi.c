/*
 * chebsi.c -- polynomial-filtered subspace iteration (reference
 * SRC/chebsi.c:39-336) and the column orthonormalisation it uses
 * (orth, SRC/misc_la.c:317-341).
 *
 * Same algorithm as the reference: V <- orth(p(A) V) with the active columns
 * orthogonalised against the locked ones; every 5 iterations a Rayleigh-Ritz
 * step with p(A) (T = V' p(A) V, dense eigensolve on the host), residuals with
 * respect to p(A) screen candidates (tol/100), candidates are confirmed with
 * A (residual < tol) and locked; stop when all nev columns are locked or
 * NBUF = 2 locked pairs fall outside [a, b].  The filter is applied to all
 * active columns at once with the block kernel (one pass over A per degree
 * for every 8 columns), which gives the same vectors as column-by-column
 * ChebAv.  vinit (n x nev), *Yo: device; *lamo, *reso: host.
 */
#include "internal.h"

#define SI_NBUF 2
#define SI_CVCHECK 5

/* Vo = orthonormalised columns of V (n x k), classical Gram-Schmidt with DGKS. */
static int orth_dev(const double *V, int n, int k, double *Vo, double *cgsw, double *d_nrm) {
  int rc;
  if ((rc = evslcu_copy(n * k, V, Vo))) return rc;
  if ((rc = evslcu_nrm2(n, Vo, d_nrm)) || (rc = evslcu_scal_inv_ds(n, d_nrm, Vo))) return rc;
  for (int i = 1; i < k; i++) {
    double *col = Vo + (size_t)i * n;
    if ((rc = evslcu_cgs_dgks(n, i, EVSL_NGS_MAX, Vo, (long long)n, col, d_nrm, cgsw))) return rc;
    if ((rc = evslcu_scal_inv_ds(n, d_nrm, col))) return rc;
  }
  return 0;
}

int ChebSI(int nev, double *intv, int maxit, double tol, double *vinit, polparams *pol, int *nevo, double **lamo,
           double **Yo, double **reso, FILE *fstats) {
  const double tall = evsl_timer();
  int rc = evsl_require_operator();
  if (rc) return rc;
  const int n = evsl_op()->n;
  const size_t n_l = (size_t)n;
  const double tolP = tol * 0.01;
  *nevo = 0;
  *lamo = NULL;
  *Yo = NULL;
  *reso = NULL;
  if (evsl_check_intv(intv, fstats) < 0) return 0;
  const double aa = intv[0], bb = intv[1];
  const int deg = pol->deg;
  const double gamB = pol->gam, bar = pol->bar;
  if (fstats) fprintf(fstats, "Cheb Poly- deg = %d, gam = %.15e, bar: %.15e\n", deg, gamB, bar);
  if (gamB > 1.0 || gamB < -1.0) {
    fprintf(stdout, "gamB error %.15e\n", gamB);
    return -1;
  }
  if (nev < 1 || nev > n) return evsl_seterr(EVSLX_ERR_ARG, "ChebSI: need 1 <= nev <= n");
  if (fstats) fprintf(fstats, "Step 2: ChebSI, block size = %d\n", nev);
  const evslcu_op *op = evsl_op();
  const size_t nnev = n_l * (size_t)nev;
  double *V = (double *)evslcu_malloc(sizeof(double) * nnev);
  double *PV = (double *)evslcu_malloc(sizeof(double) * nnev);
  double *R = (double *)evslcu_malloc(sizeof(double) * nnev);
  double *buf = (double *)evslcu_malloc(sizeof(double) * nnev);
  double *work = (double *)evslcu_malloc(sizeof(double) * 2 * nnev);
  double *T = (double *)evslcu_malloc(sizeof(double) * (size_t)nev * nev);
  double *evecT_dev = (double *)evslcu_malloc(sizeof(double) * (size_t)nev * nev);
  double *cgsw = (double *)evslcu_malloc(sizeof(double) * evslcu_cgs_work_size(n, nev));
  double *ds = (double *)evslcu_malloc(sizeof(double) * 8);
  double *T_host = (double *)malloc(sizeof(double) * (size_t)nev * nev);
  double *evecT = (double *)malloc(sizeof(double) * (size_t)nev * nev);
  double *evalT = (double *)malloc(sizeof(double) * (size_t)nev);
  double *Lam = (double *)malloc(sizeof(double) * (size_t)nev);
  double *res = (double *)malloc(sizeof(double) * (size_t)nev);
  double *resP = (double *)malloc(sizeof(double) * (size_t)nev);
  int *act_idx = (int *)malloc(sizeof(int) * (size_t)nev);
  int *lock_idx = (int *)malloc(sizeof(int) * (size_t)nev);
  double *Lam_out = NULL, *res_out = NULL, *V_out = NULL;
  int nlock = 0, nact = nev, nlock_ab = 0, it = 0, find_more = 1, nmv = 0;
  if (!V || !PV || !R || !buf || !work || !T || !evecT_dev || !cgsw || !ds || !T_host || !evecT || !evalT || !Lam ||
      !res || !resP || !act_idx || !lock_idx) {
    rc = evsl_seterr(EVSLX_ERR_NOMEM, "ChebSI: out of memory (n=%d, nev=%d)", n, nev);
    goto done;
  }
  double h[2];
  /* V = orth(vinit); PV = p(A) V */
  if ((rc = orth_dev(vinit, n, nev, V, cgsw, ds))) goto cuda_fail;
  if ((rc = evslcu_chebav_block(op, pol->mu, deg, pol->cc, pol->dd, nev, V, PV, work))) goto cuda_fail;
  nmv += deg * nev;
  while (it < maxit && find_more) {
    const size_t nnlock = n_l * (size_t)nlock, nnact = n_l * (size_t)nact;
    if ((rc = evslcu_copy((int)nnact, PV + nnlock, V + nnlock))) goto cuda_fail;
    if (nlock > 0) {
      if ((rc = evslcu_dgemm('T', 'N', nlock, nact, n, 1.0, V, n, V + nnlock, n, 0.0, T, nev)) ||
          (rc = evslcu_dgemm('N', 'N', n, nact, nlock, -1.0, V, n, T, nev, 1.0, V + nnlock, n)))
        goto cuda_fail;
    }
    if ((rc = orth_dev(V + nnlock, n, nact, buf, cgsw, ds)) || (rc = evslcu_copy((int)nnact, buf, V + nnlock)))
      goto cuda_fail;
    if ((rc = evslcu_chebav_block(op, pol->mu, deg, pol->cc, pol->dd, nact, V + nnlock, PV + nnlock, work)))
      goto cuda_fail;
    nmv += deg * nact;
    if (nlock > 0) {
      if ((rc = evslcu_dgemm('T', 'N', nlock, nact, n, 1.0, V, n, PV + nnlock, n, 0.0, T, nev)) ||
          (rc = evslcu_dgemm('N', 'N', n, nact, nlock, -1.0, V, n, T, nev, 1.0, PV + nnlock, n)))
        goto cuda_fail;
    }
    if (((it + 1) % SI_CVCHECK == 0) || ((it + 1) == maxit)) {
      /* Rayleigh-Ritz with p(A) on the active columns */
      if ((rc = evslcu_dgemm('T', 'N', nact, nact, n, 1.0, V + nnlock, n, PV + nnlock, n, 0.0, T, nev))) goto cuda_fail;
      if ((rc = evslcu_d2h(T_host, T, sizeof(double) * (size_t)nev * nev))) goto cuda_fail;
      const double te = evsl_timer();
      rc = evsl_sym_eig(nact, T_host, nev, evecT, nev, evalT + nlock);
      evslstat.t_eig += evsl_timer() - te;
      if (rc) goto done;
      if ((rc = evslcu_h2d(evecT_dev, evecT, sizeof(double) * (size_t)nev * nev))) goto cuda_fail;
      if ((rc = evslcu_dgemm('N', 'N', n, nact, nact, 1.0, V + nnlock, n, evecT_dev, nev, 0.0, buf, n)) ||
          (rc = evslcu_copy((int)nnact, buf, V + nnlock)) ||
          (rc = evslcu_dgemm('N', 'N', n, nact, nact, 1.0, PV + nnlock, n, evecT_dev, nev, 0.0, buf, n)) ||
          (rc = evslcu_copy((int)nnact, buf, PV + nnlock)))
        goto cuda_fail;
      /* R = PV - V diag(evalT) on the active columns */
      for (int i = nlock; i < nev; i++) {
        double *Ri = R + (size_t)i * n_l;
        if ((rc = evslcu_copy(n, PV + (size_t)i * n_l, Ri)) || (rc = evslcu_axpy(n, -evalT[i], V + (size_t)i * n_l, Ri)))
          goto cuda_fail;
      }
      if ((rc = evslcu_colnorms(n, nev - nlock, R + nnlock, resP + nlock))) goto cuda_fail;
      int nlock_new = 0, nlock_ab_new = 0;
      nact = 0;
      for (int i = nlock; i < nev; i++) {
        if (resP[i] < tolP) {
          /* confirm with A: Rayleigh quotient and residual */
          double *Vi = V + (size_t)i * n_l, *Ri = R + (size_t)i * n_l;
          if ((rc = evsl_apply_A(Vi, buf))) goto done;
          nmv++;
          if ((rc = evslcu_dot(n, Vi, buf, ds + 1)) || (rc = evslcu_get_scalars(ds + 1, h, 1))) goto cuda_fail;
          const double rq = h[0];
          if ((rc = evslcu_copy(n, buf, Ri)) || (rc = evslcu_axpy(n, -rq, Vi, Ri)) || (rc = evslcu_nrm2(n, Ri, ds + 2)) ||
              (rc = evslcu_get_scalars(ds + 2, h, 1)))
            goto cuda_fail;
          const double resA = h[0];
          if (resA < tol) {
            lock_idx[nlock_new] = i;
            res[nlock + nlock_new] = resA;
            Lam[nlock + nlock_new] = rq;
            nlock_new++;
            if (rq >= aa - EVSL_DBL_EPS_MULT * DBL_EPSILON && rq <= bb + EVSL_DBL_EPS_MULT * DBL_EPSILON) nlock_ab_new++;
          } else {
            act_idx[nact++] = i;
          }
        } else {
          act_idx[nact++] = i;
        }
      }
      /* locked columns first, then the active ones */
      for (int i = 0; i < nlock_new; i++) {
        if ((rc = evslcu_copy(n, V + (size_t)lock_idx[i] * n_l, buf + nnlock + (size_t)i * n_l)) ||
            (rc = evslcu_copy(n, PV + (size_t)lock_idx[i] * n_l, R + nnlock + (size_t)i * n_l)))
          goto cuda_fail;
      }
      for (int i = 0; i < nact; i++) {
        if ((rc = evslcu_copy(n, V + (size_t)act_idx[i] * n_l, buf + nnlock + (size_t)(nlock_new + i) * n_l)) ||
            (rc = evslcu_copy(n, PV + (size_t)act_idx[i] * n_l, R + nnlock + (size_t)(nlock_new + i) * n_l)))
          goto cuda_fail;
      }
      const size_t nn_rest = n_l * (size_t)(nev - nlock);
      if ((rc = evslcu_copy((int)nn_rest, buf + nnlock, V + nnlock)) ||
          (rc = evslcu_copy((int)nn_rest, R + nnlock, PV + nnlock)))
        goto cuda_fail;
      nlock += nlock_new;
      nlock_ab += nlock_ab_new;
      if (fstats) fprintf(fstats, "it %4d:   nMV %7d,  nlock %3d, nlock_ab  %3d\n", it + 1, nmv, nlock, nlock_ab);
      if (((nlock - nlock_ab) >= SI_NBUF) || (nlock == nev)) {
        find_more = 0;
        if (fstats) fprintf(fstats, " No ev.s left to be computed\n Number of evals found = %d\n", nlock_ab);
      }
    }
    it++;
  }
  /* keep the locked pairs inside [a, b] */
  Lam_out = (double *)malloc(sizeof(double) * (size_t)nev);
  res_out = (double *)malloc(sizeof(double) * (size_t)nev);
  V_out = (double *)evslcu_malloc(sizeof(double) * nnev);
  if (!Lam_out || !res_out || !V_out) {
    rc = evsl_seterr(EVSLX_ERR_NOMEM, "ChebSI: out of memory");
    goto done;
  }
  int idx = 0;
  for (int i = 0; i < nlock; i++) {
    const double t = Lam[i];
    if (t >= aa - EVSL_DBL_EPS_MULT * DBL_EPSILON && t <= bb + EVSL_DBL_EPS_MULT * DBL_EPSILON) {
      Lam_out[idx] = t;
      res_out[idx] = res[i];
      if ((rc = evslcu_copy(n, V + (size_t)i * n_l, V_out + (size_t)idx * n_l))) goto cuda_fail;
      idx++;
    }
  }
  if ((rc = evslcu_sync())) goto cuda_fail;
  *nevo = idx;
  *lamo = Lam_out;
  *reso = res_out;
  *Yo = V_out;
  Lam_out = res_out = V_out = NULL;
  evslstat.t_iter = evsl_timer() - tall;
  rc = 0;
  goto done;
cuda_fail:
  rc = evsl_seterr(rc, "%s", evslcu_errstr());
done:
  evslcu_free(V);
  evslcu_free(PV);
  evslcu_free(R);
  evslcu_free(buf);
  evslcu_free(work);
  evslcu_free(T);
  evslcu_free(evecT_dev);
  evslcu_free(cgsw);
  evslcu_free(ds);
  evslcu_free(V_out);
  free(T_host);
  free(evecT);
  free(evalT);
  free(Lam);
  free(res);
  free(resP);
  free(act_idx);
  free(lock_idx);
  free(Lam_out);
  free(res_out);
  return rc;
}

/*
 * landos.c -- Lanczos density of states and the slicer that uses it:
 * LanDos (SRC/landos.c:37-200), simpson (SRC/simpson.c:25-50), spslicer2
 * (SRC/spslice2.c:25-45) and the exact-spectrum DOS exDOS
 * (SRC/exDOS.c:17-67).
 *
 * LanDos runs nvec Lanczos processes of msteps steps on A, each from a
 * normal random vector of the library generator, with full
 * reorthogonalisation; the Ritz values and the squared first components of
 * the tridiagonal eigenvectors (Lanczos quadrature) place Gaussians on the
 * grid linspace(max(a, lmin), min(b, lmax), npts).  The Lanczos vectors,
 * products and reorthogonalisation run on the GPU (reorthogonalisation as
 * classical Gram-Schmidt with the DGKS test, where the reference runs one
 * modified Gram-Schmidt pass); the quadrature weights come from QL applied
 * to e_1 only; the Gaussian sums, scaling and Simpson integration are the
 * reference's host loops.  As in the reference, a lucky breakdown shortens
 * msteps for all later vectors, and a small beta takes the reference's
 * restart branch (one generator draw, a second reorthogonalisation, beta
 * set to 0).
 */
#include "internal.h"

void simpson(double *xi, double *yi, int npts) {
  double tc = 0.0, ti, tm, ysav;
  int i = 1;
  ysav = yi[0];
  yi[0] = 0;
  while (i < npts - 1) {
    ti = (xi[i] - xi[i - 1]) * (ysav + yi[i]) / 2.0;
    tm = tc + ti;
    ti = (xi[i + 1] - xi[i - 1]) * (ysav + 4 * yi[i] + yi[i + 1]) / 6.0;
    tc += ti;
    yi[i] = tm;
    ysav = yi[i + 1];
    yi[i + 1] = tc;
    i += 2;
  }
  if (i == npts - 1) {
    ti = (xi[i] - xi[i - 1]) * (yi[i] + ysav) / 2.0;
    yi[i] = tc + ti;
  }
}

void spslicer2(double *xi, double *yi, int n_int, int npts, double *sli) {
  simpson(xi, yi, npts);
  double t = yi[0];
  const double want = (yi[npts - 1] - yi[0]) / (double)n_int;
  int ls = 0;
  sli[0] = xi[0];
  for (int k = 1; k < npts; k++) {
    if (yi[k] - t >= want) {
      ls = ls + 1;
      /* the reference writes sli[ls] unchecked; a crossing past the last
       * slice would be overwritten by the final boundary anyway */
      if (ls <= n_int) sli[ls] = xi[k];
      t = yi[k];
    }
  }
  sli[n_int] = xi[npts - 1];
}

int exDOS(double *vals, int n, int npts, double *x, double *y, double *intv) {
  int j = 0;
  const double lm = intv[2], lM = intv[3];
  const double kappa = 1.25;
  const int M = evsl_min(n, 30);
  const double H = (lM - lm) / (M - 1);
  const double sigma = H / sqrt(8 * log(kappa));
  const double a = intv[0], b = intv[1];
  const double sigma2 = 2 * sigma * sigma;
  const double tol = 1e-08;
  const double width = sigma * sqrt(-2.0 * log(tol));
  linspace(a, b, npts, x);
  const double h = x[1] - x[0];
  memset(y, 0, sizeof(double) * (size_t)npts);
  for (int i = 0; i < n; i++) {
    const double t = vals[i];
    if (t < a || t > b) continue;
    j = evsl_max((int)((t - a - width) / h), 0);
    for (double xi = a + j * h; xi <= evsl_min(t + width, b); xi += h) {
      if (j >= npts) break; /* the reference relies on rounding to stop here */
      y[j++] += exp(-(xi - t) * (xi - t) / sigma2);
    }
  }
  if (j == 0) return 1;
  const double scaling = 1.0 / (n * sqrt(sigma2 * EVSL_PI));
  for (int i = 0; i < npts; i++) y[i] = scaling * y[i];
  return 0;
}

int LanDos(const int nvec, int msteps, const int npts, double *xdos, double *ydos, double *neig,
           const double *const intv) {
  int rc = evsl_require_operator();
  if (rc) return rc;
  if (nvec < 1 || msteps < 1 || npts < 2 || !xdos || !ydos || !neig || !intv)
    return evsl_seterr(EVSLX_ERR_ARG, "LanDos: bad arguments");
  const int n = evsl_op()->n;
  const size_t n_l = (size_t)n;
  const double lm = intv[2], lM = intv[3];
  const double tolBdwn = 1.e-13 * (fabs(lM) + fabs(lm));
  const double aa = evsl_max(intv[0], intv[2]);
  const double bb = evsl_min(intv[1], intv[3]);
  const double kappa = 1.25;
  const int M = evsl_min(msteps, 30);
  const double H = (lM - lm) / (M - 1);
  const double sigma = H / sqrt(8 * log(kappa));
  const double sigma2 = 2 * sigma * sigma;
  const double tol = 1e-08;
  const double width = sigma * sqrt(-2.0 * log(tol));
  linspace(aa, bb, npts, xdos);
  double *y = (double *)calloc((size_t)npts, sizeof(double));
  double *alp = (double *)malloc(sizeof(double) * (size_t)msteps);
  double *bet = (double *)malloc(sizeof(double) * (size_t)msteps);
  double *ritz = (double *)malloc(sizeof(double) * (size_t)msteps);
  double *z1 = (double *)malloc(sizeof(double) * (size_t)msteps);
  double *v = (double *)evslcu_malloc(sizeof(double) * n_l);
  double *V = (double *)evslcu_malloc(sizeof(double) * n_l * ((size_t)msteps + 1));
  double *cgsw = (double *)evslcu_malloc(sizeof(double) * evslcu_cgs_work_size(n, msteps + 1));
  double *ds = (double *)evslcu_malloc(sizeof(double) * 4);
  double h[2];
  if (!y || !alp || !bet || !ritz || !z1 || !v || !V || !cgsw || !ds) {
    rc = evsl_seterr(EVSLX_ERR_NOMEM, "LanDos: out of memory (n=%d, msteps=%d)", n, msteps);
    goto done;
  }
  for (int m = 0; m < nvec; m++) {
    randn_double_device(n, v);
    if ((rc = evslcu_dot(n, v, v, ds)) || (rc = evslcu_get_scalars(ds, h, 1))) goto cuda_fail;
    if ((rc = evslcu_scal(n, 1.0 / sqrt(h[0]), v)) || (rc = evslcu_copy(n, v, V))) goto cuda_fail;
    double wn = 0.0;
    for (int j = 0; j < msteps; j++) {
      double *vj = V + (size_t)j * n_l, *z = V + (size_t)(j + 1) * n_l;
      if ((rc = evsl_apply_A(vj, z))) goto done;
      if (j && (rc = evslcu_axpy(n, -bet[j - 1], V + (size_t)(j - 1) * n_l, z))) goto cuda_fail;
      if ((rc = evslcu_dot(n, z, vj, ds)) || (rc = evslcu_axpy_ds(n, ds, -1.0, vj, z))) goto cuda_fail;
      if ((rc = evslcu_cgs_dgks(n, j + 1, EVSL_NGS_MAX, V, (long long)n, z, ds + 2, cgsw))) goto cuda_fail;
      if ((rc = evslcu_dot(n, z, z, ds + 1)) || (rc = evslcu_get_scalars(ds, h, 2))) goto cuda_fail;
      alp[j] = h[0];
      wn += alp[j] * alp[j];
      bet[j] = h[1];
      if (bet[j] * (j + 1) < EVSL_ORTH_TOL * wn) {
        fprintf(stdout, "lanbounds: lucky break, j=%d, beta=%e, break\n", j, bet[j]);
        msteps = j + 1;
        break;
      }
      if (bet[j] > tolBdwn) {
        wn += 2.0 * bet[j];
        bet[j] = sqrt(bet[j]);
        if ((rc = evslcu_scal(n, 1.0 / bet[j], z))) goto cuda_fail;
      } else {
        randn_double_device(n, v); /* drawn but unused, as in the reference */
        if ((rc = evslcu_cgs_dgks(n, j + 1, EVSL_NGS_MAX, V, (long long)n, z, ds + 2, cgsw)) ||
            (rc = evslcu_dot(n, z, z, ds + 1)) || (rc = evslcu_get_scalars(ds + 1, h, 1)))
          goto cuda_fail;
        bet[j] = h[0];
        wn += 2.0 * bet[j];
        bet[j] = sqrt(bet[j]);
        if ((rc = evslcu_scal(n, 1.0 / bet[j], z))) goto cuda_fail;
        bet[j] = 0;
      }
    }
    const double te = evsl_timer();
    rc = evsl_trid_eig_first(msteps, alp, bet, ritz, z1);
    evslstat.t_eig += evsl_timer() - te;
    if (rc) goto done;
    for (int i = 0; i < msteps; i++) {
      const double g2 = z1[i] * z1[i];
      const double t = ritz[i];
      for (int j = 0; j < npts; j++)
        if (fabs(xdos[j] - t) < width) y[j] += g2 * exp(-((xdos[j] - t) * (xdos[j] - t)) / sigma2);
    }
  }
  {
    const double scaling = 1.0 / (nvec * sqrt(sigma2 * EVSL_PI));
    for (int i = 0; i < npts; i++) y[i] = scaling * y[i];
    memcpy(ydos, y, sizeof(double) * (size_t)npts);
    simpson(xdos, y, npts);
    *neig = y[npts - 1] * n;
  }
  rc = 0;
  goto done;
cuda_fail:
  rc = evsl_seterr(rc, "%s", evslcu_errstr());
done:
  free(y);
  free(alp);
  free(bet);
  free(ritz);
  free(z1);
  evslcu_free(v);
  evslcu_free(V);
  evslcu_free(cgsw);
  evslcu_free(ds);
  return rc;
}

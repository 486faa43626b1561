/*
 * spslice.c -- KPM density of states and equal-count spectrum slicing.
 *
 * kpmdos follows SRC/spslice.c:29-148.  The reference runs the damped
 * Chebyshev recurrence probe by probe (nvec x Mdeg SpMVs, one D->H dot per
 * step).  Here all probes advance together as one block recurrence on the GPU
 * (one pass over A per degree, dot products fused into the same kernel); the
 * raw dot products come back once and are accumulated into mu and the count
 * on the host in the reference's order (probe-major, then degree), so the
 * only difference from the reference is the summation order inside each dot.
 *
 * spslicer / intChx follow SRC/spslice.c:155-297 (host, scalar FP64; the
 * integrals are O(npts * Mdeg) sine evaluations).
 */
#include "internal.h"

/* Accumulation of the moments and the eigenvalue count from the raw dot
 * products dots[k*nvec + m] = (T_{k+1}(A~) v_m) . v_m, in the reference's
 * order (probe-major, then degree; SRC/spslice.c:76-136).  Host only. */
int evslx_kpm_accumulate(int Mdeg, int damping, int nvec, int n, double *intv, const double *dots, double *mu,
                         double *ecnt) {
  if (evsl_check_intv(intv, stdout) < 0) return -1;
  if (Mdeg < 1 || nvec < 1 || n < 1 || !dots || !mu || !ecnt)
    return evsl_seterr(EVSLX_ERR_ARG, "kpm accumulate: bad arguments");
  const double aa = evsl_max(intv[0], intv[2]), bb = evsl_min(intv[1], intv[3]);
  const double ctr = (intv[3] + intv[2]) / 2.0, wid = (intv[3] - intv[2]) / 2.0;
  double t = evsl_max(-1.0 + DBL_EPSILON, (aa - ctr) / wid);
  const double beta1 = acos(t);
  t = evsl_min(1.0 - DBL_EPSILON, (bb - ctr) / wid);
  const double beta2 = acos(t);
  double *jac = (double *)malloc(sizeof(double) * ((size_t)Mdeg + 1));
  if (!jac) return evsl_seterr(EVSLX_ERR_NOMEM, "kpmdos: out of memory");
  dampcf(Mdeg, damping, jac);
  jac[0] = 1.0;
  memset(mu, 0, sizeof(double) * ((size_t)Mdeg + 1));
  double tcnt = 0.0;
  for (int m = 0; m < nvec; m++) {
    mu[0] += jac[0];
    tcnt -= jac[0] * (beta2 - beta1);
    for (int k = 0; k < Mdeg; k++) {
      const int k1 = k + 1;
      const double tk = 2 * jac[k1] * dots[(size_t)k * nvec + m];
      mu[k1] += tk;
      tcnt -= tk * (sin(k1 * beta2) - sin(k1 * beta1)) / k1;
    }
  }
  t = 1.0 / (((double)nvec) * EVSL_PI);
  for (int k = 0; k <= Mdeg; k++) mu[k] = t * mu[k];
  tcnt *= t * ((double)n);
  *ecnt = tcnt;
  free(jac);
  return 0;
}

/* Raw KPM dot products for device probes (column-major n x nvec), computed
 * 64 probes at a time as block recurrences. dots: host, Mdeg x nvec. */
int evslx_kpm_dots(int Mdeg, int nvec, double *intv, const double *probes, double *dots) {
  int rc = evsl_require_operator();
  if (rc) return rc;
  if (evsl_check_intv(intv, stdout) < 0) return -1;
  if (Mdeg < 1 || nvec < 1 || !probes || !dots) return evsl_seterr(EVSLX_ERR_ARG, "kpm dots: bad arguments");
  const int n = evsl_op()->n;
  const double ctr = (intv[3] + intv[2]) / 2.0, wid = (intv[3] - intv[2]) / 2.0;
  const int group = 64;
  evslcu_timer *tm = evslcu_timer_start();
  for (int g0 = 0; g0 < nvec && !rc; g0 += group) {
    const int cnt = evsl_min(group, nvec - g0);
    double *gd = (double *)malloc(sizeof(double) * (size_t)Mdeg * cnt);
    if (!gd) {
      rc = evsl_seterr(EVSLX_ERR_NOMEM, "kpmdos: out of memory");
      break;
    }
    rc = evslcu_kpm_dots(evsl_op(), n, Mdeg, cnt, probes + (size_t)g0 * n, ctr, wid, gd);
    if (rc) rc = evsl_seterr(rc, "%s", evslcu_errstr());
    for (int k = 0; !rc && k < Mdeg; k++)
      for (int p = 0; p < cnt; p++) dots[(size_t)k * nvec + g0 + p] = gd[(size_t)k * cnt + p];
    free(gd);
  }
  evslh.last_kpm_seconds = evslcu_timer_stop(tm);
  return rc;
}

static int kpm_run(int Mdeg, int damping, int nvec, double *intv, const double *probes, double *mu, double *ecnt) {
  int rc = evsl_require_operator();
  if (rc) return rc;
  if (evsl_check_intv(intv, stdout) < 0) return -1;
  if (Mdeg < 1 || nvec < 1) return evsl_seterr(EVSLX_ERR_ARG, "kpmdos: Mdeg and nvec must be positive");
  const int n = evsl_op()->n;
  if (intv[0] < intv[2] || intv[1] > intv[3])
    fprintf(stdout, " warning [%s (%d)]: interval (%e, %e) is adjusted to (%e, %e)\n", __FILE__, __LINE__, intv[0],
            intv[1], evsl_max(intv[0], intv[2]), evsl_min(intv[1], intv[3]));
  double *dots = (double *)malloc(sizeof(double) * (size_t)Mdeg * (size_t)nvec);
  if (!dots) return evsl_seterr(EVSLX_ERR_NOMEM, "kpmdos: out of memory");
  rc = evslx_kpm_dots(Mdeg, nvec, intv, probes, dots);
  if (!rc) rc = evslx_kpm_accumulate(Mdeg, damping, nvec, n, intv, dots, mu, ecnt);
  free(dots);
  return rc;
}

int kpmdos(int Mdeg, int damping, int nvec, double *intv, double *mu, double *ecnt) {
  int rc = evsl_require_operator();
  if (rc) return rc;
  if (evsl_check_intv(intv, stdout) < 0) return -1;
  if (nvec < 1) return evsl_seterr(EVSLX_ERR_ARG, "kpmdos: nvec must be positive");
  const int n = evsl_op()->n;
  /* probes are drawn on the device, one draw per probe as in the reference
   * (rand_double_device, SRC/spslice.c:90) */
  double *probes = (double *)evslcu_malloc(sizeof(double) * (size_t)n * nvec);
  if (!probes) return evsl_seterr(EVSLX_ERR_NOMEM, "kpmdos: out of device memory");
  rc = evsl_rand_device(n, nvec, probes);
  if (!rc) rc = kpm_run(Mdeg, damping, nvec, intv, probes, mu, ecnt);
  evslcu_free(probes);
  return rc;
}

int evslx_kpmdos_probes(int Mdeg, int damping, int nvec, double *intv, const double *probes, double *mu,
                        double *ecnt) {
  if (!probes) return evsl_seterr(EVSLX_ERR_ARG, "kpmdos: probes must be a device array");
  return kpm_run(Mdeg, damping, nvec, intv, probes, mu, ecnt);
}

/* Allocation-free kpmdos with caller probes (no counterpart in the
 * reference).  Same algorithm and arithmetic as evslx_kpmdos_probes; the
 * damping factors and sine differences are formed on this thread's stack and
 * everything else lives in the library's fixed device scratch. */
int evslx_kpmdos_probes_noalloc(int Mdeg, int damping, int nvec, double *intv, const double *probes, double *mu,
                                double *ecnt) {
  int rc = evsl_require_operator();
  if (rc) return rc;
  if (evsl_check_intv(intv, stdout) < 0) return -1;
  if (!probes || !mu || !ecnt) return evsl_seterr(EVSLX_ERR_ARG, "kpmdos: probes, mu and ecnt are required");
  if (Mdeg < 1 || Mdeg > EVSLX_NOALLOC_KPM_MAX_DEG || nvec < 1 || nvec > 128)
    return evsl_seterr(EVSLX_ERR_ARG,
                       "allocation-free kpmdos: need 1 <= Mdeg <= %d and 1 <= nvec <= 128 (got Mdeg=%d nvec=%d)",
                       EVSLX_NOALLOC_KPM_MAX_DEG, Mdeg, nvec);
  const int n = evsl_op()->n;
  const double aa = evsl_max(intv[0], intv[2]), bb = evsl_min(intv[1], intv[3]);
  const double ctr = (intv[3] + intv[2]) / 2.0, wid = (intv[3] - intv[2]) / 2.0;
  double t = evsl_max(-1.0 + DBL_EPSILON, (aa - ctr) / wid);
  const double beta1 = acos(t);
  t = evsl_min(1.0 - DBL_EPSILON, (bb - ctr) / wid);
  const double beta2 = acos(t);
  double jac[EVSLX_NOALLOC_KPM_MAX_DEG + 1];
  double sdiff[EVSLX_NOALLOC_KPM_MAX_DEG];
  dampcf(Mdeg, damping, jac);
  jac[0] = 1.0;
  for (int k = 0; k < Mdeg; k++) {
    const int k1 = k + 1;
    sdiff[k] = sin(k1 * beta2) - sin(k1 * beta1);
  }
  const double scale = 1.0 / (((double)nvec) * EVSL_PI);
  rc = evslcu_kpm_noalloc(evsl_op(), n, Mdeg, nvec, probes, ctr, wid, jac, sdiff, beta2 - beta1, scale, mu, ecnt);
  if (rc) return evsl_seterr(rc, "%s", evslcu_errstr());
  return 0;
}

/* integrals of the KPM DOS from xi[0] to each xi[j] */
static int int_chx(int Mdeg, const double *mu, int npts, const double *xi, double *yi) {
  double *thetas = (double *)malloc(sizeof(double) * (size_t)npts);
  if (!thetas) return evsl_seterr(EVSLX_ERR_NOMEM, "spslicer: out of memory");
  for (int j = 0; j < npts; j++) thetas[j] = acos(xi[j]);
  const double theta0 = thetas[0];
  for (int j = 0; j < npts; j++) yi[j] = mu[0] * (theta0 - thetas[j]);
  for (int k = 1; k < Mdeg + 1; k++) {
    const double val0 = sin(k * theta0) / k;
    for (int j = 0; j < npts; j++) yi[j] += mu[k] * (val0 - sin(k * thetas[j]) / k);
  }
  free(thetas);
  return 0;
}

int spslicer(double *sli, double *mu, int Mdeg, double *intv, int n_int, int npts) {
  int err = 0;
  if (evsl_check_intv(intv, stdout) < 0) return -1;
  if (n_int < 1) return evsl_seterr(EVSLX_ERR_ARG, "spslicer: n_int must be positive");
  const double aa = evsl_max(intv[0], intv[2]), bb = evsl_min(intv[1], intv[3]);
  if (intv[0] < intv[2] || intv[1] > intv[3])
    fprintf(stdout, " warning [%s (%d)]:  interval (%e, %e) is adjusted to (%e, %e)\n", __FILE__, __LINE__,
            intv[0], intv[1], aa, bb);
  memset(sli, 0, sizeof(double) * ((size_t)n_int + 1));
  if (n_int == 1) {
    sli[0] = intv[0];
    sli[1] = intv[1];
    return 0;
  }
  const double ctr = (intv[3] + intv[2]) / 2, wid = (intv[3] - intv[2]) / 2;
  double aL = (aa - ctr) / wid, bL = (bb - ctr) / wid;
  aL = evsl_max(aL, -1.0);
  bL = evsl_min(bL, 1.0);
  npts = evsl_max(npts, 2 * n_int + 1);
  double *xi = (double *)malloc(sizeof(double) * (size_t)npts);
  double *yi = (double *)malloc(sizeof(double) * (size_t)npts);
  if (!xi || !yi) {
    free(xi);
    free(yi);
    return evsl_seterr(EVSLX_ERR_NOMEM, "spslicer: out of memory");
  }
  linspace(aL, bL, npts, xi);
  if (int_chx(Mdeg, mu, npts, xi, yi)) {
    free(xi);
    free(yi);
    return EVSLX_ERR_NOMEM;
  }
  double target = yi[npts - 1] / (double)n_int;
  int ls = 0, ii = 0;
  sli[ls] = intv[0];
  while (++ls < n_int) {
    while (ii < npts && yi[ii] < target) ii++;
    if (ii == npts) break;
    /* take the closer of the two grid points around the target */
    if (ii > 0 && (target - yi[ii - 1]) < (yi[ii] - target)) ii--;
    sli[ls] = ctr + wid * xi[ii];
    target = yi[ii] + (yi[npts - 1] - yi[ii]) / (n_int - ls);
  }
  sli[n_int] = intv[1];
  if (ls != n_int) err = 1;
  for (ii = 1; ii <= n_int; ii++) {
    if (sli[ii] < sli[ii - 1]) {
      err += 2;
      break;
    }
  }
  free(xi);
  free(yi);
  return err;
}

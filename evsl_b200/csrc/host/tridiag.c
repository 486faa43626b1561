/*
 * tridiag.c -- host FP64 eigensolvers for the small projected problems of
 * filtered Lanczos.
 *
 * The reference calls vendored f2c LAPACK for these (SRC/misc_la.c:33-209:
 * dstev for the tridiagonal T_k, dsyev for the dense thick-restart T).  This
 * file provides its own implementations of standard published methods:
 *
 *   evsl_trid_eigvals  implicit QL iteration with Wilkinson shifts on a
 *                      symmetric tridiagonal matrix (Wilkinson & Reinsch,
 *                      "Handbook for Automatic Computation II", tql1/tql2;
 *                      Golub & Van Loan, Matrix Computations, sec. 8.3),
 *                      eigenvalues only, O(n^2).
 *   evsl_trid_eigvecs  eigenvectors of selected eigenvalues by inverse
 *                      iteration with a pivoted tridiagonal LU and
 *                      re-orthogonalisation inside clusters of close
 *                      eigenvalues (Peters & Wilkinson 1971; the approach
 *                      of LAPACK's dstein), O(n) per vector and iteration.
 *   evsl_tr_eig        the thick-restart matrix (diagonal block + spike row
 *                      + tridiagonal tail): the leading block is reduced to
 *                      tridiagonal form by a Lanczos run on the diagonal
 *                      block started from the spike (full
 *                      reorthogonalisation), which leaves the whole matrix
 *                      tridiagonal; then QL for all eigenvalues and inverse
 *                      iteration for the wanted vectors only.
 *   evsl_sym_eig       dense symmetric eigenproblem: Householder
 *                      tridiagonalisation, then implicit QL with rotations
 *                      accumulated (eigenvalues ascending, vectors in Q).
 *
 * Eigenvalues agree with LAPACK's to a few ulps of ||T||; eigenvectors for
 * eigenvalues closer than CLUSTER_TOL * ||T|| are made mutually orthogonal.
 */
#include "internal.h"

#include <pthread.h>
#include <unistd.h>

#define QL_MAX_ITER 60
#define INVIT_ITERS 3
#define CLUSTER_TOL 1e-7

/* Implicit QL sweep on (d, e); e[n-1] is scratch.  Z (zrows x n,
 * column-major, ld ldz) accumulates the rotations when not NULL: zrows = n
 * gives the eigenvectors, zrows = 1 with Z = e_1^T only their first
 * components. */
static int ql_implicit_rows(int n, double *d, double *e, double *Z, int ldz, int zrows) {
  if (n <= 1) return 0;
  e[n - 1] = 0.0;
  for (int l = 0; l < n; l++) {
    int iter = 0, m;
    do {
      for (m = l; m < n - 1; m++) {
        const double dd = fabs(d[m]) + fabs(d[m + 1]);
        if (fabs(e[m]) <= DBL_EPSILON * dd) break;
      }
      if (m != l) {
        if (iter++ == QL_MAX_ITER) return -1;
        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        double r = hypot(g, 1.0);
        g = d[m] - d[l] + e[l] / (g + copysign(r, g));
        double s = 1.0, c = 1.0, p = 0.0;
        int i;
        for (i = m - 1; i >= l; i--) {
          double f = s * e[i];
          const double b = c * e[i];
          r = hypot(f, g);
          e[i + 1] = r;
          if (r == 0.0) {
            d[i + 1] -= p;
            e[m] = 0.0;
            break;
          }
          s = f / r;
          c = g / r;
          g = d[i + 1] - p;
          r = (d[i] - g) * s + 2.0 * c * b;
          p = s * r;
          d[i + 1] = g + p;
          g = c * r - b;
          if (Z) {
            double *zi = Z + (size_t)i * ldz, *zi1 = Z + (size_t)(i + 1) * ldz;
            for (int k = 0; k < zrows; k++) {
              f = zi1[k];
              zi1[k] = s * zi[k] + c * f;
              zi[k] = c * zi[k] - s * f;
            }
          }
        }
        if (r == 0.0 && i >= l) continue;
        d[l] -= p;
        e[l] = g;
        e[m] = 0.0;
      }
    } while (m != l);
  }
  return 0;
}

static int ql_implicit(int n, double *d, double *e, double *Z, int ldz) {
  return ql_implicit_rows(n, d, e, Z, ldz, n);
}

/* Sort eigenvalues ascending (and the matching columns of Z). */
static void sort_pairs_rows(int n, double *w, double *Z, int ldz, double *tmp, int zrows) {
  for (int i = 0; i < n - 1; i++) {
    int k = i;
    double p = w[i];
    for (int j = i + 1; j < n; j++)
      if (w[j] < p) {
        k = j;
        p = w[j];
      }
    if (k != i) {
      w[k] = w[i];
      w[i] = p;
      if (Z) {
        memcpy(tmp, Z + (size_t)i * ldz, sizeof(double) * zrows);
        memcpy(Z + (size_t)i * ldz, Z + (size_t)k * ldz, sizeof(double) * zrows);
        memcpy(Z + (size_t)k * ldz, tmp, sizeof(double) * zrows);
      }
    }
  }
}

static void sort_pairs(int n, double *w, double *Z, int ldz, double *tmp) { sort_pairs_rows(n, w, Z, ldz, tmp, n); }

static int cmp_double(const void *a, const void *b) {
  const double x = *(const double *)a, y = *(const double *)b;
  return (x > y) - (x < y);
}

int evsl_trid_eigvals(int n, const double *d, const double *e, double *w) {
  if (n <= 0) return 0;
  double *ee = (double *)malloc(sizeof(double) * (size_t)n);
  if (!ee) return evsl_seterr(EVSLX_ERR_NOMEM, "tridiagonal eigensolver: out of memory");
  memcpy(w, d, sizeof(double) * (size_t)n);
  if (n > 1) memcpy(ee, e, sizeof(double) * (size_t)(n - 1));
  int rc = ql_implicit(n, w, ee, NULL, 0);
  free(ee);
  if (rc) return evsl_seterr(EVSLX_ERR_NUMERIC, "tridiagonal QL did not converge");
  qsort(w, (size_t)n, sizeof(double), cmp_double);
  return 0;
}

/* Eigenvalues for the Lanczos convergence tests: on the GPU (multisection,
 * evslcu_trid_eigvals_above) from TRID_GPU_MIN rows on, where the host QL's
 * O(k^2) work per test would dominate small-matrix solves; the host QL below
 * that.  Both are backward stable; they agree to a few ulps.  The trace test
 * reads only the eigenvalues >= xmin: on the GPU the others are not
 * computed (their entries hold values below xmin). */
#define TRID_GPU_MIN 64
int evsl_trid_eigvals_test(int n, const double *d, const double *e, double xmin, double *w) {
  if (n < TRID_GPU_MIN) return evsl_trid_eigvals(n, d, e, w);
  const int rc = evslcu_trid_eigvals_above(n, d, e, xmin, w);
  if (rc) return evsl_seterr(EVSLX_ERR_CUDA, "%s", evslcu_errstr());
  return 0;
}

int evsl_trid_test_start(int n, const double *d, const double *e, double xmin) {
  if (n < TRID_GPU_MIN) return 0;
  const int rc = evslcu_trid_eigvals_async(n, d, e, xmin);
  if (rc) return evsl_seterr(EVSLX_ERR_CUDA, "%s", evslcu_errstr());
  return 1;
}

int evsl_trid_test_ready(void) { return evslcu_trid_eigvals_async_ready(); }

int evsl_trid_test_wait(double *w) {
  const int rc = evslcu_trid_eigvals_async_wait(w);
  if (rc) return evsl_seterr(EVSLX_ERR_CUDA, "%s", evslcu_errstr());
  return 0;
}

/* Eigenvalues (ascending) of the symmetric tridiagonal (d, e) and the first
 * component of each normalised eigenvector (the Lanczos quadrature weights
 * come from their squares): the QL rotations are applied to e_1^T only. */
int evsl_trid_eig_first(int n, const double *d, const double *e, double *w, double *z1) {
  if (n <= 0) return 0;
  double *ee = (double *)malloc(sizeof(double) * (size_t)n);
  if (!ee) return evsl_seterr(EVSLX_ERR_NOMEM, "tridiagonal eigensolver: out of memory");
  memcpy(w, d, sizeof(double) * (size_t)n);
  if (n > 1) memcpy(ee, e, sizeof(double) * (size_t)(n - 1));
  for (int i = 0; i < n; i++) z1[i] = (i == 0) ? 1.0 : 0.0;
  int rc = ql_implicit_rows(n, w, ee, z1, 1, 1);
  if (!rc) {
    double tmp;
    sort_pairs_rows(n, w, z1, 1, &tmp, 1);
  }
  free(ee);
  if (rc) return evsl_seterr(EVSLX_ERR_NUMERIC, "tridiagonal QL did not converge");
  return 0;
}

/* SplitMix64 output function; used for reproducible start vectors. */
static uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* Inverse iteration for the vectors j0 <= j < j1 (shifts and cluster starts
 * precomputed); a vector depends only on its shift and the earlier vectors of
 * its cluster, so ranges that start at a cluster start run independently. */
typedef struct {
  int n, ldz, j0, j1, rc;
  const double *d, *e, *shift;
  const int *cst;
  double *Z, tiny;
} invit_job;

static int invit_range(invit_job *jb) {
  const int n = jb->n, ldz = jb->ldz;
  const double *d = jb->d, *e = jb->e;
  const double tiny = jb->tiny;
  double *Z = jb->Z;
  double *buf = (double *)malloc(sizeof(double) * (size_t)n * 8);
  unsigned char *swp = (unsigned char *)malloc((size_t)n);
  if (!buf || !swp) {
    free(buf);
    free(swp);
    return EVSLX_ERR_NOMEM;
  }
  double *dg = buf, *du = buf + n, *u0 = buf + 2 * n, *u1 = buf + 3 * n, *u2 = buf + 4 * n, *ml = buf + 5 * n,
         *x = buf + 6 * n;
  for (int j = jb->j0; j < jb->j1; j++) {
    const double lam = jb->shift[j];
    const int cstart = jb->cst[j];
    /* LU with partial pivoting of T - lam I */
    for (int i = 0; i < n; i++) {
      dg[i] = d[i] - lam;
      du[i] = (i < n - 1) ? e[i] : 0.0;
    }
    for (int i = 0; i < n - 1; i++) {
      const double sub = e[i];
      if (fabs(dg[i]) >= fabs(sub)) {
        const double l = (dg[i] != 0.0) ? sub / dg[i] : 0.0;
        u0[i] = dg[i];
        u1[i] = du[i];
        u2[i] = 0.0;
        dg[i + 1] = dg[i + 1] - l * du[i];
        ml[i] = l;
        swp[i] = 0;
      } else {
        const double l = dg[i] / sub;
        const double old_dg1 = dg[i + 1];
        u0[i] = sub;
        u1[i] = old_dg1;
        u2[i] = (i < n - 2) ? du[i + 1] : 0.0;
        dg[i + 1] = du[i] - l * old_dg1;
        if (i < n - 2) du[i + 1] = -l * du[i + 1];
        ml[i] = l;
        swp[i] = 1;
      }
    }
    u0[n - 1] = dg[n - 1];
    for (int i = 0; i < n; i++)
      if (fabs(u0[i]) < tiny) u0[i] = (u0[i] < 0.0) ? -tiny : tiny;
    /* reproducible start vector */
    for (int i = 0; i < n; i++)
      x[i] = (double)(mix64(((uint64_t)j << 32) + (uint64_t)i) >> 11) * (1.0 / 9007199254740992.0) - 0.5;
    for (int it = 0; it < INVIT_ITERS; it++) {
      /* forward: P L */
      for (int i = 0; i < n - 1; i++) {
        if (swp[i]) {
          const double t = x[i];
          x[i] = x[i + 1];
          x[i + 1] = t;
        }
        x[i + 1] -= ml[i] * x[i];
      }
      /* back: U */
      x[n - 1] /= u0[n - 1];
      x[n - 2] = (x[n - 2] - u1[n - 2] * x[n - 1]) / u0[n - 2];
      for (int i = n - 3; i >= 0; i--) x[i] = (x[i] - u1[i] * x[i + 1] - u2[i] * x[i + 2]) / u0[i];
      /* orthogonalise against the earlier vectors of the cluster (twice) */
      for (int pass = 0; pass < 2 && cstart < j; pass++) {
        for (int q = cstart; q < j; q++) {
          const double *zq = Z + (size_t)q * ldz;
          double dot = 0.0;
          for (int i = 0; i < n; i++) dot += zq[i] * x[i];
          for (int i = 0; i < n; i++) x[i] -= dot * zq[i];
        }
      }
      double nrm = 0.0, amax = 0.0;
      for (int i = 0; i < n; i++) amax = evsl_max(amax, fabs(x[i]));
      if (amax == 0.0) {
        x[j % n] = 1.0;
        amax = 1.0;
      }
      for (int i = 0; i < n; i++) {
        x[i] /= amax;
        nrm += x[i] * x[i];
      }
      nrm = sqrt(nrm);
      for (int i = 0; i < n; i++) x[i] /= nrm;
    }
    /* sign convention: largest component positive */
    int imax = 0;
    for (int i = 1; i < n; i++)
      if (fabs(x[i]) > fabs(x[imax])) imax = i;
    const double sgn = (x[imax] < 0.0) ? -1.0 : 1.0;
    double *zj = Z + (size_t)j * ldz;
    for (int i = 0; i < n; i++) zj[i] = sgn * x[i];
  }
  free(buf);
  free(swp);
  return 0;
}

static void *invit_thread(void *arg) {
  invit_job *jb = (invit_job *)arg;
  jb->rc = invit_range(jb);
  return NULL;
}

#define INVIT_MAX_THREADS 16
#define INVIT_MIN_WORK (1L << 21) /* vectors x rows per thread */

int evsl_trid_eigvecs(int n, const double *d, const double *e, int m, const double *w, double *Z, int ldz) {
  if (m <= 0 || n <= 0) return 0;
  if (n == 1) {
    for (int j = 0; j < m; j++) Z[(size_t)j * ldz] = 1.0;
    return 0;
  }
  double tnorm = 0.0;
  for (int i = 0; i < n; i++) {
    double r = fabs(d[i]);
    if (i > 0) r += fabs(e[i - 1]);
    if (i < n - 1) r += fabs(e[i]);
    tnorm = evsl_max(tnorm, r);
  }
  if (tnorm == 0.0) tnorm = 1.0;
  const double pert = 10.0 * DBL_EPSILON * tnorm;
  const double clus = CLUSTER_TOL * tnorm;
  /* shifts (separated by at least pert) and cluster starts, in order */
  double *shift = (double *)malloc(sizeof(double) * (size_t)m);
  int *cst = (int *)malloc(sizeof(int) * (size_t)m);
  if (!shift || !cst) {
    free(shift);
    free(cst);
    return evsl_seterr(EVSLX_ERR_NOMEM, "inverse iteration: out of memory");
  }
  int cstart = 0;
  double lam_prev = 0.0;
  for (int j = 0; j < m; j++) {
    double lam = w[j];
    if (j > 0) {
      if (w[j] - w[j - 1] > clus) cstart = j;
      if (lam - lam_prev < pert) lam = lam_prev + pert;
    }
    lam_prev = lam;
    shift[j] = lam;
    cst[j] = cstart;
  }
  /* ranges split at cluster starts over host threads; every vector is
   * computed the same way whatever the split */
  long nth = sysconf(_SC_NPROCESSORS_ONLN);
  nth = evsl_min(evsl_min(nth, (long)INVIT_MAX_THREADS), ((long)m * n) / INVIT_MIN_WORK);
  invit_job jobs[INVIT_MAX_THREADS];
  pthread_t tid[INVIT_MAX_THREADS];
  int nj = 0, j0 = 0;
  for (int t = 0; t < (nth > 1 ? nth : 1) && j0 < m; t++) {
    int j1 = (t == nth - 1 || nth <= 1) ? m : (int)(((long)m * (t + 1)) / nth);
    if (j1 < j0 + 1) j1 = j0 + 1;
    while (j1 < m && cst[j1] != j1) j1++;
    jobs[nj] = (invit_job){n, ldz, j0, j1, 0, d, e, shift, cst, Z, DBL_EPSILON * tnorm};
    nj++;
    j0 = j1;
  }
  int started = 0;
  for (int t = 1; t < nj; t++) {
    if (pthread_create(&tid[t], NULL, invit_thread, &jobs[t]) != 0) break;
    started = t;
  }
  jobs[0].rc = invit_range(&jobs[0]);
  for (int t = 1; t <= started; t++) pthread_join(tid[t], NULL);
  for (int t = started + 1; t < nj; t++) jobs[t].rc = invit_range(&jobs[t]); /* threads that did not start */
  int rc = 0;
  for (int t = 0; t < nj; t++)
    if (jobs[t].rc) rc = jobs[t].rc;
  free(shift);
  free(cst);
  if (rc) return evsl_seterr(EVSLX_ERR_NOMEM, "inverse iteration: out of memory");
  return 0;
}

/* Dense symmetric eigensolver.  A (n x n, column-major, lda) is read from
 * its full storage (assumed symmetric); eigenvalues ascending in w, vectors
 * in the columns of Q (ldq). */
int evsl_sym_eig(int n, const double *A, int lda, double *Q, int ldq, double *w) {
  if (n <= 0) return 0;
  double *a = (double *)malloc(sizeof(double) * (size_t)n * n);
  double *e = (double *)malloc(sizeof(double) * (size_t)n);
  double *v = (double *)malloc(sizeof(double) * (size_t)n);
  double *p = (double *)malloc(sizeof(double) * (size_t)n);
  double *V = (double *)calloc((size_t)n * n, sizeof(double)); /* Householder vectors */
  if (!a || !e || !v || !p || !V) {
    free(a);
    free(e);
    free(v);
    free(p);
    free(V);
    return evsl_seterr(EVSLX_ERR_NOMEM, "dense eigensolver: out of memory");
  }
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) a[(size_t)j * n + i] = A[(size_t)j * lda + i];
  /* Householder reduction: column k, rows k+1..n-1 */
  for (int k = 0; k < n - 2; k++) {
    const int len = n - k - 1;
    double *x = a + (size_t)k * n + k + 1;
    double sig = 0.0;
    for (int i = 0; i < len; i++) sig += x[i] * x[i];
    double *vk = V + (size_t)k * n + k + 1;
    if (sig == 0.0) {
      e[k] = 0.0;
      continue;
    }
    const double nx = sqrt(sig);
    const double alpha = (x[0] > 0.0) ? -nx : nx;
    for (int i = 0; i < len; i++) vk[i] = x[i];
    vk[0] -= alpha;
    double vn = 0.0;
    for (int i = 0; i < len; i++) vn += vk[i] * vk[i];
    vn = sqrt(vn);
    if (vn == 0.0) {
      e[k] = x[0];
      continue;
    }
    for (int i = 0; i < len; i++) vk[i] /= vn;
    /* p = 2 A22 v; q = p - (v.p) v; A22 -= v q^T + q v^T */
    double *A22 = a + (size_t)(k + 1) * n + (k + 1);
    for (int i = 0; i < len; i++) {
      double s = 0.0;
      for (int j = 0; j < len; j++) s += A22[(size_t)j * n + i] * vk[j];
      p[i] = 2.0 * s;
    }
    double K = 0.0;
    for (int i = 0; i < len; i++) K += vk[i] * p[i];
    for (int i = 0; i < len; i++) p[i] -= K * vk[i];
    for (int j = 0; j < len; j++)
      for (int i = 0; i < len; i++) A22[(size_t)j * n + i] -= vk[i] * p[j] + p[i] * vk[j];
    e[k] = alpha;
    x[0] = alpha;
    for (int i = 1; i < len; i++) x[i] = 0.0;
  }
  for (int i = 0; i < n; i++) w[i] = a[(size_t)i * n + i];
  if (n >= 2) e[n - 2] = a[(size_t)(n - 2) * n + (n - 1)];
  /* Q = H_0 H_1 ... H_{n-3} */
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) Q[(size_t)j * ldq + i] = (i == j) ? 1.0 : 0.0;
  for (int k = n - 3; k >= 0; k--) {
    const int len = n - k - 1;
    const double *vk = V + (size_t)k * n + k + 1;
    double nv = 0.0;
    for (int i = 0; i < len; i++) nv += vk[i] * vk[i];
    if (nv == 0.0) continue;
    for (int j = k + 1; j < n; j++) {
      double *qj = Q + (size_t)j * ldq + k + 1;
      double s = 0.0;
      for (int i = 0; i < len; i++) s += vk[i] * qj[i];
      s *= 2.0;
      for (int i = 0; i < len; i++) qj[i] -= s * vk[i];
    }
  }
  /* QL on the tridiagonal with the rotations applied to Q's columns */
  int rc = ql_implicit(n, w, e, Q, ldq);
  if (!rc) sort_pairs(n, w, Q, ldq, p);
  free(a);
  free(e);
  free(v);
  free(p);
  free(V);
  if (rc) return evsl_seterr(EVSLX_ERR_NUMERIC, "dense symmetric QL did not converge");
  return 0;
}

/* Thick-restart projected matrix T (k x k, column-major, ld ldt):
 *   T[i,i] = theta_i for i < m (m = trlen), T[m,i] = T[i,m] = s_i for i < m,
 *   tridiagonal from index m on.
 * All eigenvalues go to w (ascending).  When Z is not NULL, the eigenvector
 * of every w[i] >= thresh is written to column i of Z (ld ldz).
 * Method: orthogonal Q (m x m) with Q^T D Q tridiagonal and Q^T s = |s| e_{m-1}
 * from a Lanczos run on D = diag(theta) started at s/|s| (vectors placed in
 * reverse order), so diag(Q, I)^T T diag(Q, I) is tridiagonal. */
int evsl_tr_eig(int k, int m, const double *T, int ldt, double thresh, double *w, double *Z, int ldz) {
  return evsl_tr_eig_sel(k, m, T, ldt, 0, thresh, w, Z, ldz);
}

/* As evsl_tr_eig; select = 0: vectors of w[i] >= thresh; select = 1: vectors
 * of the smallest and the largest eigenvalue only (columns 0 and k-1). */
int evsl_tr_eig_sel(int k, int m, const double *T, int ldt, int select, double thresh, double *w, double *Z,
                    int ldz) {
  if (k <= 0) return 0;
  double *d = (double *)malloc(sizeof(double) * (size_t)k);
  double *e = (double *)calloc((size_t)k, sizeof(double));
  double *Q = NULL;
  if (!d || !e) {
    free(d);
    free(e);
    return evsl_seterr(EVSLX_ERR_NOMEM, "thick-restart eigensolver: out of memory");
  }
  for (int i = 0; i < k; i++) d[i] = T[(size_t)i * ldt + i];
  for (int i = (m > 0 ? m : 0); i < k - 1; i++) e[i] = T[(size_t)i * ldt + i + 1];
  if (m > 0) {
    Q = (double *)calloc((size_t)m * m, sizeof(double));
    double *r = (double *)malloc(sizeof(double) * (size_t)m);
    if (!Q || !r) {
      free(d);
      free(e);
      free(Q);
      free(r);
      return evsl_seterr(EVSLX_ERR_NOMEM, "thick-restart eigensolver: out of memory");
    }
    double dmax = 0.0, sig = 0.0;
    for (int i = 0; i < m; i++) {
      dmax = evsl_max(dmax, fabs(T[(size_t)i * ldt + i]));
      const double si = T[(size_t)i * ldt + m];
      sig += si * si;
    }
    sig = sqrt(sig);
    const double tiny = 1e3 * DBL_EPSILON * evsl_max(dmax, 1.0);
    /* start vector */
    if (sig > 0.0) {
      for (int i = 0; i < m; i++) r[i] = T[(size_t)i * ldt + m] / sig;
    } else {
      for (int i = 0; i < m; i++) r[i] = (i == m - 1) ? 1.0 : 0.0;
    }
    double bprev = 0.0;
    for (int j = 0; j < m; j++) {
      const int t = m - 1 - j; /* placement of Lanczos vector j */
      double *q = Q + (size_t)t * m;
      memcpy(q, r, sizeof(double) * (size_t)m);
      double a = 0.0;
      for (int i = 0; i < m; i++) a += q[i] * T[(size_t)i * ldt + i] * q[i];
      d[t] = a;
      if (j == m - 1) break;
      /* r = D q - a q - bprev q_prev, then full reorthogonalisation (twice) */
      for (int i = 0; i < m; i++) r[i] = T[(size_t)i * ldt + i] * q[i] - a * q[i];
      if (j > 0) {
        const double *qp = Q + (size_t)(t + 1) * m;
        for (int i = 0; i < m; i++) r[i] -= bprev * qp[i];
      }
      for (int pass = 0; pass < 2; pass++)
        for (int jj = 0; jj <= j; jj++) {
          const double *qq = Q + (size_t)(m - 1 - jj) * m;
          double dot = 0.0;
          for (int i = 0; i < m; i++) dot += qq[i] * r[i];
          for (int i = 0; i < m; i++) r[i] -= dot * qq[i];
        }
      double b = 0.0;
      for (int i = 0; i < m; i++) b += r[i] * r[i];
      b = sqrt(b);
      if (b <= tiny) {
        /* invariant subspace found: continue with a unit vector orthogonal to
         * the previous ones; the coupling is exactly zero */
        b = 0.0;
        int found = 0;
        for (int cand = 0; cand < m && !found; cand++) {
          for (int i = 0; i < m; i++) r[i] = (i == cand) ? 1.0 : 0.0;
          for (int pass = 0; pass < 2; pass++)
            for (int jj = 0; jj <= j; jj++) {
              const double *qq = Q + (size_t)(m - 1 - jj) * m;
              double dot = 0.0;
              for (int i = 0; i < m; i++) dot += qq[i] * r[i];
              for (int i = 0; i < m; i++) r[i] -= dot * qq[i];
            }
          double nr = 0.0;
          for (int i = 0; i < m; i++) nr += r[i] * r[i];
          nr = sqrt(nr);
          if (nr > 0.5) {
            for (int i = 0; i < m; i++) r[i] /= nr;
            found = 1;
          }
        }
      } else {
        for (int i = 0; i < m; i++) r[i] /= b;
      }
      e[t - 1] = b; /* coupling between positions t-1 and t */
      bprev = b;
    }
    e[m - 1] = sig; /* Q^T s = sig e_{m-1} couples position m-1 to the head m */
    free(r);
  }
  int rc = evsl_trid_eigvals(k, d, e, w);
  if (!rc && Z) {
#define TR_WANT(i) (select ? ((i) == 0 || (i) == k - 1) : (w[(i)] >= thresh))
    int msel = 0;
    for (int i = 0; i < k; i++)
      if (TR_WANT(i)) msel++;
    if (msel > 0) {
      double *ws = (double *)malloc(sizeof(double) * (size_t)msel);
      double *Y = (double *)malloc(sizeof(double) * (size_t)k * msel);
      if (!ws || !Y) {
        rc = evsl_seterr(EVSLX_ERR_NOMEM, "thick-restart eigensolver: out of memory");
      } else {
        int j = 0;
        for (int i = 0; i < k; i++)
          if (TR_WANT(i)) ws[j++] = w[i];
        rc = evsl_trid_eigvecs(k, d, e, msel, ws, Y, k);
        j = 0;
        for (int i = 0; !rc && i < k; i++) {
          if (!TR_WANT(i)) continue;
          const double *y = Y + (size_t)j * k;
          double *z = Z + (size_t)i * ldz;
          for (int r = 0; r < m; r++) {
            double acc = 0.0;
            for (int c = 0; c < m; c++) acc += Q[(size_t)c * m + r] * y[c];
            z[r] = acc;
          }
          for (int r = m; r < k; r++) z[r] = y[r];
          j++;
        }
      }
      free(ws);
      free(Y);
    }
#undef TR_WANT
  }
  free(d);
  free(e);
  free(Q);
  return rc;
}

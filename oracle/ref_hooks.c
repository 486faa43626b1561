/*
 * Test-infrastructure hooks linked into the oracle build of the reference
 * EVSL CPU library (oracle/_ref/libevsl_ref.so).  This file is NOT part of
 * the shipped library; only tests/, the smoke check and bench.py's
 * CPU-baseline leg load the oracle.
 *
 * What it adds to the reference build:
 *   1. A replacement for rand_double_device() (reference SRC/vect.c:52-55,
 *      which wraps libc rand()).  The reference draws its KPM probe vectors
 *      (SRC/spslice.c:79,90) and its lucky-breakdown restart vectors
 *      (SRC/cheblanNr.c:231, SRC/cheblanTr.c:291,387) through that call, so the
 *      oracle can be fed exactly the vectors given to the GPU library:
 *        - vectors queued with evslref_queue_vectors() are handed out first;
 *        - after that the counter-based generator below is used.  The GPU
 *          library's rand_double_device() evaluates the same formula on the
 *          device, so restart vectors agree between the two as well.
 *   2. Thin helpers for the harness: Laplacian CSR generation through the
 *      reference's own lapgen/cooMat_to_csrMat (TESTS/COMMON/lapl.c:13,
 *      SRC/spmat.c:160), the analytic spectrum exeiglap3
 *      (TESTS/COMMON/lapl.c:79), and a slice driver that runs find_pol +
 *      ChebLanNr over slices in an OpenMP parallel-for, the pattern of the
 *      reference's TESTS/PLanR/MMPLanR_omp.c:183-241.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <time.h>
#include <omp.h>
#include "evsl.h"
#include "lapl.h"

/* ---------------------------------------------------------------------------
 * Counter-based uniform generator: value i of draw d under seed s is
 *   mix64(s * 0x9E3779B97F4A7C15 + (d << 32) + i),  mapped to [-1, 1).
 * mix64 is the SplitMix64 output function (Steele, Lea, Flood 2014).
 * ------------------------------------------------------------------------- */
static uint64_t g_seed = 0x5EEDULL;
static uint64_t g_draw = 0;

static uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

static double uniform_pm1(uint64_t seed, uint64_t draw, uint64_t i) {
  uint64_t key = seed * 0x9E3779B97F4A7C15ULL + (draw << 32) + i;
  double u = (double)(mix64(key) >> 11) * (1.0 / 9007199254740992.0);
  return 2.0 * u - 1.0;
}

static double *g_queue = NULL;
static int g_qcount = 0, g_qpos = 0, g_qn = 0;

void evslref_set_seed(uint64_t seed) {
#pragma omp critical(evslref_rng)
  {
    g_seed = seed;
    g_draw = 0;
  }
}

int evslref_queue_vectors(const double *buf, int count, int n) {
  int rc = 0;
#pragma omp critical(evslref_rng)
  {
    free(g_queue);
    g_queue = NULL;
    g_qcount = g_qpos = g_qn = 0;
    if (count > 0 && n > 0) {
      g_queue = (double *)malloc((size_t)count * (size_t)n * sizeof(double));
      if (!g_queue) {
        rc = -1;
      } else {
        memcpy(g_queue, buf, (size_t)count * (size_t)n * sizeof(double));
        g_qcount = count;
        g_qn = n;
      }
    }
  }
  return rc;
}

int evslref_queue_remaining(void) { return g_qcount - g_qpos; }

void rand_double_device(int n, double *v) {
#pragma omp critical(evslref_rng)
  {
    if (g_qpos < g_qcount && n == g_qn) {
      memcpy(v, g_queue + (size_t)g_qpos * (size_t)n, (size_t)n * sizeof(double));
      g_qpos++;
    } else {
      uint64_t d = g_draw++;
      for (int i = 0; i < n; i++) v[i] = uniform_pm1(g_seed, d, (uint64_t)i);
    }
  }
}

void randn_double_device(int n, double *v) {
  /* Box-Muller on the same stream; not used on the spectrum-slicing path. */
#pragma omp critical(evslref_rng)
  {
    uint64_t d = g_draw++;
    for (int i = 0; i < n; i++) {
      double u1 = 0.5 * (uniform_pm1(g_seed, d, 2 * (uint64_t)i) + 1.0);
      double u2 = 0.5 * (uniform_pm1(g_seed, d, 2 * (uint64_t)i + 1) + 1.0);
      if (u1 < 1e-300) u1 = 1e-300;
      v[i] = sqrt(-2.0 * log(u1)) * cos(2.0 * EVSL_PI * u2);
    }
  }
}

/* ---------------------------------------------------------------------------
 * Harness helpers
 * ------------------------------------------------------------------------- */
static csrMat g_A;
static int g_A_set = 0;

/* Generate the nx*ny*nz Laplacian with the reference's generator and CSR
 * conversion (rows sorted).  Arrays are malloc'd; free with evslref_free. */
int evslref_lap_csr(int nx, int ny, int nz, int *n_out, int **ia, int **ja, double **a) {
  cooMat coo;
  csrMat csr;
  if (lapgen(nx, ny, nz, &coo)) return -1;
  if (cooMat_to_csrMat(0, &coo, &csr)) return -1;
  free_coo(&coo);
  *n_out = csr.nrows;
  *ia = csr.ia;
  *ja = csr.ja;
  *a = csr.a;
  return 0;
}

void evslref_free(void *p) { free(p); }

/* Analytic Laplacian eigenvalues in [a, b] (sorted). Returns the count; at
 * most cap values are written to out. */
int evslref_exeig(int nx, int ny, int nz, double a, double b, double *out, int cap) {
  int m = 0;
  double *v = NULL;
  exeiglap3(nx, ny, nz, a, b, &m, &v);
  for (int i = 0; i < m && i < cap; i++) out[i] = v[i];
  free(v);
  return m;
}

/* Register a host CSR matrix (arrays borrowed, not copied) as A. */
int evslref_set_csr(int n, int *ia, int *ja, double *a) {
  g_A.owndata = 0;
  g_A.nrows = n;
  g_A.ncols = n;
  g_A.nnz = ia[n];
  g_A.ia = ia;
  g_A.ja = ja;
  g_A.a = a;
  g_A_set = 1;
  return SetAMatrix(&g_A);
}

/* Plain CSR matvec through the reference (matvec_csr, SRC/spmat.c:309). */
void evslref_matvec(double *x, double *y) { matvec_csr(x, y, (void *)&g_A); }

/* Reference ChebAv (SRC/chebpoly.c:519) on the registered matrix. */
int evslref_chebav(polparams *pol, double *v, double *y) {
  int n = g_A.nrows;
  double *w = (double *)malloc(3 * (size_t)n * sizeof(double));
  int rc = ChebAv(pol, v, y, w);
  free(w);
  return rc;
}

/* Run find_pol + ChebLanNr on every slice with an OpenMP parallel-for over
 * slices (reference pattern TESTS/PLanR/MMPLanR_omp.c:183-241).  Polynomial
 * settings follow the reference drivers (TESTS/PLanN/LapPLanN.c:197-204):
 * damping, thresholds and max degree given by the caller.
 * Outputs per slice: nev[s], degree[s], seconds[s]; eigenvalues are written
 * to evals[s*evcap ...] (at most evcap per slice) and residuals likewise.
 * Returns wall seconds of the whole parallel region. */
double evslref_slices_nr(int nslices, const double *sli, double lmin, double lmax,
                         int maxit, double tol, const double *vinit, int damping,
                         double thresh_int, double thresh_ext, int max_deg,
                         int nthreads, int *nev, int *degree, double *seconds,
                         double *evals, double *resids, int evcap) {
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
  for (int s = 0; s < nslices; s++) {
    struct timespec s0, s1;
    clock_gettime(CLOCK_MONOTONIC, &s0);
    double xintv[4] = {sli[s], sli[s + 1], lmin, lmax};
    polparams pol;
    set_pol_def(&pol);
    pol.damping = damping;
    pol.thresh_int = thresh_int;
    pol.thresh_ext = thresh_ext;
    pol.max_deg = max_deg;
    find_pol(xintv, &pol);
    int nev2 = 0;
    double *lam = NULL, *Y = NULL, *res = NULL;
    ChebLanNr(xintv, maxit, tol, (double *)vinit, &pol, &nev2, &lam, &Y, &res, NULL);
    nev[s] = nev2;
    degree[s] = pol.deg;
    for (int i = 0; i < nev2 && i < evcap; i++) {
      evals[(size_t)s * evcap + i] = lam[i];
      resids[(size_t)s * evcap + i] = res[i];
    }
    free(lam);
    free(Y);
    free(res);
    free_pol(&pol);
    clock_gettime(CLOCK_MONOTONIC, &s1);
    seconds[s] = (s1.tv_sec - s0.tv_sec) + 1e-9 * (s1.tv_nsec - s0.tv_nsec);
  }
  clock_gettime(CLOCK_MONOTONIC, &t1);
  return (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
}

/* CPU baseline sampler: run `nthreads` independent reference ChebAv calls
 * (SRC/chebpoly.c:519) concurrently, one per OpenMP thread, each on its own
 * copy of v and its own workspace, with the filter truncated to `deg`
 * degrees (the per-degree cost of ChebAv is constant).  This is the
 * reference's own concurrency pattern (independent solves per thread,
 * TESTS/PLanR/MMPLanR_omp.c:183).  Returns the wall seconds of the region. */
double evslref_chebav_multi(polparams *pol, int deg, const double *v, int nthreads) {
  const int n = g_A.nrows;
  polparams p = *pol;
  if (deg > 0 && deg < p.deg) p.deg = deg;
  if (nthreads < 1) nthreads = 1;
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
#pragma omp parallel num_threads(nthreads)
  {
    double *x = (double *)malloc((size_t)n * sizeof(double));
    double *y = (double *)malloc((size_t)n * sizeof(double));
    double *w = (double *)malloc(3 * (size_t)n * sizeof(double));
    memcpy(x, v, (size_t)n * sizeof(double));
    polparams q = p;
    ChebAv(&q, x, y, w);
    free(x);
    free(y);
    free(w);
  }
  clock_gettime(CLOCK_MONOTONIC, &t1);
  return (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
}

/* Reference ChebSI (SRC/chebsi.c:39) writes its statistics to fstats without
 * a NULL check; run it with fstats on /dev/null. */
int evslref_cheb_si(int nev, double *intv, int maxit, double tol, double *vinit, polparams *pol, int *nevo,
                    double **lamo, double **Yo, double **reso) {
  FILE *f = fopen("/dev/null", "w");
  if (!f) return -1;
  int rc = ChebSI(nev, intv, maxit, tol, vinit, pol, nevo, lamo, Yo, reso, f);
  fclose(f);
  return rc;
}

/*
 * vect.c -- vector utilities, timer and statistics of the EVSL API
 * (reference SRC/vect.c, SRC/timing.c, SRC/stats.c).
 */
#define _POSIX_C_SOURCE 199309L
#include <time.h>

#include "internal.h"

/* Host uniform vector in [-1, 1] from libc rand(), as SRC/vect.c:14-20. */
void rand_double(int n, double *v) {
  const double t = ((double)RAND_MAX) / 2.0;
  for (int i = 0; i < n; i++) v[i] = (rand() - t) / t;
}

/* Host normal vector from libc rand() by Box-Muller; as SRC/vect.c:29-49,
 * every element takes the cosine branch and consumes two rand() values. */
void randn_double(int n, double *v) {
  const double two_pi = 2.0 * 3.1415926535;
  for (int i = 0; i < n; i++) {
    const double U1 = rand() * (1.0 / RAND_MAX);
    const double U2 = rand() * (1.0 / RAND_MAX);
    v[i] = sqrt(-2.0 * log(U1)) * cos(two_pi * U2);
  }
}

/* Device vectors from the library's counter-based generator (the reference
 * CUDA build draws on the host with rand() and copies, SRC/evsl_cuda.cu:97). */
void rand_double_device(int n, double *v) {
  if (evsl_require_started()) return;
  if (!evsl_rand_device(n, 1, v)) evslcu_sync();
}

void randn_double_device(int n, double *v) {
  if (evsl_require_started()) return;
  if (!evslcu_randn(n, evslh.seed, evslh.draw, v)) evslcu_sync();
  evslh.draw++;
}

void linspace(double a, double b, int num, double *arr) {
  const double h = (num == 1 ? 0 : (b - a) / (num - 1));
  arr[0] = a;
  arr[num - 1] = b;
  for (int i = 1; i < num - 1; i++) arr[i] = a + i * h;
}

static int cmp_d(const void *a, const void *b) {
  const double x = *(const double *)a, y = *(const double *)b;
  return (x < y) ? -1 : (x == y ? 0 : 1);
}

typedef struct {
  int i;
  double d;
} dint;

static int cmp_di(const void *a, const void *b) {
  const double x = ((const dint *)a)->d, y = ((const dint *)b)->d;
  return (x < y) ? -1 : (x == y ? 0 : 1);
}

void sort_double(int n, double *v, int *ind) {
  if (!ind) {
    qsort(v, (size_t)n, sizeof(double), cmp_d);
    return;
  }
  dint *vv = (dint *)malloc(sizeof(dint) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) {
    vv[i].d = v[i];
    vv[i].i = i;
  }
  qsort(vv, (size_t)n, sizeof(dint), cmp_di);
  for (int i = 0; i < n; i++) {
    v[i] = vv[i].d;
    ind[i] = vv[i].i;
  }
  free(vv);
}

/* Wall clock in seconds.  Like the reference CUDA build (SRC/timing.c:60-74)
 * it first waits for the library's queued GPU work, so a difference of two
 * readings covers the device time of the calls between them. */
double evsl_timer(void) {
  struct timespec t;
  if (evslcu_initialized()) evslcu_sync();
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

void StatsReset(void) { memset(&evslstat, 0, sizeof(evslStat)); }

void StatsPrint(FILE *fstats) {
  const evslStat *s = &evslstat;
  fprintf(fstats, " Timing (sec):\n");
  if (s->t_iter) fprintf(fstats, "   Iteration time (tot)     :  %f\n", s->t_iter);
  fprintf(fstats, "   - - - - - - - - - - - - - - - - -\n");
  if (s->n_polAv)
    fprintf(fstats, "   Pol(A)*v                 :  %f (%8zu, avg %f)\n", s->t_polAv, s->n_polAv,
            s->t_polAv / (double)s->n_polAv);
  if (s->n_mvA)
    fprintf(fstats, "   Matvec matrix A          :  %f (%8zu, avg %f)\n", s->t_mvA, s->n_mvA,
            s->t_mvA / (double)s->n_mvA);
  if (s->t_reorth) fprintf(fstats, "   Reorthogonalization      :  %f\n", s->t_reorth);
  if (s->t_eig) fprintf(fstats, "   Tridiagonal/dense eig    :  %f\n", s->t_eig);
  if (s->t_ritz) fprintf(fstats, "   Compute Ritz vectors     :  %f\n", s->t_ritz);
  fflush(fstats);
}

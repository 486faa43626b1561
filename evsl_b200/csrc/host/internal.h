/*
 * internal.h -- declarations shared by the C host sources of libevsl_b200.
 * Not installed; the public API is include/evsl.h and include/evslx.h.
 */
#ifndef EVSL_B200_INTERNAL_H
#define EVSL_B200_INTERNAL_H

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/evsl.h"
#include "../../../include/evslx.h"
#include "../evslcu.h"

/* Algorithm constants of the reference (INC/internal_header.h:21-24). */
#define EVSL_ORTH_TOL 1e-14
#define EVSL_NGS_MAX 2

/* Host-side library state (the device side lives in cuda/context.cu). */
typedef struct {
  int started;
  evslcu_op op;              /* operator used by the filter */
  evslcu_mat *mat;           /* prepared matrix behind op (owned) */
  const void *mat_key;       /* csrMat registered with SetAMatrix* */
  uint64_t seed;             /* device RNG seed */
  uint64_t draw;             /* next draw index of the device RNG */
  int kernel;                /* filter kernel choice, -1 = library default */
  int persistent;            /* 1: one cooperative launch per filter application */
  int l2_resident;           /* 1: keep the stored matrix persisting in L2 */
  int wave;                  /* 1: pipelined single-launch filter */
  double last_kpm_seconds;   /* device time of the last kpmdos moment loop */
  int last_kdim;             /* Lanczos dimension of the last ChebLanNr/ChebLanTr */
  int last_candidates;       /* Ritz values >= bar examined at the end */
  double last_filter_seconds;
  int sync_tests;            /* 1: ChebLanNr waits for each convergence test */
} evsl_host_state;

extern evsl_host_state evslh;

/* error reporting */
int evsl_seterr(int code, const char *fmt, ...);
int evsl_require_started(void);
int evsl_require_operator(void);

/* interval check (INC/internal_header.h:194-217) */
int evsl_check_intv(const double *intv, FILE *fstats);

/* tridiagonal / dense symmetric eigensolvers (host, FP64; tridiag.c) */
int evsl_trid_eig_first(int n, const double *d, const double *e, double *w, double *z1);
int evsl_trid_eigvals(int n, const double *d, const double *e, double *w);
int evsl_trid_eigvals_test(int n, const double *d, const double *e, double xmin, double *w);
/* the same test on a side stream: 1 when started, 0 when the size is below
 * the GPU threshold (the caller runs it directly), a negative error code */
int evsl_trid_test_start(int n, const double *d, const double *e, double xmin);
int evsl_trid_test_ready(void);
int evsl_trid_test_wait(double *w);
int evsl_trid_eigvecs(int n, const double *d, const double *e, int m, const double *w, double *Z, int ldz);
int evsl_sym_eig(int n, const double *A, int lda, double *Q, int ldq, double *w);
int evsl_tr_eig(int k, int m, const double *T, int ldt, double thresh, double *w, double *Z, int ldz);
int evsl_tr_eig_sel(int k, int m, const double *T, int ldt, int select, double thresh, double *w, double *Z,
                    int ldz);
/* y = A x on device vectors with the registered operator (asynchronous for a
 * registered matrix; a user matvec runs after the stream has drained). */
int evsl_apply_A(const double *x, double *y);

/* device random vectors drawn from the library stream */
int evsl_rand_device(int n, int count, double *v);

/* the global operator of the filter, checked */
const evslcu_op *evsl_op(void);

#endif

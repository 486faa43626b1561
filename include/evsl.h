/*
 * evsl.h -- public C API of the B200 spectrum-slicing library (libevsl_b200.so).
 *
 * This header declares the EVSL entry points of the polynomial-filtered
 * spectrum-slicing path with the same names, signatures, argument meaning,
 * ownership rules and struct layouts as the reference's CUDA build, so that
 * programs written against the reference link against this library unchanged.
 * Each declaration cites the reference interface it replaces (paths relative
 * to the EVSL_1.1.1 project directory).
 *
 * Memory conventions (as in the reference CUDA build, INC/evsl.h:137-272):
 *   - vinit passed to ChebLanNr/ChebLanTr is DEVICE memory;
 *   - the eigenvector block returned in *Wo / *W is DEVICE memory (n x nev,
 *     column-major), freed by the caller with evsl_Free_device;
 *   - eigenvalues and residuals are HOST memory, freed with evsl_Free;
 *   - polparams.mu is allocated by find_pol and freed by free_pol.
 * Everything numerical runs on the GPU; there is no CPU code path.
 */
#ifndef EVSL_B200_EVSL_H
#define EVSL_B200_EVSL_H

#include <stdio.h>
#include <stddef.h>
#include <stdint.h>

#define EVSL_PI 3.14159265358979323846
/* Slack used when comparing doubles: a >= b is tested as a + 10*DBL_EPSILON >= b
 * (INC/evsl.h:22-27). */
#define EVSL_DBL_EPS_MULT 10

#define evsl_max(a, b) ((a) > (b) ? (a) : (b))
#define evsl_min(a, b) ((a) < (b) ? (a) : (b))

/* ---------------------------------------------------------------------------
 * Types.  Layouts are identical to INC/struct.h of the reference CUDA build.
 * ------------------------------------------------------------------------- */

/* COO matrix, 0-based (INC/struct.h:14-21). */
typedef struct _cooMat {
  int nrows, ncols, nnz, *ir, *jc;
  double *vv;
} cooMat;

/* CSR matrix, 0-based, 3-array form (INC/struct.h:29-42).  In the reference
 * CUDA build the struct ends with a cuSPARSE descriptor and a work buffer;
 * both slots are kept (as opaque pointers) so the layout matches.  This
 * library stores its own prepared copy of the matrix behind `descr`. */
typedef struct _csrMat {
  int owndata, nrows, ncols, nnz, *ia, *ja;
  double *a;
  void *descr;
  char *dBuffer;
} csrMat;

/* Polynomial filter parameters (INC/struct.h:68-98).  Inputs: max_deg,
 * min_deg, damping (0 none, 1 Jackson, 2 Lanczos sigma), thresh_ext,
 * thresh_int, intvtol, deg (0 = choose).  Outputs of find_pol: type (0 middle,
 * 1 left, 2 right interval), mu[0..deg], cc, dd, gam, bar, deg. */
typedef struct _polparams {
  int max_deg;
  int min_deg;
  int damping;
  double thresh_ext;
  double thresh_int;
  double intvtol;
  int type;
  double *mu;
  double cc;
  double dd;
  double gam;
  double bar;
  int deg;
} polparams;

/* y = A x on device vectors (INC/struct.h:118). */
typedef void (*MVFunc)(double *x, double *y, void *data);
typedef void (*SolFuncR)(double *b, double *x, void *data);

typedef struct _EVSLMatvec {
  MVFunc func;
  void *data;
} EVSLMatvec;

typedef struct _EVSLBSol {
  SolFuncR func;
  void *data;
} EVSLBSol;

typedef struct _EVSLLTSol {
  SolFuncR func;
  void *data;
} EVSLLTSol;

/* Global state (INC/struct.h:186-200).  The three handle slots of the
 * reference CUDA build (cuBLAS, cuSPARSE, cuRAND) are kept as opaque pointers
 * for layout compatibility; this library does not use those libraries. */
typedef struct _evsldata {
  int n;
  int ifGenEv;
  EVSLMatvec *Amv;
  EVSLMatvec *Bmv;
  EVSLBSol *Bsol;
  EVSLLTSol *LTsol;
  double *ds;
  void *cublasH;
  void *cusparseH;
  void *curandGen;
} evslData;

extern evslData evsldata;

/* Timing statistics (INC/struct.h:223-253).  Filled from CUDA events, so
 * reading them never forces a device-wide synchronisation. */
typedef struct _evslstat {
  double t_setBsv, t_setASigBsv, t_iter;
  double t_polAv, t_reorth, t_siorth, t_ritz, t_eig;
  double t_mvA, t_mvB, t_svB, t_svLT, t_svASigB, t_blas, t_ratAv;
  size_t n_mvA, n_mvB, n_svB, n_svLT, n_svASigB, n_polAv, n_ratAv;
  size_t alloced, alloced_total, alloced_max;
} evslStat;

extern evslStat evslstat;

/* ---------------------------------------------------------------------------
 * Memory helpers (INC/evsl.h:41-131, SRC/evsl_memory.c).
 * ------------------------------------------------------------------------- */
#define evsl_Malloc(count, type) ((type *)_evsl_Malloc((size_t)(sizeof(type) * (count))))
#define evsl_Calloc(count, type) ((type *)_evsl_Calloc((size_t)(count), (size_t)sizeof(type)))
#define evsl_Realloc(ptr, count, type) \
  ((type *)_evsl_Realloc((void *)ptr, (size_t)(sizeof(type) * (count))))
#define evsl_Free(ptr) (_evsl_Free((void *)ptr), ptr = NULL)
#define evsl_Malloc_device(count, type) \
  ((type *)_evsl_Malloc_device((size_t)(sizeof(type) * (count))))
#define evsl_Calloc_device(count, type) \
  ((type *)_evsl_Calloc_device((size_t)(count), (size_t)sizeof(type)))
#define evsl_Realloc_device(ptr, old_count, old_type, new_count, new_type)             \
  ((new_type *)_evsl_Realloc_device((void *)ptr, (size_t)(sizeof(old_type) * (old_count)), \
                                    (size_t)(sizeof(new_type) * (new_count))))
#define evsl_Free_device(ptr) (_evsl_Free_device((void *)ptr), ptr = NULL)

#ifdef __cplusplus
extern "C" {
#endif

/* SRC/evsl_memory.c:9-151 */
void *_evsl_Malloc(size_t nbytes);
void *_evsl_Calloc(size_t count, size_t nbytes);
void *_evsl_Realloc(void *ptr, size_t nbytes);
void _evsl_Free(void *ptr);
void *_evsl_Malloc_device(size_t nbytes);
void *_evsl_Calloc_device(size_t count, size_t nbytes);
void *_evsl_Realloc_device(void *old_ptr, size_t old_nbytes, size_t new_nbytes);
void _evsl_Free_device(void *ptr);
void evsl_memcpy_device_to_host(void *dst, void *src, size_t nbytes);
void evsl_memcpy_device_to_device(void *dst, void *src, size_t nbytes);
void evsl_memcpy_host_to_device(void *dst, void *src, size_t nbytes);
void evsl_memset_device(void *ptr, int value, size_t nbytes);

/* ---------------------------------------------------------------------------
 * Setup (SRC/evsl.c).
 * ------------------------------------------------------------------------- */
int EVSLStart(void);                      /* SRC/evsl.c:24 */
int EVSLFinish(void);                     /* SRC/evsl.c:60 */
int SetAMatrix(csrMat *A);                /* SRC/evsl.c:95  (host CSR; uploaded once) */
int SetAMatvec(int n, MVFunc func, void *data); /* SRC/evsl.c:132 (device x, y) */
int SetAMatrix_device_csr(csrMat *A);     /* SRC/evsl.c:256 (device CSR, borrowed) */
int SetStdEig(void);                      /* SRC/evsl.c:185 */
int SetGenEig(void);                      /* SRC/evsl.c:195: generalized problem not on this path; returns -1 */
void evsl_device_query(int dev);          /* SRC/evsl_cuda.cu:14 */
void evsl_last_device_err(void);          /* SRC/evsl.c:317 */

/* SRC/spmat.c */
int cooMat_to_csrMat(int cooidx, cooMat *coo, csrMat *csr); /* :160 */
void free_csr(csrMat *csr);                                   /* :107 */
void free_coo(cooMat *coo);                                   /* :148 */
void csr_copy(csrMat *A, csrMat *B, int allocB);              /* :126 */
int arrays_copyto_csrMat(int nrow, int ncol, int *ia, int *ja, double *a, csrMat *A); /* :206 */
void evsl_create_csr_gpu(csrMat *Acpu, csrMat *Agpu);         /* :626 */
void evsl_free_csr_gpu(csrMat *csr);                          /* :655 */

/* ---------------------------------------------------------------------------
 * Polynomial filter (SRC/chebpoly.c).
 * ------------------------------------------------------------------------- */
void set_pol_def(polparams *pol);              /* :15 */
int find_pol(double *intv, polparams *pol);    /* :363 */
void free_pol(polparams *pol);                 /* :497 */
int ChebAv(polparams *pol, double *v, double *y, double *w); /* :519 (device v, y, w[3n]) */
int dampcf(int m, int damping, double *jac);   /* :39 */
/* Fused Chebyshev update (SRC/evsl_cuda.cu:175-191), device vectors. */
void evsl_chebAv_device(int n, int k, double t, double s, double cc, double *vkp1,
                        double *vk, double *vkm1, double *y);

/* ---------------------------------------------------------------------------
 * Filtered Lanczos (SRC/cheblanNr.c:57, SRC/cheblanTr.c:59).
 * ------------------------------------------------------------------------- */
int ChebLanNr(double *intv, int maxit, double tol, double *vinit, polparams *pol,
              int *nevOut, double **lamo, double **Wo, double **reso, FILE *fstats);
int ChebLanTr(int lanm, int nev, double *intv, int maxit, double tol, double *vinit,
              polparams *pol, int *nev2, double **vals, double **W, double **resW,
              FILE *fstats);

/* ---------------------------------------------------------------------------
 * Polynomial-filtered subspace iteration (SRC/chebsi.c:39); vinit is a device
 * block n x nev, *Yo device, *lamo and *reso host.
 * ------------------------------------------------------------------------- */
int ChebSI(int nev, double *intv, int maxit, double tol, double *vinit, polparams *pol, int *nevo,
           double **lamo, double **Yo, double **reso, FILE *fstats);

/* ---------------------------------------------------------------------------
 * Spectrum bounds by Lanczos (SRC/lanbounds.c:21, SRC/lanTrbounds.c:35);
 * v / vinit are device vectors.
 * ------------------------------------------------------------------------- */
int LanBounds(int msteps, double *v, double *lmin, double *lmax);
int LanTrbounds(int lanm, int maxit, double tol, double *vinit, int bndtype, double *lammin, double *lammax,
                FILE *fstats);

/* ---------------------------------------------------------------------------
 * Density of states and slicing (SRC/spslice.c:29, :205).
 * ------------------------------------------------------------------------- */
int kpmdos(int Mdeg, int damping, int nvec, double *intv, double *mu, double *ecnt);
int spslicer(double *sli, double *mu, int Mdeg, double *intv, int n_int, int npts);

/* Lanczos DOS (SRC/landos.c:37) and its slicer (SRC/spslice2.c:25); xdos,
 * ydos host arrays of npts.  exDOS (SRC/exDOS.c:17): DOS of known
 * eigenvalues on the same kind of grid.  simpson (SRC/simpson.c:25, declared
 * in the reference's INC/internal_header.h:75): cumulative Simpson integral
 * in place. */
int LanDos(const int nvec, int msteps, const int npts, double *xdos, double *ydos, double *neig,
           const double *const intv);
void spslicer2(double *xi, double *yi, int n_int, int npts, double *sli);
int exDOS(double *vals, int n, int npts, double *x, double *y, double *intv);
void simpson(double *xi, double *yi, int npts);

/* ---------------------------------------------------------------------------
 * Vector helpers (SRC/vect.c, SRC/timing.c, SRC/stats.c).
 * ------------------------------------------------------------------------- */
void rand_double(int n, double *v);            /* vect.c:14  host vector, uniform [-1,1) */
void randn_double(int n, double *v);           /* vect.c:29  host vector, N(0,1) */
void rand_double_device(int n, double *v);     /* evsl_cuda.cu:97  device vector */
void randn_double_device(int n, double *v);    /* evsl_cuda.cu:134 device vector */
void sort_double(int n, double *v, int *ind);  /* vect.c:140 */
void linspace(double a, double b, int num, double *arr); /* vect.c:82 */
double evsl_timer(void);                       /* timing.c:60 */
void StatsPrint(FILE *fstats);                 /* stats.c:16 */
void StatsReset(void);                         /* stats.c:87 */

/* Device BLAS shims (SRC/vect.c:212-284), device vectors, column-major. */
double evsl_dnrm2_device(int *n, double *x, int *incr);
void evsl_dscal_device(int *n, double *a, double *x, int *incr);
double evsl_ddot_device(int *n, double *x, int *incx, double *y, int *incy);
void evsl_daxpy_device(int *n, double *a, double *x, int *incx, double *y, int *incy);
void evsl_dcopy_device(int *n, double *x, int *incx, double *y, int *incy);
void evsl_dgemv_device(const char *trans, int *m, int *n, double *alpha, double *a, int *lda,
                       double *x, int *incx, double *beta, double *y, int *incy);
void evsl_dgemm_device(const char *transa, const char *transb, int *m, int *n, int *k,
                       double *alpha, double *a, int *lda, double *b, int *ldb, double *beta,
                       double *c, int *ldc);

#ifdef __cplusplus
}
#endif

#endif /* EVSL_B200_EVSL_H */

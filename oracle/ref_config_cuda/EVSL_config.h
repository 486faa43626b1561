/*
 * Configuration header for building the reference EVSL library with its CUDA
 * path (cuSPARSE SpMV, cuBLAS BLAS-1/2/3, device-resident vectors), as the
 * reference's `configure --with-cuda` would (EVSL_1.1.1/CONFIG/configure.in:
 * 614-652 defines EVSL_USING_CUDA_GPU and EVSL_USING_DEVICE_MEMORY; types as
 * in :768-776).  Used only by the oracle recipe's `cuda` target, which builds
 * the reference's own GPU implementation as a timed baseline.
 *
 * Test infrastructure only: nothing in the shipped library includes this.
 */
#ifndef EVSL_ORACLE_CONFIG_H
#define EVSL_ORACLE_CONFIG_H

#define EVSL_ARCH_LINUX 1
#define EVSL_USING_EVSL_BLAS 1
#define EVSL_USING_EVSL_LAPACK 1
#define EVSL_USING_OPENMP 1
#define EVSL_USING_CUDA_GPU 1
#define EVSL_USING_DEVICE_MEMORY 1

#define EVSL_Int int
#define EVSL_Unsigned unsigned
#define EVSL_LongInt long int
#define EVSL_Real double
#define EVSL_Complex double _Complex

/* Fortran name mangling (only the f90 wrappers use it; they are not built). */
#define FC_FUNC(name, NAME) name##_
#define FC_FUNC_(name, NAME) name##_
#define EVSLFORT(name, NAME) FC_FUNC_(name##_f90, NAME##_f90)

#endif

/*
 * Configuration header for building the reference EVSL CPU library as a test
 * oracle.  The reference normally generates this file with autoconf
 * (EVSL_1.1.1/CONFIG/configure.in), which needs a Fortran compiler that this
 * image lacks; the oracle recipe (oracle/Makefile) uses this hand-written
 * header instead.  The type choices follow CONFIG/configure.in:768-776:
 * 32-bit int indices, double values, vendored f2c BLAS/LAPACK, OpenMP on.
 *
 * Test infrastructure only: nothing in the shipped library includes this.
 */
#ifndef EVSL_ORACLE_CONFIG_H
#define EVSL_ORACLE_CONFIG_H

#define EVSL_ARCH_LINUX 1
#define EVSL_USING_EVSL_BLAS 1
#define EVSL_USING_EVSL_LAPACK 1
#define EVSL_USING_OPENMP 1

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

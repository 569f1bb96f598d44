/* Prototype-only LAPACKE header for the CPU test oracle (see cblas.h). */
#pragma once
#include "lapack.h"
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
extern "C" {
lapack_int LAPACKE_dsygvx(int, lapack_int, char, char, char, lapack_int, double*, lapack_int, double*, lapack_int,
                          double, double, lapack_int, lapack_int, double, lapack_int*, double*, double*, lapack_int, lapack_int*);
lapack_int LAPACKE_dsygvd(int, lapack_int, char, char, lapack_int, double*, lapack_int, double*, lapack_int, double*);
lapack_int LAPACKE_zhegvd(int, lapack_int, char, char, lapack_int, lapack_complex_double*, lapack_int,
                          lapack_complex_double*, lapack_int, double*);
lapack_int LAPACKE_zheevd(int, char, char, lapack_int, lapack_complex_double*, lapack_int, double*);
lapack_int LAPACKE_dsyevd(int, char, char, lapack_int, double*, lapack_int, double*);
lapack_int LAPACKE_dpotrf(int, char, lapack_int, double*, lapack_int);
lapack_int LAPACKE_zpotrf(int, char, lapack_int, lapack_complex_double*, lapack_int);
lapack_int LAPACKE_dtrtrs(int, char, char, char, lapack_int, lapack_int, const double*, lapack_int, double*, lapack_int);
lapack_int LAPACKE_ztrtrs(int, char, char, char, lapack_int, lapack_int, const lapack_complex_double*, lapack_int,
                          lapack_complex_double*, lapack_int);
}

/* Prototype-only LAPACK header for the CPU test oracle (see cblas.h). */
#pragma once
#include <complex>
#ifndef lapack_int
#define lapack_int int
#endif
#ifndef lapack_complex_double
#define lapack_complex_double std::complex<double>
#endif
#ifndef lapack_logical
#define lapack_logical int
#endif

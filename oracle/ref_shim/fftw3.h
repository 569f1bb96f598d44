/*
 * Stand-in for FFTW 3's <fftw3.h>, used only to compile and run the
 * reference's own FFT code paths on the CPU as a test oracle (oracle/_ref).
 * FFTW itself is not installed in this image; the reference links the system
 * FFTW 3 (any 3.x: it uses only the basic and "advanced" complex interfaces and
 * the 3-D real-data planners, all unchanged across 3.x).
 *
 * What is restated is FFTW 3's documented transform, not its implementation:
 *   Y[k] = sum_j X[j] exp(sign * 2 pi i j k / n),   sign = FFTW_FORWARD (-1) or
 *   FFTW_BACKWARD (+1), unnormalised, separable over the dimensions of a
 *   row-major array (the first dimension varies slowest);
 *   fftw_plan_many_dft: transform b of `howmany` starts at in + b * idist, and
 *   element (i0, .., i_{r-1}) sits at istride * (row-major index of the
 *   element in the `inembed` array, or in `n` when inembed is NULL);
 *   r2c keeps the n_{r-1}/2 + 1 non-redundant outputs of the last dimension,
 *   c2r is its unnormalised inverse (the input is treated as Hermitian);
 *   fftw_execute_dft applies a plan to new arrays of the same layout.
 * The transforms are direct sums per line with exactly reduced twiddle
 * indices ((j k) mod n) and twiddles evaluated in long double, so each 1-D
 * line is accurate to a few ulps times log n at the small grids the tests use.
 *
 * Test infrastructure only; nothing in the product links it.
 */
#pragma once
#include <cstddef>

typedef double fftw_complex[2];
typedef struct qsref_fftw_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

extern "C" {
void* fftw_malloc(size_t n);
void fftw_free(void* p);
void fftw_destroy_plan(fftw_plan p);
void fftw_execute(const fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out);
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_dft(int rank, const int* n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out, unsigned flags);
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed, int istride,
                             int idist, fftw_complex* out, const int* onembed, int ostride, int odist, int sign,
                             unsigned flags);
void fftw_cleanup(void);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);
}

/*
 * FP64 FFTW3-API shim -- TEST INFRASTRUCTURE ONLY (part of the oracle).
 *
 * The reference solver's CPU path calls FFTW3 (double + threads), a third-party
 * library that is not vendored with it and whose version the reference does not
 * pin (reference: src/CMakeLists.txt:51 `find_package(FFTW3 REQUIRED COMPONENTS
 * double threads)`, cmake/FindFFTW3.cmake, README.md:35).  FFTW3 is absent from
 * this image, so this header declares the 13 symbols the reference uses and
 * oracle/fftw_shim/fftw_shim.c implements them with FFTW's published semantics:
 *
 *   - unnormalised transforms; FFTW_FORWARD = -1 (exp(-2*pi*i*jk/n)),
 *     FFTW_BACKWARD = +1;
 *   - row-major n0 x n1 x n2 arrays;
 *   - r2c output is n0 x n1 x (n2/2+1); c2r consumes that half spectrum, uses
 *     only the Hermitian part (imaginary parts of the self-conjugate bins are
 *     ignored) and writes n0*n1*n2 reals;
 *   - plans bind the in/out pointers given at plan time (fftw_execute).
 *
 * Call sites in the reference: src/solver/fft_solvers/fft_context.cpp:25-26,33,
 * src/solver/fft_solvers/cpu/fftw_poisson_solver.cpp:72,83,112-118,
 * src/solver/fft_solvers/cpu/fftw_split_solver.cpp:62,74,101-107.
 *
 * Only tests/, the bench's CPU baseline and the golden-vector generator use it.
 */
#ifndef GPE_ORACLE_FFTW_SHIM_H
#define GPE_ORACLE_FFTW_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct gpe_shim_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out,
                               unsigned flags);
void fftw_execute(const fftw_plan plan);
void fftw_destroy_plan(fftw_plan plan);

void *fftw_malloc(size_t n);
void fftw_free(void *p);

/* Shim-only extras (not part of FFTW's API): strided batched 1D transform used
 * by the shim's own known-answer tests. */
void gpe_shim_fft1d(int n, const double *in, double *out, int sign);

#ifdef __cplusplus
}
#endif

#endif

/*
 * Oracle (test infrastructure only): the subset of the FFTW3 C interface that
 * the reference's serial FFT wrapper binds (janus/fft/serial/fftw.pxd:3-43),
 * implemented by fftw_shim.c in this directory.  libfftw3 is not installed in
 * this image, so the reference's Cython modules are compiled against this
 * header to act as the checker.  The flag values are FFTW's documented public
 * constants (an interface, so they are kept identical).
 *
 * Nothing in the janus_b200 product links or includes this file.
 */
#ifndef JANUS_ORACLE_FFTW3_SHIM_H
#define JANUS_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_CONSERVE_MEMORY (1U << 2)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_WISDOM_ONLY (1U << 21)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
double *fftw_alloc_real(size_t n);
fftw_complex *fftw_alloc_complex(size_t n);

void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in,
                               fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in,
                               double *out, unsigned flags);

#ifdef __cplusplus
}
#endif

#endif

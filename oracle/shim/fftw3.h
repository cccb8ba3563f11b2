/*
 * Minimal FFTW3-API subset so that the reference's src/pppm.c compiles and
 * runs in the oracle build (FFTW3 is not installed in this image).  It covers
 * exactly the calls pppm.c makes (src/pppm.c:434-462, 479-492, 567, 596-601):
 * 3D r2c/c2r plans, execute and destroy.  The arithmetic is the oracle's own
 * mixed-radix FFT (oracle/fft235.c) with FFTW's conventions: row-major, last
 * dimension halved to n/2+1, forward sign -1, nothing normalised.
 * TEST INFRASTRUCTURE ONLY.
 */
#ifndef ORACLE_FFTW3_SHIM_H
#define ORACLE_FFTW3_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif

/*
 * fft235 — double-precision mixed-radix FFT (radices 2, 3, 4, 5, 7) written
 * for the CPU oracle.  TEST INFRASTRUCTURE ONLY: the GPU product uses cuFFT.
 *
 * Conventions are FFTW's, because the reference's P3M (src/pppm.c:434-462,
 * 567, 596-601) is written against FFTW3:
 *   - forward transform uses exp(-2 pi i j k / n), backward exp(+2 pi i j k / n);
 *   - nothing is normalised (a forward+backward pair multiplies by n);
 *   - 3D real transforms are row-major [nx][ny][nz] with the last dimension
 *     halved to nz/2+1 complex values.
 * Lengths must factor completely into 2, 3, 5 and 7 (the reference only ever
 * asks for such sizes: multiple_of_2357_near, src/pppm.c:277-292).
 */
#ifndef FFT235_H
#define FFT235_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } fft235_cplx;

typedef struct fft235_plan1d fft235_plan1d;

/* sign = -1 forward, +1 backward.  Returns 0 if n has a prime factor > 7. */
fft235_plan1d *fft235_plan1d_new(int n, int sign);
void fft235_plan1d_delete(fft235_plan1d *p);
/* out[k] = sum_j in[j*stride] * exp(sign 2 pi i j k / n); out is contiguous. */
void fft235_exec1d(const fft235_plan1d *p, const fft235_cplx *in, int stride, fft235_cplx *out);

/* 3D real-to-complex forward transform, FFTW layout. */
void fft235_r2c_3d(int nx, int ny, int nz, const double *in, fft235_cplx *out);
/* 3D complex-to-real backward transform (unnormalised), FFTW layout.
   The input is treated as the non-redundant half of a Hermitian array. */
void fft235_c2r_3d(int nx, int ny, int nz, const fft235_cplx *in, double *out);

#ifdef __cplusplus
}
#endif

#endif

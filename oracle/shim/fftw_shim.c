/*
 * FFTW3-API subset over the oracle's own FFT (see shim/fftw3.h).
 * TEST INFRASTRUCTURE ONLY.
 */
#include <stdlib.h>
#include "fftw3.h"
#include "../fft235.h"

struct fftw_plan_s {
  int kind; /* 0 = r2c, 1 = c2r */
  int n0, n1, n2;
  double *real;
  fftw_complex *cplx;
};

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags)
{
  fftw_plan p = (fftw_plan) malloc(sizeof(*p));
  (void) flags;
  p->kind = 0;
  p->n0 = n0; p->n1 = n1; p->n2 = n2;
  p->real = in;
  p->cplx = out;
  return p;
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags)
{
  fftw_plan p = (fftw_plan) malloc(sizeof(*p));
  (void) flags;
  p->kind = 1;
  p->n0 = n0; p->n1 = n1; p->n2 = n2;
  p->real = out;
  p->cplx = in;
  return p;
}

void fftw_execute(const fftw_plan p)
{
  if (p->kind == 0)
    fft235_r2c_3d(p->n0, p->n1, p->n2, p->real, (fft235_cplx *) p->cplx);
  else
    fft235_c2r_3d(p->n0, p->n1, p->n2, (const fft235_cplx *) p->cplx, p->real);
}

void fftw_destroy_plan(fftw_plan p)
{
  free(p);
}

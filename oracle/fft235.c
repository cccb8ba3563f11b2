/*
 * fft235 — double-precision mixed-radix FFT for the CPU oracle.
 * TEST INFRASTRUCTURE ONLY (the GPU product calls cuFFT).
 *
 * Recursive decimation in time: a length-n transform with first radix r is r
 * transforms of length n/r over the decimated inputs, combined by an r-point
 * DFT with twiddles exp(sign 2 pi i j k / n).  Twiddles are evaluated in long
 * double and rounded once, with the quadrant points set exactly, so the
 * transform is accurate to a few ulp times log(n).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "fft235.h"

#define MAXFAC 64

struct fft235_plan1d {
  int n, sign, nf;
  int fac[MAXFAC];
  fft235_cplx *tw; /* tw[e] = exp(sign 2 pi i e / n), e in [0, n) */
};

static int factorize(int n, int *fac)
{
  int nf = 0, p;
  static const int primes[3] = {3, 5, 7};
  while (n % 4 == 0) { fac[nf++] = 4; n /= 4; }
  while (n % 2 == 0) { fac[nf++] = 2; n /= 2; }
  for (p = 0; p < 3; p++)
    while (n % primes[p] == 0) { fac[nf++] = primes[p]; n /= primes[p]; }
  return n == 1 ? nf : -1;
}

fft235_plan1d *fft235_plan1d_new(int n, int sign)
{
  fft235_plan1d *p;
  int e;
  if (n < 1)
    return 0;
  p = (fft235_plan1d *) calloc(1, sizeof(*p));
  p->n = n;
  p->sign = sign < 0 ? -1 : 1;
  p->nf = factorize(n, p->fac);
  if (p->nf < 0) {
    free(p);
    return 0;
  }
  p->tw = (fft235_cplx *) malloc(sizeof(fft235_cplx) * (size_t) n);
  for (e = 0; e < n; e++) {
    if ((4L * e) % n == 0) {
      /* quadrant point: exact */
      const int quad = (int) ((4L * e) / n);
      static const double c4[4] = {1, 0, -1, 0};
      static const double s4[4] = {0, 1, 0, -1};
      p->tw[e].re = c4[quad];
      p->tw[e].im = p->sign * s4[quad];
    } else {
      const long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double) e / (long double) n;
      p->tw[e].re = (double) cosl(a);
      p->tw[e].im = (double) (p->sign * sinl(a));
    }
  }
  return p;
}

void fft235_plan1d_delete(fft235_plan1d *p)
{
  if (p) {
    free(p->tw);
    free(p);
  }
}

static void rec(const fft235_plan1d *p, fft235_cplx *out, const fft235_cplx *in,
                long istride, int level, int nhere)
{
  const int r = p->fac[level];
  const int m = nhere / r;
  const long twstep = p->n / nhere;
  const long rstep = p->n / r;
  int j, k, q;
  fft235_cplx x[8], y[8];
  if (m == 1) {
    for (j = 0; j < r; j++)
      out[j] = in[j * istride];
  } else {
    for (j = 0; j < r; j++)
      rec(p, out + (long) j * m, in + j * istride, istride * r, level + 1, m);
  }
  for (k = 0; k < m; k++) {
    for (j = 0; j < r; j++) {
      fft235_cplx v = out[k + (long) j * m];
      if (j && k) {
        const fft235_cplx w = p->tw[((long) j * k * twstep) % p->n];
        const double re = v.re * w.re - v.im * w.im;
        const double im = v.re * w.im + v.im * w.re;
        v.re = re;
        v.im = im;
      }
      x[j] = v;
    }
    for (q = 0; q < r; q++) {
      double re = x[0].re, im = x[0].im;
      for (j = 1; j < r; j++) {
        const fft235_cplx w = p->tw[((j * q) % r) * rstep];
        re += x[j].re * w.re - x[j].im * w.im;
        im += x[j].re * w.im + x[j].im * w.re;
      }
      y[q].re = re;
      y[q].im = im;
    }
    for (q = 0; q < r; q++)
      out[k + (long) q * m] = y[q];
  }
}

void fft235_exec1d(const fft235_plan1d *p, const fft235_cplx *in, int stride, fft235_cplx *out)
{
  if (p->n == 1) {
    out[0] = in[0];
    return;
  }
  rec(p, out, in, stride, 0, p->n);
}

void fft235_r2c_3d(int nx, int ny, int nz, const double *in, fft235_cplx *out)
{
  const int nzh = nz / 2 + 1;
  const int nmax = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
  fft235_plan1d *px = fft235_plan1d_new(nx, -1);
  fft235_plan1d *py = fft235_plan1d_new(ny, -1);
  fft235_plan1d *pz = fft235_plan1d_new(nz, -1);
  fft235_cplx *a = (fft235_cplx *) malloc(sizeof(fft235_cplx) * (size_t) nmax);
  fft235_cplx *b = (fft235_cplx *) malloc(sizeof(fft235_cplx) * (size_t) nmax);
  int ix, iy, iz;
  for (ix = 0; ix < nx; ix++)
    for (iy = 0; iy < ny; iy++) {
      const double *src = in + ((long) ix * ny + iy) * nz;
      fft235_cplx *dst = out + ((long) ix * ny + iy) * nzh;
      for (iz = 0; iz < nz; iz++) {
        a[iz].re = src[iz];
        a[iz].im = 0;
      }
      fft235_exec1d(pz, a, 1, b);
      memcpy(dst, b, sizeof(fft235_cplx) * (size_t) nzh);
    }
  for (ix = 0; ix < nx; ix++)
    for (iz = 0; iz < nzh; iz++) {
      fft235_cplx *base = out + (long) ix * ny * nzh + iz;
      fft235_exec1d(py, base, nzh, b);
      for (iy = 0; iy < ny; iy++)
        base[(long) iy * nzh] = b[iy];
    }
  for (iy = 0; iy < ny; iy++)
    for (iz = 0; iz < nzh; iz++) {
      fft235_cplx *base = out + (long) iy * nzh + iz;
      fft235_exec1d(px, base, ny * nzh, b);
      for (ix = 0; ix < nx; ix++)
        base[(long) ix * ny * nzh] = b[ix];
    }
  free(a);
  free(b);
  fft235_plan1d_delete(px);
  fft235_plan1d_delete(py);
  fft235_plan1d_delete(pz);
}

void fft235_c2r_3d(int nx, int ny, int nz, const fft235_cplx *in, double *out)
{
  const int nzh = nz / 2 + 1;
  const int nmax = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
  fft235_plan1d *px = fft235_plan1d_new(nx, +1);
  fft235_plan1d *py = fft235_plan1d_new(ny, +1);
  fft235_plan1d *pz = fft235_plan1d_new(nz, +1);
  fft235_cplx *w = (fft235_cplx *) malloc(sizeof(fft235_cplx) * (size_t) nx * ny * nzh);
  fft235_cplx *a = (fft235_cplx *) malloc(sizeof(fft235_cplx) * (size_t) nmax);
  fft235_cplx *b = (fft235_cplx *) malloc(sizeof(fft235_cplx) * (size_t) nmax);
  int ix, iy, iz;
  memcpy(w, in, sizeof(fft235_cplx) * (size_t) nx * ny * nzh);
  for (iy = 0; iy < ny; iy++)
    for (iz = 0; iz < nzh; iz++) {
      fft235_cplx *base = w + (long) iy * nzh + iz;
      fft235_exec1d(px, base, ny * nzh, b);
      for (ix = 0; ix < nx; ix++)
        base[(long) ix * ny * nzh] = b[ix];
    }
  for (ix = 0; ix < nx; ix++)
    for (iz = 0; iz < nzh; iz++) {
      fft235_cplx *base = w + (long) ix * ny * nzh + iz;
      fft235_exec1d(py, base, nzh, b);
      for (iy = 0; iy < ny; iy++)
        base[(long) iy * nzh] = b[iy];
    }
  for (ix = 0; ix < nx; ix++)
    for (iy = 0; iy < ny; iy++) {
      const fft235_cplx *src = w + ((long) ix * ny + iy) * nzh;
      double *dst = out + ((long) ix * ny + iy) * nz;
      /* Hermitian completion of the last dimension */
      for (iz = 0; iz < nzh; iz++)
        a[iz] = src[iz];
      for (iz = nzh; iz < nz; iz++) {
        a[iz].re = src[nz - iz].re;
        a[iz].im = -src[nz - iz].im;
      }
      fft235_exec1d(pz, a, 1, b);
      for (iz = 0; iz < nz; iz++)
        dst[iz] = b[iz].re;
    }
  free(w);
  free(a);
  free(b);
  fft235_plan1d_delete(px);
  fft235_plan1d_delete(py);
  fft235_plan1d_delete(pz);
}

/* LAPACK subset for the reference's src/linalg.cpp -- TEST INFRASTRUCTURE ONLY.
   dgesv_ solves A x = b by Gaussian elimination with partial pivoting (written
   here from the method; column-major storage and the Fortran calling
   convention of the LAPACK interface, which LinearSolve, src/linalg.cpp:29-37,
   calls).  The other routines linalg.cpp references are not reached by the
   constraint solver and stop the program if called. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

void dgesv_(int *n_, int *nrhs_, double *a, int *lda_, int *ipiv, double *b, int *ldb_, int *info)
{
  const int n = *n_, nrhs = *nrhs_, lda = *lda_, ldb = *ldb_;
  *info = 0;
  for (int k = 0; k < n; k++) {
    int p = k;
    for (int i = k + 1; i < n; i++)
      if (fabs(a[i + k * lda]) > fabs(a[p + k * lda]))
        p = i;
    ipiv[k] = p + 1;
    if (a[p + k * lda] == 0) {
      *info = k + 1;
      return;
    }
    if (p != k) {
      for (int j = 0; j < n; j++) {
        const double t = a[k + j * lda];
        a[k + j * lda] = a[p + j * lda];
        a[p + j * lda] = t;
      }
      for (int j = 0; j < nrhs; j++) {
        const double t = b[k + j * ldb];
        b[k + j * ldb] = b[p + j * ldb];
        b[p + j * ldb] = t;
      }
    }
    for (int i = k + 1; i < n; i++) {
      const double l = a[i + k * lda] / a[k + k * lda];
      a[i + k * lda] = l;
      for (int j = k + 1; j < n; j++)
        a[i + j * lda] -= l * a[k + j * lda];
      for (int j = 0; j < nrhs; j++)
        b[i + j * ldb] -= l * b[k + j * ldb];
    }
  }
  for (int j = 0; j < nrhs; j++)
    for (int i = n - 1; i >= 0; i--) {
      double s = b[i + j * ldb];
      for (int c = i + 1; c < n; c++)
        s -= a[i + c * lda] * b[c + j * ldb];
      b[i + j * ldb] = s / a[i + i * lda];
    }
}

static void unavailable(const char *name)
{
  fprintf(stderr, "lapack_shim: %s is not provided\n", name);
  abort();
}

void dsysv_(void) { unavailable("dsysv"); }
void dgels_(void) { unavailable("dgels"); }
void dgglse_(void) { unavailable("dgglse"); }
void dgesvd_(void) { unavailable("dgesvd"); }
void dsyev_(void) { unavailable("dsyev"); }
void dgeev_(void) { unavailable("dgeev"); }

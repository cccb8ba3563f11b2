/*
 * GSL stub: declarations only, so that the reference's src/pppm.c compiles in
 * the oracle build (GSL is not installed in this image).  The only user is
 * p3m_optimize (src/pppm.c:682-716), which the oracle never calls: every
 * workload fixes the Ewald screening parameter, so ElecLJ takes the p3m_init
 * branch (src/eleclj.cpp:204-211).  Every function here aborts if reached.
 * TEST INFRASTRUCTURE ONLY.
 */
#ifndef ORACLE_GSL_MULTIMIN_STUB_H
#define ORACLE_GSL_MULTIMIN_STUB_H

#include <stdio.h>
#include <stdlib.h>
#include <stddef.h>

#define GSL_SUCCESS 0

typedef struct { size_t size; double *data; } gsl_vector;
typedef struct { double (*f)(const gsl_vector *, void *); size_t n; void *params; } gsl_multimin_function;
typedef struct { const char *name; } gsl_multimin_fminimizer_type;
typedef struct { gsl_vector *x; } gsl_multimin_fminimizer;

static const gsl_multimin_fminimizer_type oracle_gsl_nmsimplex_stub = {"nmsimplex"};
#define gsl_multimin_fminimizer_nmsimplex (&oracle_gsl_nmsimplex_stub)

static inline void oracle_gsl_unavailable(void)
{
  fprintf(stderr, "oracle GSL stub: p3m_optimize needs GSL; set ewald_screening > 0\n");
  abort();
}
static inline gsl_vector *gsl_vector_alloc(size_t n) { (void) n; oracle_gsl_unavailable(); return 0; }
static inline void gsl_vector_free(gsl_vector *v) { (void) v; }
static inline void gsl_vector_set(gsl_vector *v, size_t i, double x) { (void) v; (void) i; (void) x; oracle_gsl_unavailable(); }
static inline double gsl_vector_get(const gsl_vector *v, size_t i) { (void) v; (void) i; oracle_gsl_unavailable(); return 0; }
static inline gsl_multimin_fminimizer *gsl_multimin_fminimizer_alloc(const gsl_multimin_fminimizer_type *t, size_t n)
{ (void) t; (void) n; oracle_gsl_unavailable(); return 0; }
static inline void gsl_multimin_fminimizer_free(gsl_multimin_fminimizer *s) { (void) s; }
static inline int gsl_multimin_fminimizer_set(gsl_multimin_fminimizer *s, gsl_multimin_function *f, const gsl_vector *x, const gsl_vector *step)
{ (void) s; (void) f; (void) x; (void) step; oracle_gsl_unavailable(); return 0; }
static inline int gsl_multimin_fminimizer_iterate(gsl_multimin_fminimizer *s) { (void) s; oracle_gsl_unavailable(); return 0; }
static inline double gsl_multimin_fminimizer_size(const gsl_multimin_fminimizer *s) { (void) s; oracle_gsl_unavailable(); return 0; }
static inline int gsl_multimin_test_size(double size, double tol) { (void) size; (void) tol; oracle_gsl_unavailable(); return 0; }

#endif

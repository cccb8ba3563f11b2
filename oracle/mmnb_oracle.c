/*
 * mmnb_oracle.c — CPU restatement of msim's nonbonded force path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the GPU library is compared
 * against; the product never links, loads or calls it.  It restates, in plain
 * C, the reference algorithm function by function (citations are paths inside
 * the reference project):
 *
 *   Chebyshev erfc(eta r)/r table      src/cheby.c:7-45, src/rspace.c:18-37
 *   PairBinary pair sets               src/pbin.c:6-137
 *   cell neighbour list                src/nbrlist.cpp:9-251, include/pbc.h:6-59
 *   real-space Ewald + LJ              src/rspace.c:51-156, 219-242, 258-347, 382-558
 *   P3M                                src/pppm.c:56-59, 277-468, 498-641
 *   ordinary Ewald k-sum               src/kspace.c:35-174
 *   ElecLJ orchestration               src/eleclj.cpp:140-265, 273-308, 712-770,
 *                                      785-807, 912-976, 1247-1266
 *
 * The B-spline charge-assignment weights are not transcribed from the
 * reference's per-order polynomial tables (src/pppm.c:69-275): they come from
 * the Cox-de Boor recursion for cardinal B-splines, an independent route to
 * the same functions, so the oracle also checks those tables.
 *
 * Parity of this restatement is pinned two ways: against the reference's own
 * code compiled by oracle/Makefile (oracle/_ref/libref.so), and against the
 * golden vectors committed under tests/golden/ (generated by that build), plus
 * the one known-answer test the reference ships (src/pbin.c:152-214).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fft235.h"
#include "oracle_api.h"

#define HAS_Q 1  /* include/rspace.h:7 */
#define HAS_LJ 2 /* include/rspace.h:8 */
#define NCHEB 512
#define MAXORDER 7

static double sq(double x) { return x * x; }

/* n mod m, also for negative n (include/fns.h:48-58) */
static int wrapi(int n, int m)
{
  const int k = n % m;
  return k < 0 ? k + m : k;
}

/* 64 machine epsilons (src/fns.c:8-31) */
static int almost_zero(double x) { return fabs(x) < 64 * 2.220446049250313e-16; }

/* ------------------------------------------------------------------------ */
/* Chebyshev table: 512 segments over r^2, each a cubic for erfc(eta r)/r and
   a quadratic for -2 d/d(r^2) of it, from a 50-node Chebyshev fit. */

typedef struct {
  double min, max, inv_dx;
  double c[NCHEB][7];
} cheb_t;

static void cheb_fit_segment(double a, double b, double eta, double *out)
{
  double g[50], c[4];
  const double fac = 2.0 / 50;
  const double bma = 0.5 * (b - a);
  const double bpa = 0.5 * (b + a);
  int k, j;
  for (k = 0; k < 50; k++) {
    const double r2 = cos(M_PI * (k + 0.5) / 50) * bma + bpa;
    const double r = sqrt(r2);
    g[k] = erfc(eta * r) / r;
  }
  for (j = 0; j < 4; j++) {
    double s = 0;
    for (k = 0; k < 50; k++)
      s += g[k] * cos(M_PI * j * (k + 0.5) / 50);
    c[j] = fac * s;
  }
  /* Chebyshev series on [-1,1] rewritten as a power series in x in [0,1) */
  out[0] = c[0] / 2 - c[1] + c[2] - c[3];
  out[1] = 2 * c[1] - 8 * c[2] + 18 * c[3];
  out[2] = 8 * c[2] - 48 * c[3];
  out[3] = 32 * c[3];
  out[4] = -2 * out[1] / (b - a);
  out[5] = -2 * 2 * out[2] / (b - a);
  out[6] = -2 * 3 * out[3] / (b - a);
}

static void cheb_build(cheb_t *t, double rhi, double eta)
{
  const double r2max = 1.2 * sq(rhi);
  const double r2min = r2max > 4 ? 4 : 0.9 * r2max;
  const double dx = (r2max - r2min) / NCHEB;
  int i;
  t->min = r2min;
  t->max = r2max;
  t->inv_dx = 1.0 / dx;
  for (i = 0; i < NCHEB; i++)
    cheb_fit_segment(i * dx + r2min, (i + 1) * dx + r2min, eta, t->c[i]);
}

static void cheb_eval(const cheb_t *t, double r2, double *b0, double *b1)
{
  double x = (r2 - t->min) * t->inv_dx;
  const unsigned i = (unsigned) x;
  const double *c = t->c[i];
  x -= i;
  *b0 = ((c[3] * x + c[2]) * x + c[1]) * x + c[0];
  *b1 = (c[6] * x + c[5]) * x + c[4];
}

int orc_chebyshev(double rc, double eta, double *min, double *max, double *inv_dx, double *coeff)
{
  cheb_t *t = (cheb_t *) malloc(sizeof(cheb_t));
  cheb_build(t, rc, eta);
  *min = t->min;
  *max = t->max;
  *inv_dx = t->inv_dx;
  memcpy(coeff, t->c, sizeof(t->c));
  free(t);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Pair sets.  An unordered pair lives in one row only: the row of the smaller
   index when i+j is odd, of the larger when i+j is even. */

typedef struct {
  int n;
  int *cnt, *cap;
  int **row;
} pset;

static void canon(int *i, int *j)
{
  if (((*i + *j) % 2) ^ (*i < *j)) {
    const int t = *i;
    *i = *j;
    *j = t;
  }
}

static pset *pset_new(int n)
{
  pset *p = (pset *) calloc(1, sizeof(pset));
  int i;
  p->n = n;
  p->cnt = (int *) calloc(n > 0 ? n : 1, sizeof(int));
  p->cap = (int *) calloc(n > 0 ? n : 1, sizeof(int));
  p->row = (int **) calloc(n > 0 ? n : 1, sizeof(int *));
  for (i = 0; i < n; i++) {
    p->cap[i] = 16;
    p->row[i] = (int *) malloc(16 * sizeof(int));
  }
  return p;
}

static void pset_free(pset *p)
{
  int i;
  if (!p)
    return;
  for (i = 0; i < p->n; i++)
    free(p->row[i]);
  free(p->row);
  free(p->cnt);
  free(p->cap);
  free(p);
}

static void pset_add(pset *p, int i, int j)
{
  canon(&i, &j);
  if (p->cnt[i] == p->cap[i]) {
    p->cap[i] *= 2;
    p->row[i] = (int *) realloc(p->row[i], p->cap[i] * sizeof(int));
  }
  p->row[i][p->cnt[i]++] = j;
}

static int cmp_int(const void *a, const void *b)
{
  const int x = *(const int *) a, y = *(const int *) b;
  return (x > y) - (x < y);
}

static void pset_sort_unique(pset *p)
{
  int i;
  for (i = 0; i < p->n; i++) {
    int *r = p->row[i];
    int k = 0, j;
    qsort(r, p->cnt[i], sizeof(int), cmp_int);
    for (j = 1; j < p->cnt[i]; j++)
      if (r[j] != r[k])
        r[++k] = r[j];
    if (p->cnt[i] > 0)
      p->cnt[i] = k + 1;
  }
}

static int pset_has(const pset *p, int i, int j)
{
  int lo = 0, hi;
  const int *r;
  canon(&i, &j);
  r = p->row[i];
  hi = p->cnt[i] - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) / 2;
    if (j < r[mid])
      hi = mid - 1;
    else if (j > r[mid])
      lo = mid + 1;
    else
      return 1;
  }
  return 0;
}

static long pset_total(const pset *p)
{
  long s = 0;
  int i;
  for (i = 0; i < p->n; i++)
    s += p->cnt[i];
  return s;
}

static void pset_dump(const pset *p, int *out)
{
  long k = 0;
  int i, j;
  for (i = 0; i < p->n; i++)
    for (j = 0; j < p->cnt[i]; j++) {
      out[2 * k] = i;
      out[2 * k + 1] = p->row[i][j];
      k++;
    }
}

int orc_pairset_demo(int n, int nadd, const int *adds, int *cnt, int *rows, int *exists)
{
  pset *p = pset_new(n);
  int i, j;
  for (i = 0; i < nadd; i++)
    pset_add(p, adds[2 * i], adds[2 * i + 1]);
  pset_sort_unique(p);
  for (i = 0; i < n; i++) {
    cnt[i] = p->cnt[i];
    for (j = 0; j < p->cnt[i] && j < n; j++)
      rows[i * n + j] = p->row[i][j];
    for (j = 0; j < n; j++)
      exists[i * n + j] = pset_has(p, i, j);
  }
  pset_free(p);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Boxes: cubic (type 1) and orthorhombic (type 2), include/bcondtype.h:8. */

typedef struct {
  int type;
  double l[3];
} box_t;

/* x - L round(x/L) per axis (include/pbc.h:8-14, 33-40) */
static void box_wrap(const box_t *b, double *v)
{
  int d;
  for (d = 0; d < 3; d++) {
    const double L = b->l[d];
    v[d] -= L * floor(v[d] * (1 / L) + 0.5);
  }
}

static double box_volume(const box_t *b) { return b->l[0] * b->l[1] * b->l[2]; }

static double box_min_diameter(const box_t *b)
{
  const double m = b->l[0] < b->l[1] ? b->l[0] : b->l[1];
  return m < b->l[2] ? m : b->l[2];
}

/* ------------------------------------------------------------------------ */
/* Cell neighbour list over group anchors. */

typedef struct {
  int n, ncell, ncell3, first;
  double cutoff, width;
  box_t box, cellbox;
  double *last;
  pset *pairs, *cellpairs;
  int *head, *next;
} nbr_t;

static int cell_of(const nbr_t *nl, const double *x)
{
  int ijk[3], d;
  for (d = 0; d < 3; d++)
    ijk[d] = (int) floor(x[d] / nl->cellbox.l[d] + 0.5);
  return (wrapi(ijk[0], nl->ncell) * nl->ncell + wrapi(ijk[1], nl->ncell)) * nl->ncell +
         wrapi(ijk[2], nl->ncell);
}

static void nbr_set_box(nbr_t *nl, const box_t *b)
{
  const int nc = nl->ncell;
  double maxdiam, mindiam, c2, vol, a01, a02, a12, amax;
  int nmax, jx, jy, jz, d, ix, iy, iz;
  nl->box = *b;
  nl->cellbox = *b;
  for (d = 0; d < 3; d++)
    nl->cellbox.l[d] = b->l[d] * (1.0 / nc);
  {
    const double *c = nl->cellbox.l;
    if (b->type == 1)
      maxdiam = sqrt(3.0) * c[0];
    else
      maxdiam = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    /* inscribed-sphere diameter of the cell as a general parallelepiped */
    vol = fabs(c[0] * c[1] * c[2]);
    a01 = sqrt(sq(c[0] * c[1]));
    a02 = sqrt(sq(c[0] * c[2]));
    a12 = sqrt(sq(c[1] * c[2]));
    amax = a01 > a02 ? a01 : a02;
    amax = amax > a12 ? amax : a12;
    mindiam = vol / amax;
  }
  c2 = sq(nl->cutoff + nl->width + maxdiam);
  nmax = (int) ceil((nl->cutoff + nl->width + maxdiam) / mindiam);
  if (nmax > nc / 2 + 1)
    nmax = nc / 2 + 1;
  pset_free(nl->cellpairs);
  nl->cellpairs = pset_new(nl->ncell3);
  for (jx = 0; jx <= nmax; jx++)
    for (jy = (jx == 0 ? 0 : -nmax); jy <= nmax; jy++)
      for (jz = (jx == 0 && jy == 0 ? 1 : -nmax); jz <= nmax; jz++) {
        double v[3];
        v[0] = nl->cellbox.l[0] * jx;
        v[1] = nl->cellbox.l[1] * jy;
        v[2] = nl->cellbox.l[2] * jz;
        box_wrap(&nl->cellbox, v);
        if (v[0] * v[0] + v[1] * v[1] + v[2] * v[2] < c2)
          for (ix = 0; ix < nc; ix++)
            for (iy = 0; iy < nc; iy++)
              for (iz = 0; iz < nc; iz++) {
                const int ia = (wrapi(ix, nc) * nc + wrapi(iy, nc)) * nc + wrapi(iz, nc);
                const int ib = (wrapi(ix + jx, nc) * nc + wrapi(iy + jy, nc)) * nc + wrapi(iz + jz, nc);
                if (ia != ib)
                  pset_add(nl->cellpairs, ia, ib);
              }
      }
  pset_sort_unique(nl->cellpairs);
  nl->first = 1;
}

static nbr_t *nbr_new(int n, double cutoff, double width, const box_t *b)
{
  nbr_t *nl = (nbr_t *) calloc(1, sizeof(nbr_t));
  nl->n = n;
  nl->ncell = (int) floor(cbrt(n / 2 + 3));
  nl->ncell3 = nl->ncell * nl->ncell * nl->ncell;
  nl->cutoff = cutoff;
  nl->width = width;
  nl->last = (double *) calloc(3 * (size_t) (n > 0 ? n : 1), sizeof(double));
  nl->pairs = pset_new(n);
  nl->head = (int *) malloc(sizeof(int) * nl->ncell3);
  nl->next = (int *) malloc(sizeof(int) * (n > 0 ? n : 1));
  nbr_set_box(nl, b);
  return nl;
}

static void nbr_free(nbr_t *nl)
{
  if (!nl)
    return;
  free(nl->last);
  pset_free(nl->pairs);
  pset_free(nl->cellpairs);
  free(nl->head);
  free(nl->next);
  free(nl);
}

static void nbr_rebuild(nbr_t *nl, const double *r)
{
  const double c2 = sq(nl->cutoff + nl->width);
  int i, c;
  for (i = 0; i < nl->n; i++)
    nl->pairs->cnt[i] = 0;
  for (c = 0; c < nl->ncell3; c++)
    nl->head[c] = -1;
  for (i = 0; i < nl->n; i++) {
    const int ic = cell_of(nl, r + 3 * i);
    nl->next[i] = nl->head[ic];
    nl->head[ic] = i;
  }
  for (c = 0; c < nl->ncell3; c++) {
    const int nj = nl->cellpairs->cnt[c];
    const int *cj = nl->cellpairs->row[c];
    int k, l, m;
    for (k = nl->head[c]; k != -1; k = nl->next[k]) {
      for (l = nl->next[k]; l != -1; l = nl->next[l])
        pset_add(nl->pairs, k, l); /* same cell: no distance test */
      for (m = 0; m < nj; m++)
        for (l = nl->head[cj[m]]; l != -1; l = nl->next[l]) {
          double v[3];
          v[0] = r[3 * k] - r[3 * l];
          v[1] = r[3 * k + 1] - r[3 * l + 1];
          v[2] = r[3 * k + 2] - r[3 * l + 2];
          box_wrap(&nl->box, v);
          if (v[0] * v[0] + v[1] * v[1] + v[2] * v[2] < c2)
            pset_add(nl->pairs, k, l);
        }
    }
  }
  memcpy(nl->last, r, sizeof(double) * 3 * (size_t) nl->n);
}

/* Rebuild when the two largest anchor moves since the last build add up to
   more than the skin (src/nbrlist.cpp:51-77). */
static int nbr_update(nbr_t *nl, const double *r)
{
  double largest = 0, second = 0;
  int i;
  if (nl->first) {
    nl->first = 0;
    nbr_rebuild(nl, r);
    return 1;
  }
  for (i = 0; i < nl->n; i++) {
    const double dx = r[3 * i] - nl->last[3 * i];
    const double dy = r[3 * i + 1] - nl->last[3 * i + 1];
    const double dz = r[3 * i + 2] - nl->last[3 * i + 2];
    const double d = sqrt(dx * dx + dy * dy + dz * dz);
    if (d > largest) {
      second = largest;
      largest = d;
    } else if (d > second) {
      second = d;
    }
  }
  if (second + largest > nl->width) {
    nbr_rebuild(nl, r);
    return 1;
  }
  return 0;
}

static box_t make_box(int bctype, const double *l)
{
  box_t b;
  b.type = bctype;
  b.l[0] = l[0];
  b.l[1] = bctype == 1 ? l[0] : l[1];
  b.l[2] = bctype == 1 ? l[0] : l[2];
  return b;
}

void *orc_nbrlist_new(int ngroup, double cutoff, double width, int bctype, const double box[3])
{
  box_t b;
  if (bctype != 1 && bctype != 2)
    return 0;
  b = make_box(bctype, box);
  return nbr_new(ngroup, cutoff, width, &b);
}

int orc_nbrlist_update(void *h, const double *gr) { return nbr_update((nbr_t *) h, gr); }
long orc_nbrlist_npairs(void *h) { return pset_total(((nbr_t *) h)->pairs); }
void orc_nbrlist_pairs(void *h, int *pairs) { pset_dump(((nbr_t *) h)->pairs, pairs); }
int orc_nbrlist_ncell(void *h) { return ((nbr_t *) h)->ncell; }

void orc_nbrlist_cells(void *h, int *cell)
{
  nbr_t *nl = (nbr_t *) h;
  int c, k;
  for (k = 0; k < nl->n; k++)
    cell[k] = -1;
  for (c = 0; c < nl->ncell3; c++)
    for (k = nl->head[c]; k != -1; k = nl->next[k])
      cell[k] = c;
}

long orc_nbrlist_ncellpairs(void *h) { return pset_total(((nbr_t *) h)->cellpairs); }
void orc_nbrlist_cellpairs(void *h, int *pairs) { pset_dump(((nbr_t *) h)->cellpairs, pairs); }
void orc_nbrlist_delete(void *h) { nbr_free((nbr_t *) h); }

/* ------------------------------------------------------------------------ */
/* Real-space pair terms (src/rspace.c:51-347). */

typedef struct {
  const double *q, *sig, *eps, *rscreen;
  double *phi, *evec, *ljf, *lj_energy;
  int geometric;
} pairctx;

/* quintic switch in z = (r^2 - rlo^2)/(rhi^2 - rlo^2) and 2 dS/d(r^2) */
static void switch_fn(double r2, double rlo2, double rhi2, double *s, double *ds)
{
  const double a = 1.0 / (rhi2 - rlo2);
  const double z = (r2 - rlo2) * a;
  *s = ((-6 * z + 15) * z - 10) * z * z * z + 1;
  *ds = ((60 * z - 120) * z + 60) * z * z * a;
}

static void coulomb_add(const pairctx *c, int i, int j, const double *d, double b0, double b1)
{
  const double qib1 = c->q[i] * b1, qjb1 = c->q[j] * b1;
  c->phi[i] += c->q[j] * b0;
  c->evec[3 * i] += qjb1 * d[0];
  c->evec[3 * i + 1] += qjb1 * d[1];
  c->evec[3 * i + 2] += qjb1 * d[2];
  c->phi[j] += c->q[i] * b0;
  c->evec[3 * j] -= qib1 * d[0];
  c->evec[3 * j + 1] -= qib1 * d[1];
  c->evec[3 * j + 2] -= qib1 * d[2];
}

/* erfc-screened Coulomb, with the short-range screening correction
   (src/rspace.c:60-64, 104-156) */
static void ewald_pair(const pairctx *c, int i, int j, const double *d, double r2, double eta,
                       const cheb_t *t, int smoothing, double s, double *tmps)
{
  double b0, b1;
  const double rs = c->rscreen[i] + c->rscreen[j];
  if (t->min < r2 && r2 < t->max) {
    cheb_eval(t, r2, &b0, &b1);
  } else {
    const double r = sqrt(r2);
    const double er = eta * r;
    const double e = exp(-sq(er));
    b0 = erfc(er) / r;
    b1 = (b0 + eta * M_2_SQRTPI * e) / r2;
  }
  if (r2 < rs * rs) {
    const double invr = 1.0 / sqrt(r2);
    const double inv3 = 1.0 / (rs * rs * rs);
    b0 += (-0.5 * r2 * inv3 + 1.5 / rs) - invr;
    b1 += inv3 - invr * invr * invr;
  }
  if (smoothing) {
    *tmps += c->q[i] * c->q[j] * b0;
    b0 *= s;
    b1 *= s;
  }
  coulomb_add(c, i, j, d, b0, b1);
}

/* plain Coulomb with optional screening and scaling (src/rspace.c:66-102) */
static void coulomb_plain(const pairctx *c, int i, int j, const double *d, double r2,
                          int scaling, double scale)
{
  double b0, b1;
  const double rs = c->rscreen[i] + c->rscreen[j];
  if (r2 < rs * rs) {
    b1 = 1.0 / (rs * rs * rs);
    b0 = -0.5 * r2 * b1 + 1.5 / rs;
  } else {
    const double invr = 1.0 / sqrt(r2);
    b0 = invr;
    b1 = invr * invr * invr;
  }
  if (scaling) {
    b0 *= scale;
    b1 *= scale;
  }
  coulomb_add(c, i, j, d, b0, b1);
}

/* 12-6 LJ with arithmetic (or geometric) sigma and geometric epsilon
   (src/rspace.c:258-297) */
static void lj_pair(const pairctx *c, int i, int j, const double *d, double r2,
                    int smoothing, double s, double *tmps, int scaling, double scale)
{
  const double s2 = c->geometric ? c->sig[i] * c->sig[j] : sq(0.5 * (c->sig[i] + c->sig[j]));
  const double s6 = s2 * s2 * s2;
  const double b = 4 * sqrt(c->eps[i] * c->eps[j]) * s6;
  const double a = b * s6;
  const double invr2 = 1.0 / r2;
  const double invr6 = invr2 * invr2 * invr2;
  const double binvr6 = b * invr6;
  const double ainvr12 = a * invr6 * invr6;
  double du = 12 * ainvr12 * invr2 - 6 * binvr6 * invr2;
  double u = ainvr12 - binvr6;
  int k;
  if (smoothing) {
    *tmps += u;
    u *= s;
    du *= s;
  }
  if (scaling) {
    u *= scale;
    du *= scale;
  }
  *c->lj_energy += u;
  for (k = 0; k < 3; k++) {
    c->ljf[3 * i + k] += du * d[k];
    c->ljf[3 * j + k] -= du * d[k];
  }
}

/* ------------------------------------------------------------------------ */
/* Ordinary Ewald k-sum (src/kspace.c:35-174). */

typedef struct { int x, y, z, n2; } kint;

static int kint_desc(const void *a, const void *b)
{
  const int x = ((const kint *) a)->n2, y = ((const kint *) b)->n2;
  return (x < y) - (x > y);
}

/* recip: reciprocal lattice (2 pi inv(latv)^T) in tensor_t layout */
static int kspace_sum(double kc, int nsite, const double *r, const double *q, const double *recip,
                      double volume, double eta, double *phi, double *evec)
{
  const double n2max = kc * kc + 1e-8;
  const int nmax = (int) floor(kc);
  int nk = 0, nx, ny, nz, i, k;
  kint *kv;
  double *kvec, *ak, *cs, *sn, *cQ, *sQ, *ct, *st;
  for (nx = 0; nx <= nmax; nx++)
    for (ny = (nx == 0 ? 0 : -nmax); ny <= nmax; ny++)
      for (nz = (nx == 0 && ny == 0 ? 1 : -nmax); nz <= nmax; nz++)
        if (nx * nx + ny * ny + nz * nz <= n2max)
          nk++;
  kv = (kint *) malloc(sizeof(kint) * (nk > 0 ? nk : 1));
  nk = 0;
  for (nx = 0; nx <= nmax; nx++)
    for (ny = (nx == 0 ? 0 : -nmax); ny <= nmax; ny++)
      for (nz = (nx == 0 && ny == 0 ? 1 : -nmax); nz <= nmax; nz++)
        if (nx * nx + ny * ny + nz * nz <= n2max) {
          kv[nk].x = nx;
          kv[nk].y = ny;
          kv[nk].z = nz;
          kv[nk].n2 = nx * nx + ny * ny + nz * nz;
          nk++;
        }
  qsort(kv, nk, sizeof(kint), kint_desc);
  kvec = (double *) malloc(sizeof(double) * 3 * (nk + 1));
  ak = (double *) malloc(sizeof(double) * (nk + 1));
  cs = (double *) malloc(sizeof(double) * (size_t) nsite * (nk + 1));
  sn = (double *) malloc(sizeof(double) * (size_t) nsite * (nk + 1));
  cQ = (double *) calloc(nk + 1, sizeof(double));
  sQ = (double *) calloc(nk + 1, sizeof(double));
  ct = (double *) malloc(sizeof(double) * 3 * (2 * nmax + 1));
  st = (double *) malloc(sizeof(double) * 3 * (2 * nmax + 1));
  {
    const double c = 0.25 / (eta * eta), f = 4 * M_PI / volume;
    for (k = 0; k < nk; k++) {
      double k2;
      kvec[3 * k] = recip[0] * kv[k].x + recip[3] * kv[k].y + recip[6] * kv[k].z;
      kvec[3 * k + 1] = recip[1] * kv[k].x + recip[4] * kv[k].y + recip[7] * kv[k].z;
      kvec[3 * k + 2] = recip[2] * kv[k].x + recip[5] * kv[k].y + recip[8] * kv[k].z;
      k2 = sq(kvec[3 * k]) + sq(kvec[3 * k + 1]) + sq(kvec[3 * k + 2]);
      ak[k] = f * exp(-k2 * c) / k2;
    }
  }
  for (i = 0; i < nsite; i++) {
    double t[3], c1[3], s1[3];
    int d, m;
    /* phase along each reciprocal vector: b_d . r */
    for (d = 0; d < 3; d++) {
      t[d] = recip[3 * d] * r[3 * i] + recip[3 * d + 1] * r[3 * i + 1] + recip[3 * d + 2] * r[3 * i + 2];
      c1[d] = cos(t[d]);
      s1[d] = sin(t[d]);
    }
    /* cos/sin of m*t by angle addition, m = -nmax..nmax */
    for (d = 0; d < 3; d++) {
      ct[3 * nmax + d] = 1;
      st[3 * nmax + d] = 0;
      for (m = 1; m <= nmax; m++) {
        const double cp = ct[3 * (nmax + m - 1) + d], sp = st[3 * (nmax + m - 1) + d];
        ct[3 * (nmax + m) + d] = c1[d] * cp - s1[d] * sp;
        st[3 * (nmax + m) + d] = s1[d] * cp + c1[d] * sp;
        ct[3 * (nmax - m) + d] = ct[3 * (nmax + m) + d];
        st[3 * (nmax - m) + d] = -st[3 * (nmax + m) + d];
      }
    }
    for (k = 0; k < nk; k++) {
      const double cx = ct[3 * (nmax + kv[k].x)], sx = st[3 * (nmax + kv[k].x)];
      const double cy = ct[3 * (nmax + kv[k].y) + 1], sy = st[3 * (nmax + kv[k].y) + 1];
      const double cz = ct[3 * (nmax + kv[k].z) + 2], sz = st[3 * (nmax + kv[k].z) + 2];
      const double cc = cx * cy - sx * sy;
      const double sc = sx * cy + cx * sy;
      cs[(size_t) i * nk + k] = cc * cz - sc * sz;
      sn[(size_t) i * nk + k] = sc * cz + cc * sz;
    }
  }
  for (i = 0; i < nsite; i++)
    for (k = 0; k < nk; k++) {
      sQ[k] += q[i] * sn[(size_t) i * nk + k];
      cQ[k] += q[i] * cs[(size_t) i * nk + k];
    }
  for (i = 0; i < nsite; i++) {
    double gx = 0, gy = 0, gz = 0, p = 0;
    for (k = 0; k < nk; k++) {
      const double a2 = 2 * ak[k];
      const double s = sn[(size_t) i * nk + k], c = cs[(size_t) i * nk + k];
      const double im = a2 * (cQ[k] * s - sQ[k] * c);
      gx += im * kvec[3 * k];
      gy += im * kvec[3 * k + 1];
      gz += im * kvec[3 * k + 2];
      p += a2 * (sQ[k] * s + cQ[k] * c);
    }
    phi[i] += p;
    evec[3 * i] += gx;
    evec[3 * i + 1] += gy;
    evec[3 * i + 2] += gz;
  }
  free(kv); free(kvec); free(ak); free(cs); free(sn); free(cQ); free(sQ); free(ct); free(st);
  return nk;
}

/* 3x3 helpers in tensor_t layout: T[row r][col c] = t[3c + r] */
static double t_det(const double *t)
{
  const double xx = t[0], yx = t[1], zx = t[2], xy = t[3], yy = t[4], zy = t[5], xz = t[6], yz = t[7], zz = t[8];
  return -xz * yy * zx + xy * yz * zx + xz * yx * zy - xx * yz * zy - xy * yx * zz + xx * yy * zz;
}

static void t_inverse(double *a, const double *b)
{
  const double xx = b[0], yx = b[1], zx = b[2], xy = b[3], yy = b[4], zy = b[5], xz = b[6], yz = b[7], zz = b[8];
  const double id = 1.0 / t_det(b);
  a[0] = id * (-yz * zy + yy * zz);
  a[3] = id * (xz * zy - xy * zz);
  a[6] = id * (-xz * yy + xy * yz);
  a[1] = id * (yz * zx - yx * zz);
  a[4] = id * (-xz * zx + xx * zz);
  a[7] = id * (xz * yx - xx * yz);
  a[2] = id * (-yy * zx + yx * zy);
  a[5] = id * (xy * zx - xx * zy);
  a[8] = id * (-xy * yx + xx * yy);
}

/* 2 pi inv(latv)^T */
static void t_reciprocal(double *rec, const double *latv)
{
  double inv[9];
  int r, c;
  t_inverse(inv, latv);
  for (r = 0; r < 3; r++)
    for (c = 0; c < 3; c++)
      rec[3 * c + r] = 2 * M_PI * inv[3 * r + c];
}

int orc_kspace_field(double kspace_cutoff, int nsite, const double *r, const double *q,
                     const double latv[9], double eta, double *phi, double *evec, int *nk)
{
  double rec[9];
  int n;
  t_reciprocal(rec, latv);
  n = kspace_sum(kspace_cutoff, nsite, r, q, rec, fabs(t_det(latv)), eta, phi, evec);
  if (nk)
    *nk = n;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* P3M. */

typedef struct {
  int nsite, nalias, ik, order;
  double spacing;
  double latv[9], invlatv[9];
  int n[3];
  double *green;   /* [nx][ny][nz/2+1] */
  double *kvec;    /* [nx][ny][nz/2+1][3] */
  double *mesh;
  fft235_cplx *meshk;
  double *egrid[3];
  fft235_cplx *egridk[3];
} p3m_o;

/* nearest 2^a 3^b 5^c 7^d to x; ties keep the first found (src/pppm.c:277-292) */
static int near_2357(double x)
{
  int p2, p3, p5, p7, best = 1;
  double bestdiff = fabs(x - 1);
  for (p2 = 1; p2 <= x; p2 *= 2)
    for (p3 = p2; p3 <= x; p3 *= 3)
      for (p5 = p3; p5 <= x; p5 *= 5)
        for (p7 = p5; p7 <= x; p7 *= 7) {
          const double diff = fabs(x - p7);
          if (diff < bestdiff) {
            bestdiff = diff;
            best = p7;
          }
        }
  return best;
}

static double sincpi(double x)
{
  const double y = M_PI * x;
  return fabs(y) < 1e-16 ? 1 - sq(y) / 6 : sin(y) / y;
}

/* Cardinal B-spline weights of order P at offset w in [0,1]: m[i] = M_P(w + i),
   dm[i] = M_P'(w + i), from M_P(x) = (x M_{P-1}(x) + (P - x) M_{P-1}(x-1)) / (P-1). */
static void bspline(int P, double w, double *m, double *dm)
{
  double prev[MAXORDER + 1];
  int k, i;
  m[0] = 1;
  for (k = 2; k <= P; k++) {
    const double inv = 1.0 / (k - 1);
    for (i = 0; i < k - 1; i++)
      prev[i] = m[i];
    for (i = 0; i < k; i++) {
      const double a = i < k - 1 ? prev[i] : 0;
      const double b = i > 0 ? prev[i - 1] : 0;
      m[i] = ((w + i) * a + (k - w - i) * b) * inv;
    }
    if (k == P && dm)
      for (i = 0; i < P; i++)
        dm[i] = (i < P - 1 ? prev[i] : 0) - (i > 0 ? prev[i - 1] : 0);
  }
  if (P == 1 && dm)
    dm[0] = 0;
}

/* Hockney-Eastwood optimal influence function with alias sum |p| <= nalias
   (src/pppm.c:313-393).  Returns the dimensionless RMS force error estimate. */
static double p3m_green(p3m_o *t, double eta)
{
  const int nx = t->n[0], ny = t->n[1], nz = t->n[2], nzh = nz / 2 + 1;
  const int na = t->nalias, P = t->order;
  const double inv_4eta2 = 1 / sq(2 * eta);
  const double inv_v = 1.0 / fabs(t_det(t->latv));
  double rec[9], chi = 0;
  double *u2x = (double *) malloc(sizeof(double) * (2 * na + 1));
  double *u2y = (double *) malloc(sizeof(double) * (2 * na + 1));
  double *u2z = (double *) malloc(sizeof(double) * (2 * na + 1));
  int ix, iy, iz;
  t_reciprocal(rec, t->latv);
  for (ix = 0; ix < nx; ix++) {
    const double jx = ix > nx / 2 ? ix - nx : ix;
    for (iy = 0; iy < ny; iy++) {
      const double jy = iy > ny / 2 ? iy - ny : iy;
      for (iz = 0; iz < nzh; iz++) {
        const double jz = iz;
        const size_t g = ((size_t) ix * ny + iy) * nzh + iz;
        double kv[3], k2, num = 0, den1 = 0, den2 = 0, den;
        int a, px, py, pz;
        kv[0] = rec[0] * jx + rec[3] * jy + rec[6] * jz;
        kv[1] = rec[1] * jx + rec[4] * jy + rec[7] * jz;
        kv[2] = rec[2] * jx + rec[5] * jy + rec[8] * jz;
        t->kvec[3 * g] = kv[0];
        t->kvec[3 * g + 1] = kv[1];
        t->kvec[3 * g + 2] = kv[2];
        if (ix == 0 && iy == 0 && iz == 0) {
          t->green[g] = 0;
          continue;
        }
        k2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
        for (a = -na; a <= na; a++) {
          u2x[a + na] = pow(sincpi(jx / nx + a), 2 * P);
          u2y[a + na] = pow(sincpi(jy / ny + a), 2 * P);
          u2z[a + na] = pow(sincpi(jz / nz + a), 2 * P);
        }
        for (px = -na; px <= na; px++) {
          const double mx = jx + px * nx;
          for (py = -na; py <= na; py++) {
            const double my = jy + py * ny;
            for (pz = -na; pz <= na; pz++) {
              const double mz = jz + pz * nz;
              double kp[3], kp2, u2, gg;
              if (fabs(mx) < 1e-16 && fabs(my) < 1e-16 && fabs(mz) < 1e-16)
                continue;
              kp[0] = rec[0] * mx + rec[3] * my + rec[6] * mz;
              kp[1] = rec[1] * mx + rec[4] * my + rec[7] * mz;
              kp[2] = rec[2] * mx + rec[5] * my + rec[8] * mz;
              kp2 = kp[0] * kp[0] + kp[1] * kp[1] + kp[2] * kp[2];
              u2 = u2x[px + na] * u2y[py + na] * u2z[pz + na];
              gg = 4 * M_PI / kp2 * exp(-kp2 * inv_4eta2);
              if (t->ik) {
                num += gg * u2 * (kv[0] * kp[0] + kv[1] * kp[1] + kv[2] * kp[2]);
                den1 += u2;
              } else {
                num += gg * kp2 * u2;
                den1 += u2;
                den2 += u2 * kp2;
              }
              chi += gg * gg * kp2;
            }
          }
        }
        den = t->ik ? sq(den1) * k2 : den1 * den2;
        t->green[g] = inv_v * num / den;
        chi -= sq(num) / den;
      }
    }
  }
  free(u2x);
  free(u2y);
  free(u2z);
  return pow(inv_v, 1.0 / 3.0) * sqrt(2 * fabs(chi));
}

void *orc_p3m_new(int nsite, const double latv[9], double grid_spacing, int nalias,
                  int ik_differentiate, int assignment_order, double eta, int ngrid[3], double *chi)
{
  p3m_o *t;
  int d;
  size_t nr, nk;
  if (assignment_order < 2 || assignment_order > MAXORDER || nalias < 1 || !(grid_spacing > 0))
    return 0;
  t = (p3m_o *) calloc(1, sizeof(p3m_o));
  t->nsite = nsite;
  t->nalias = nalias;
  t->ik = ik_differentiate;
  t->order = assignment_order;
  t->spacing = grid_spacing;
  memcpy(t->latv, latv, sizeof(t->latv));
  t_inverse(t->invlatv, latv);
  for (d = 0; d < 3; d++) {
    const double a = sqrt(sq(latv[3 * d]) + sq(latv[3 * d + 1]) + sq(latv[3 * d + 2]));
    t->n[d] = near_2357(floor(a / grid_spacing + 0.5));
    ngrid[d] = t->n[d];
  }
  nr = (size_t) t->n[0] * t->n[1] * t->n[2];
  nk = (size_t) t->n[0] * t->n[1] * (t->n[2] / 2 + 1);
  t->green = (double *) malloc(sizeof(double) * nk);
  t->kvec = (double *) malloc(sizeof(double) * 3 * nk);
  t->mesh = (double *) malloc(sizeof(double) * nr);
  t->meshk = (fft235_cplx *) malloc(sizeof(fft235_cplx) * nk);
  if (t->ik)
    for (d = 0; d < 3; d++) {
      t->egrid[d] = (double *) malloc(sizeof(double) * nr);
      t->egridk[d] = (fft235_cplx *) malloc(sizeof(fft235_cplx) * nk);
    }
  {
    const double c = p3m_green(t, eta);
    if (chi)
      *chi = c;
  }
  return t;
}

void orc_p3m_delete(void *p)
{
  p3m_o *t = (p3m_o *) p;
  int d;
  if (!t)
    return;
  free(t->green);
  free(t->kvec);
  free(t->mesh);
  free(t->meshk);
  for (d = 0; d < 3; d++) {
    free(t->egrid[d]);
    free(t->egridk[d]);
  }
  free(t);
}

/* spread, r2c, influence multiply, c2r, gather (src/pppm.c:498-641) */
static void p3m_apply(p3m_o *t, const double *r, const double *q, double *phi, double *evec)
{
  const int nx = t->n[0], ny = t->n[1], nz = t->n[2], nzh = nz / 2 + 1, P = t->order;
  const int lo = -((P + 1) / 2 - 1);
  const size_t nr = (size_t) nx * ny * nz, nk = (size_t) nx * ny * nzh;
  double A[9]; /* mesh-scaled inverse lattice: s = A r */
  double *W = (double *) malloc(sizeof(double) * 3 * P * (size_t) t->nsite);
  double *D = (double *) malloc(sizeof(double) * 3 * P * (size_t) t->nsite);
  int *I = (int *) malloc(sizeof(int) * 3 * P * (size_t) t->nsite);
  int i, d, a, b, c;
  size_t g;
  for (d = 0; d < 9; d++)
    A[d] = t->invlatv[d] * t->n[d % 3];
  memset(t->mesh, 0, sizeof(double) * nr);
  for (i = 0; i < t->nsite; i++) {
    double *w = W + 3 * P * (size_t) i, *dw = D + 3 * P * (size_t) i;
    int *ix = I + 3 * P * (size_t) i;
    for (d = 0; d < 3; d++) {
      const double s = A[d] * r[3 * i] + A[3 + d] * r[3 * i + 1] + A[6 + d] * r[3 * i + 2];
      double m[MAXORDER], dm[MAXORDER], delta;
      int j, p;
      if (P % 2) {
        j = (int) floor(s + 0.5);
        delta = s - j;
      } else {
        j = (int) floor(s);
        delta = s - (j + 0.5);
      }
      bspline(P, delta + 0.5, m, dm);
      /* point j+lo+p carries m[P-1-p] */
      for (p = 0; p < P; p++) {
        w[p * 3 + d] = m[P - 1 - p];
        dw[p * 3 + d] = -dm[P - 1 - p];
        ix[p * 3 + d] = wrapi(j + lo + p, t->n[d]);
      }
    }
    for (a = 0; a < P; a++)
      for (b = 0; b < P; b++) {
        const double qw = w[a * 3] * w[b * 3 + 1] * q[i];
        for (c = 0; c < P; c++)
          t->mesh[((size_t) ix[a * 3] * ny + ix[b * 3 + 1]) * nz + ix[c * 3 + 2]] += qw * w[c * 3 + 2];
      }
  }
  fft235_r2c_3d(nx, ny, nz, t->mesh, t->meshk);
  for (g = 0; g < nk; g++) {
    t->meshk[g].re *= t->green[g];
    t->meshk[g].im *= t->green[g];
  }
  if (evec && t->ik) {
    for (d = 0; d < 3; d++) {
      for (g = 0; g < nk; g++) {
        const double k = t->kvec[3 * g + d];
        t->egridk[d][g].re = k * t->meshk[g].im;
        t->egridk[d][g].im = -k * t->meshk[g].re;
      }
      fft235_c2r_3d(nx, ny, nz, t->egridk[d], t->egrid[d]);
    }
  }
  fft235_c2r_3d(nx, ny, nz, t->meshk, t->mesh);
  for (i = 0; i < t->nsite; i++) {
    const double *w = W + 3 * P * (size_t) i, *dw = D + 3 * P * (size_t) i;
    const int *ix = I + 3 * P * (size_t) i;
    for (a = 0; a < P; a++)
      for (b = 0; b < P; b++)
        for (c = 0; c < P; c++) {
          const size_t m = ((size_t) ix[a * 3] * ny + ix[b * 3 + 1]) * nz + ix[c * 3 + 2];
          const double wxy = w[a * 3] * w[b * 3 + 1];
          const double pv = t->mesh[m];
          phi[i] += wxy * w[c * 3 + 2] * pv;
          if (evec) {
            if (t->ik) {
              const double ww = wxy * w[c * 3 + 2];
              evec[3 * i] += ww * t->egrid[0][m];
              evec[3 * i + 1] += ww * t->egrid[1][m];
              evec[3 * i + 2] += ww * t->egrid[2][m];
            } else {
              /* -grad_s of the interpolated potential, then E = A^T (-grad_s) */
              const double ex = dw[a * 3] * w[b * 3 + 1] * w[c * 3 + 2] * pv;
              const double ey = w[a * 3] * dw[b * 3 + 1] * w[c * 3 + 2] * pv;
              const double ez = wxy * dw[c * 3 + 2] * pv;
              evec[3 * i] += ex * A[0] + ey * A[1] + ez * A[2];
              evec[3 * i + 1] += ex * A[3] + ey * A[4] + ez * A[5];
              evec[3 * i + 2] += ex * A[6] + ey * A[7] + ez * A[8];
            }
          }
        }
  }
  free(W);
  free(D);
  free(I);
}

void orc_p3m_field(void *p, const double *r, const double *q, double *phi, double *evec)
{
  p3m_apply((p3m_o *) p, r, q, phi, evec);
}

/* ------------------------------------------------------------------------ */
/* ElecLJ for atom sites. */

typedef struct {
  orc_config c;
  int nsite, ngroup;
  int *group, *mask;
  double *q, *sig, *eps, *rscreen;
  box_t box;
  double latv[9];
  double rc, nlw, eta, totA, totB;
  int any_q;
  pset *excl, *gexcl, *p14;
  cheb_t *cheb;
  p3m_o *p3m;
  nbr_t *nl;
  double *phi, *evec, *ljf, *gr;
} elec_t;

static void *dupa(const void *src, size_t bytes)
{
  void *p = malloc(bytes > 0 ? bytes : 1);
  if (bytes)
    memcpy(p, src, bytes);
  return p;
}

typedef struct { double s, e; int n; } ljtype;

void *orc_eleclj_new(const orc_config *c, int nsite, int ngroup, const int *group,
                     int nexcl, const int *excl, int n14, const int *pairs14,
                     const int *site_mask, const double *q, const double *sig,
                     const double *eps, const double *rscreen)
{
  elec_t *h;
  double dmin;
  int i, k;
  if (c->bctype != 1 && c->bctype != 2)
    return 0;
  h = (elec_t *) calloc(1, sizeof(elec_t));
  h->c = *c;
  h->nsite = nsite;
  h->ngroup = ngroup;
  h->group = (int *) dupa(group, sizeof(int) * 2 * ngroup);
  h->mask = (int *) dupa(site_mask, sizeof(int) * nsite);
  h->q = (double *) dupa(q, sizeof(double) * nsite);
  h->sig = (double *) dupa(sig, sizeof(double) * nsite);
  h->eps = (double *) dupa(eps, sizeof(double) * nsite);
  h->rscreen = (double *) dupa(rscreen, sizeof(double) * nsite);
  h->box = make_box(c->bctype, c->box);
  memset(h->latv, 0, sizeof(h->latv));
  h->latv[0] = h->box.l[0];
  h->latv[4] = h->box.l[1];
  h->latv[8] = h->box.l[2];
  for (i = 0; i < nsite; i++)
    if (site_mask[i] & HAS_Q)
      h->any_q = 1;
  /* cutoff and skin defaults and checks (src/eleclj.cpp:164-182) */
  dmin = box_min_diameter(&h->box);
  h->rc = c->rspace_cutoff;
  if (almost_zero(h->rc))
    h->rc = 0.45 * dmin;
  if (h->rc > 0.49 * dmin || !(h->rc > 0) || c->smoothing_width >= h->rc)
    goto fail;
  h->nlw = c->neighbor_list_width;
  if (almost_zero(h->nlw)) {
    h->nlw = 0.2 * h->rc;
    if (h->rc + h->nlw >= 0.5 * dmin)
      h->nlw = 0.499 * dmin - h->rc;
  }
  h->nl = nbr_new(ngroup, h->rc, h->nlw, &h->box);
  /* Ewald parameter and reciprocal-space set-up (src/eleclj.cpp:189-239) */
  h->eta = c->ewald_screening;
  if (h->any_q) {
    if (c->include_kspace && c->use_p3m) {
      int ng[3];
      if (h->eta < 0)
        goto fail; /* the reference would optimise eta with GSL */
      h->p3m = (p3m_o *) orc_p3m_new(nsite, h->latv, c->p3m_grid_spacing, c->p3m_alias_sum_limit,
                                     c->p3m_ik_differentiate, c->p3m_assignment_order, h->eta, ng, 0);
      if (!h->p3m)
        goto fail;
    } else if (h->eta < 0) {
      h->eta = sqrt((M_PI * c->kspace_cutoff) / (h->rc * dmin));
    }
    if (c->include_rspace) {
      h->cheb = (cheb_t *) malloc(sizeof(cheb_t));
      cheb_build(h->cheb, h->rc, h->eta);
    }
  }
  /* exclusions, group exclusions, 1-4 pairs (src/eleclj.cpp:712-770) */
  h->excl = pset_new(nsite);
  for (k = 0; k < nexcl; k++)
    pset_add(h->excl, excl[2 * k], excl[2 * k + 1]);
  pset_sort_unique(h->excl);
  if (!almost_zero(c->elec_1_4_scale_factor - 1) || !almost_zero(c->lj_1_4_scale_factor - 1)) {
    h->p14 = pset_new(nsite);
    for (k = 0; k < n14; k++)
      pset_add(h->p14, pairs14[2 * k], pairs14[2 * k + 1]);
    pset_sort_unique(h->p14);
  }
  {
    int *gs = (int *) malloc(sizeof(int) * (nsite > 0 ? nsite : 1));
    int g, j;
    for (g = 0; g < ngroup; g++)
      for (k = group[2 * g]; k < group[2 * g + 1]; k++)
        gs[k] = g;
    h->gexcl = pset_new(ngroup);
    for (i = 0; i < nsite; i++)
      for (j = 0; j < h->excl->cnt[i]; j++)
        if (gs[i] != gs[h->excl->row[i][j]])
          pset_add(h->gexcl, gs[i], gs[h->excl->row[i][j]]);
    pset_sort_unique(h->gexcl);
    free(gs);
  }
  /* LJ tail totals over distinct (sigma, epsilon) printed as %12.6g
     (src/eleclj.cpp:283-308) */
  {
    ljtype *ty = (ljtype *) calloc(nsite > 0 ? nsite : 1, sizeof(ljtype));
    int nt = 0, a, b;
    for (i = 0; i < nsite; i++) {
      char key[128];
      double s, e;
      if (!(site_mask[i] & HAS_LJ))
        continue;
      snprintf(key, sizeof key, "%12.6g %12.6g", sig[i], eps[i]);
      sscanf(key, "%lf%lf", &s, &e);
      for (a = 0; a < nt; a++)
        if (ty[a].s == s && ty[a].e == e)
          break;
      if (a == nt) {
        ty[nt].s = s;
        ty[nt].e = e;
        nt++;
      }
      ty[a].n++;
    }
    for (a = 0; a < nt; a++)
      for (b = 0; b < nt; b++) {
        const double s6 = pow(c->geometric_combining_for_sigma ? sqrt(ty[a].s * ty[b].s)
                                                              : 0.5 * (ty[a].s + ty[b].s), 6);
        const double bb = 4 * sqrt(ty[a].e * ty[b].e) * ty[a].n * ty[b].n * s6;
        h->totB -= bb;
        h->totA += bb * s6;
      }
    free(ty);
  }
  h->phi = (double *) calloc(nsite > 0 ? nsite : 1, sizeof(double));
  h->evec = (double *) calloc(3 * (size_t) (nsite > 0 ? nsite : 1), sizeof(double));
  h->ljf = (double *) calloc(3 * (size_t) (nsite > 0 ? nsite : 1), sizeof(double));
  h->gr = (double *) calloc(3 * (size_t) (ngroup > 0 ? ngroup : 1), sizeof(double));
  return h;
fail:
  orc_eleclj_delete(h);
  return 0;
}

/* minimum-image shift of a displacement (include/pbc.h:16-23, 42-50) */
static void image_shift(const box_t *b, const double *v, double *dv)
{
  int d;
  for (d = 0; d < 3; d++) {
    const double L = b->l[d];
    dv[d] = -L * floor(v[d] * (1 / L) + 0.5);
  }
}

/* RSpaceEwald (src/rspace.c:382-558) */
static void rspace(elec_t *h, const double *r, double *lj_energy)
{
  const double rlo2 = sq(h->rc - h->c.smoothing_width), rhi2 = sq(h->rc);
  const int *mask = h->mask;
  pairctx pc;
  int ig, i;
  pc.q = h->q;
  pc.sig = h->sig;
  pc.eps = h->eps;
  pc.rscreen = h->rscreen;
  pc.phi = h->phi;
  pc.evec = h->evec;
  pc.ljf = h->ljf;
  pc.lj_energy = lj_energy;
  pc.geometric = h->c.geometric_combining_for_sigma;
  for (ig = 0; ig < h->ngroup; ig++) {
    const int is = h->group[2 * ig], ie = h->group[2 * ig + 1];
    int n;
    for (n = 0; n < h->nl->pairs->cnt[ig]; n++) {
      const int jg = h->nl->pairs->row[ig][n];
      const int js = h->group[2 * jg], je = h->group[2 * jg + 1];
      const int gx = pset_has(h->gexcl, ig, jg);
      double v[3], dv[3], r2, s = 1, ds = 0, tmps = 0, dsv[3] = {0, 0, 0};
      int smoothing = 0, k;
      for (k = 0; k < 3; k++)
        v[k] = r[3 * is + k] - r[3 * js + k];
      image_shift(&h->box, v, dv);
      for (k = 0; k < 3; k++)
        v[k] += dv[k];
      r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
      if (r2 > rhi2)
        continue;
      if (r2 > rlo2) {
        smoothing = 1;
        switch_fn(r2, rlo2, rhi2, &s, &ds);
        for (k = 0; k < 3; k++)
          dsv[k] = ds * v[k];
      }
      /* the anchor pair first, then every other site pair with the anchors' shift */
      for (i = is; i < ie; i++) {
        int j;
        for (j = js; j < je; j++) {
          const int m = mask[i] & mask[j];
          double d[3], rr;
          if (i == is && j == js) {
            if (gx && pset_has(h->excl, is, js))
              continue;
            d[0] = v[0];
            d[1] = v[1];
            d[2] = v[2];
            rr = r2;
          } else {
            if (!m)
              continue;
            if (gx && pset_has(h->excl, i, j))
              continue;
            for (k = 0; k < 3; k++)
              d[k] = (r[3 * i + k] + dv[k]) - r[3 * j + k];
            rr = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
          }
          if (m & HAS_Q)
            ewald_pair(&pc, i, j, d, rr, h->eta, h->cheb, smoothing, s, &tmps);
          if (m & HAS_LJ)
            lj_pair(&pc, i, j, d, rr, smoothing, s, &tmps, 0, 1);
        }
      }
      if (smoothing)
        for (k = 0; k < 3; k++) {
          h->ljf[3 * is + k] += dsv[k] * tmps;
          h->ljf[3 * js + k] -= dsv[k] * tmps;
        }
    }
  }
  /* excluded charged pairs: remove the reciprocal-space erf part
     (src/rspace.c:219-242, 492-521) */
  for (i = 0; i < h->nsite; i++) {
    int n;
    if (!(mask[i] & HAS_Q))
      continue;
    for (n = 0; n < h->excl->cnt[i]; n++) {
      const int j = h->excl->row[i][n];
      double v[3], dv[3], r2, rm, er, e, b0, b1;
      int k;
      if (!(mask[j] & HAS_Q))
        continue;
      for (k = 0; k < 3; k++)
        v[k] = r[3 * i + k] - r[3 * j + k];
      image_shift(&h->box, v, dv);
      for (k = 0; k < 3; k++)
        v[k] += dv[k];
      r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
      rm = sqrt(r2);
      er = h->eta * rm;
      e = exp(-sq(er));
      b0 = -erf(er) / rm;
      b1 = (b0 + h->eta * M_2_SQRTPI * e) / r2;
      coulomb_add(&pc, i, j, v, b0, b1);
    }
  }
  /* scaled 1-4 pairs (src/rspace.c:522-557) */
  if (h->p14) {
    const int se = fabs(h->c.elec_1_4_scale_factor - 1) > 1e-10;
    const int sl = fabs(h->c.lj_1_4_scale_factor - 1) > 1e-10;
    for (i = 0; i < h->nsite; i++) {
      int n;
      for (n = 0; n < h->p14->cnt[i]; n++) {
        const int j = h->p14->row[i][n];
        const int m = mask[i] & mask[j];
        double v[3], dv[3], r2;
        int k;
        for (k = 0; k < 3; k++)
          v[k] = r[3 * i + k] - r[3 * j + k];
        image_shift(&h->box, v, dv);
        for (k = 0; k < 3; k++)
          v[k] += dv[k];
        r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (m & HAS_Q)
          coulomb_plain(&pc, i, j, v, r2, se, h->c.elec_1_4_scale_factor - 1);
        if (m & HAS_LJ)
          lj_pair(&pc, i, j, v, r2, 0, 0, 0, sl, h->c.lj_1_4_scale_factor - 1);
      }
    }
  }
}

/* analytic LJ tail including the switched shell (src/eleclj.cpp:1247-1266) */
static double lj_tail(const elec_t *h)
{
  const double rhi = h->rc, rlo = rhi - h->c.smoothing_width;
  const double A = h->totA, B = h->totB;
  const double l2 = rlo * rlo, l3 = l2 * rlo, l4 = l3 * rlo, l5 = l4 * rlo, l6 = l5 * rlo, l7 = l6 * rlo,
               l9 = l7 * l2;
  const double h2 = rhi * rhi, h3 = h2 * rhi, h4 = h3 * rhi, h5 = h4 * rhi, h6 = h5 * rhi, h7 = h6 * rhi;
  return 2 * M_PI / box_volume(&h->box) *
         (A / (9 * l9) + B / (3 * l3) -
          (rhi - rlo) / (63 * h3 * l9 * pow(rhi + rlo, 5)) *
              (3 * B * h3 * l6 * (7 * h4 + 42 * h3 * rlo + 112 * h2 * l2 + 150 * rhi * l3 + 25 * l4) +
               A * (7 * h7 + 42 * h6 * rlo + 112 * h5 * l2 + 182 * h4 * l3 + 217 * h3 * l4 +
                    224 * h2 * l5 + 192 * rhi * l6 + 32 * l7)));
}

int orc_eleclj_eval(void *hp, const double *r, double *f, orc_energy *e,
                    double *phi_out, double *evec_out, double *ljf_out)
{
  elec_t *h = (elec_t *) hp;
  const int n = h->nsite;
  double lj_energy = 0, ljc = 0, elec = 0;
  int i, g, d;
  for (g = 0; g < h->ngroup; g++)
    for (d = 0; d < 3; d++)
      h->gr[3 * g + d] = r[3 * h->group[2 * g] + d];
  nbr_update(h->nl, h->gr);
  memset(h->phi, 0, sizeof(double) * n);
  memset(h->evec, 0, sizeof(double) * 3 * n);
  memset(h->ljf, 0, sizeof(double) * 3 * n);
  if (h->c.include_rspace)
    rspace(h, r, &lj_energy);
  if (h->any_q) {
    if (h->c.include_kspace) {
      if (h->p3m) {
        p3m_apply(h->p3m, r, h->q, h->phi, h->evec);
      } else {
        double rec[9];
        t_reciprocal(rec, h->latv);
        kspace_sum(h->c.kspace_cutoff, n, r, h->q, rec, box_volume(&h->box), h->eta, h->phi, h->evec);
      }
    }
    if (h->c.include_self) {
      /* self term and the neutralising background (src/eleclj.cpp:961-976) */
      const double a = h->eta * M_2_SQRTPI;
      double qs = 0;
      for (i = 0; i < n; i++) {
        qs += h->q[i];
        h->phi[i] -= a * h->q[i];
      }
      if (!almost_zero(qs)) {
        const double b = -M_PI / (sq(h->eta) * box_volume(&h->box)) * qs;
        for (i = 0; i < n; i++)
          h->phi[i] += b;
      }
    }
  }
  if (h->c.include_lj_correction) {
    ljc = lj_tail(h);
    lj_energy += ljc;
  }
  for (i = 0; i < n; i++)
    for (d = 0; d < 3; d++)
      f[3 * i + d] += h->q[i] * h->evec[3 * i + d] + h->ljf[3 * i + d];
  if (h->any_q) {
    for (i = 0; i < n; i++)
      elec += h->q[i] * h->phi[i];
    elec /= 2;
  }
  if (e) {
    e->elec = elec;
    e->lj = lj_energy;
    e->lj_correction = ljc;
    e->total = elec + lj_energy;
  }
  if (phi_out)
    memcpy(phi_out, h->phi, sizeof(double) * n);
  if (evec_out)
    memcpy(evec_out, h->evec, sizeof(double) * 3 * n);
  if (ljf_out)
    memcpy(ljf_out, h->ljf, sizeof(double) * 3 * n);
  return 0;
}

/* Potential at points (ElecLJ::electrostatic_potential_at_gridpoints,
   src/eleclj.cpp:1302-1340, periodic branch).  Real space as
   RSpaceEwaldPhiAtGridpoints (src/rspace.c:892-967): site minus point, minimum
   image, cut and switched on that distance, the site's own r_screen; k-space as
   kspace_phi (src/kspace.c:176-250) over points and sites with the points
   uncharged; the neutralising term for a charged system. */
int orc_eleclj_phi_at_points(void *hp, const double *r, int npoint, const double *pts, double *phi_out)
{
  elec_t *h = (elec_t *) hp;
  const int n = h->nsite, ntot = npoint + n;
  const double rlo2 = sq(h->rc - h->c.smoothing_width), rhi2 = sq(h->rc);
  double *p = (double *) calloc(ntot > 0 ? ntot : 1, sizeof(double));
  int i, j, d;
  if (h->c.include_rspace && h->cheb) {
    for (i = 0; i < n; i++) {
      if (!h->mask[i])
        continue;
      for (j = 0; j < npoint; j++) {
        double v[3], dv[3], r2, b0, b1;
        for (d = 0; d < 3; d++)
          v[d] = r[3 * i + d] - pts[3 * j + d];
        image_shift(&h->box, v, dv);
        for (d = 0; d < 3; d++)
          v[d] += dv[d];
        r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (r2 > rhi2)
          continue;
        if (h->cheb->min < r2 && r2 < h->cheb->max) {
          cheb_eval(h->cheb, r2, &b0, &b1);
        } else {
          const double rm = sqrt(r2);
          b0 = erfc(h->eta * rm) / rm;
        }
        if (r2 < sq(h->rscreen[i])) {
          const double rs = h->rscreen[i];
          b0 += (-0.5 * r2 * (1.0 / (rs * rs * rs)) + 1.5 / rs) - 1.0 / sqrt(r2);
        }
        if (r2 > rlo2) {
          const double z = (r2 - rlo2) / (rhi2 - rlo2);
          b0 *= ((-6 * z + 15) * z - 10) * z * z * z + 1;
        }
        p[j] += h->q[i] * b0;
      }
    }
  }
  if (h->c.include_kspace) {
    double rec[9];
    double *rt = (double *) malloc(sizeof(double) * 3 * (ntot > 0 ? ntot : 1));
    double *qt = (double *) calloc(ntot > 0 ? ntot : 1, sizeof(double));
    double *et = (double *) calloc(3 * (ntot > 0 ? ntot : 1), sizeof(double));
    memcpy(rt, pts, sizeof(double) * 3 * npoint);
    memcpy(rt + 3 * npoint, r, sizeof(double) * 3 * n);
    memcpy(qt + npoint, h->q, sizeof(double) * n);
    t_reciprocal(rec, h->latv);
    kspace_sum(h->c.kspace_cutoff, ntot, rt, qt, rec, box_volume(&h->box), h->eta, p, et);
    free(rt);
    free(qt);
    free(et);
  }
  if (h->c.include_self) {
    double qs = 0;
    for (i = 0; i < n; i++)
      qs += h->q[i];
    if (!almost_zero(qs)) {
      const double b = -M_PI / (sq(h->eta) * box_volume(&h->box)) * qs;
      for (j = 0; j < npoint; j++)
        p[j] += b;
    }
  }
  memcpy(phi_out, p, sizeof(double) * npoint);
  free(p);
  return 0;
}

double orc_eleclj_eta(void *hp) { return ((elec_t *) hp)->eta; }
double orc_eleclj_nlw(void *hp) { return ((elec_t *) hp)->nlw; }
void *orc_eleclj_nbrlist(void *hp) { return ((elec_t *) hp)->nl; }

void orc_eleclj_delete(void *hp)
{
  elec_t *h = (elec_t *) hp;
  if (!h)
    return;
  free(h->group);
  free(h->mask);
  free(h->q);
  free(h->sig);
  free(h->eps);
  free(h->rscreen);
  pset_free(h->excl);
  pset_free(h->gexcl);
  pset_free(h->p14);
  free(h->cheb);
  orc_p3m_delete(h->p3m);
  nbr_free(h->nl);
  free(h->phi);
  free(h->evec);
  free(h->ljf);
  free(h->gr);
  free(h);
}

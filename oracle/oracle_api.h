/*
 * Common C interface of the two CPU oracles (TEST INFRASTRUCTURE ONLY):
 *
 *   oracle/_build/liborc.so  — the oracle's own restatement of the reference
 *                              algorithm (oracle/mmnb_oracle.c, plain C);
 *   oracle/_ref/libref.so    — the reference's own sources (src/rspace.c,
 *                              src/pppm.c, src/kspace.c, src/cheby.c,
 *                              src/pbin.c, src/nbrlist.cpp, src/bcond.cpp …)
 *                              compiled unmodified and driven by
 *                              oracle/ref_harness.cpp.
 *
 * Both export exactly these symbols, so tests load either one through the
 * same Python wrapper (oracle/oracle.py) and compare them, and compare the GPU
 * library against them.  Nothing in the product links or loads either.
 *
 * Units follow the reference: lengths in Angstrom, energies in kcal/mol,
 * charges in the reference's internal unit sqrt(kcal A / mol)
 * (e_to_charge_unit, include/units.h:91-94).  Vectors are AoS double[3]
 * (cart_t, include/cart.h:9).  Lattice tensors use the reference's tensor_t
 * layout {xx, yx, zx, xy, yy, zy, xz, yz, zz} (include/cart.h:11): the three
 * lattice vectors are its columns.
 */
#ifndef ORACLE_API_H
#define ORACLE_API_H

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors the ElecLJ input fields on the hot path (include/eleclj.hpp:310-328,
   defaults src/eleclj.cpp:13-40). */
typedef struct {
  int bctype;                  /* enum bcondtype_t (include/bcondtype.h:8): 1 cubic, 2 orthorhombic */
  double box[3];               /* edge lengths; cubic uses box[0] */
  double rspace_cutoff;        /* 0 -> 0.45 * min diameter */
  double smoothing_width;      /* reference default 1 */
  double neighbor_list_width;  /* 0 -> 0.2 rc, clipped to 0.499 d - rc */
  double kspace_cutoff;        /* ordinary Ewald |n| cutoff (default 5) */
  double ewald_screening;      /* eta; < 0 -> automatic (ordinary Ewald only) */
  int use_p3m;
  double p3m_grid_spacing;
  int p3m_assignment_order;
  int p3m_alias_sum_limit;
  int p3m_ik_differentiate;
  int include_lj_correction;
  int geometric_combining_for_sigma;
  int include_rspace, include_kspace, include_self;
  double elec_1_4_scale_factor, lj_1_4_scale_factor;
} orc_config;

/* Energies of one evaluation, kcal/mol. */
typedef struct {
  double elec;           /* (q . phi) / 2  (src/eleclj.cpp:796-799) */
  double lj;             /* pair LJ + tail correction (lj_energy after recalculate_lj_correction) */
  double lj_correction;  /* analytic tail alone (src/eleclj.cpp:1247-1266) */
  double total;          /* elec + lj, what add_to_energy_and_forces adds to u */
} orc_energy;

/* Chebyshev erfc(eta r)/r table over r^2 (src/rspace.c:25-37, src/cheby.c:35-45).
   coeff receives 512*7 doubles. */
int orc_chebyshev(double rc, double eta, double *min, double *max, double *inv_dx, double *coeff);

/* Ordinary Ewald k-sum (src/kspace.c:35-174); latv is the direct lattice. */
int orc_kspace_field(double kspace_cutoff, int nsite, const double *r, const double *q,
                     const double latv[9], double eta, double *phi, double *evec, int *nk);

/* P3M (src/pppm.c:313-641). */
void *orc_p3m_new(int nsite, const double latv[9], double grid_spacing, int nalias,
                  int ik_differentiate, int assignment_order, double eta, int ngrid[3], double *chi);
void orc_p3m_field(void *p, const double *r, const double *q, double *phi, double *evec);
void orc_p3m_delete(void *p);

/* Group cell neighbour list (src/nbrlist.cpp). */
void *orc_nbrlist_new(int ngroup, double cutoff, double width, int bctype, const double box[3]);
int orc_nbrlist_update(void *h, const double *gr);      /* 1 if the list was rebuilt */
long orc_nbrlist_npairs(void *h);
void orc_nbrlist_pairs(void *h, int *pairs);            /* 2*npairs: row, entry as stored */
int orc_nbrlist_ncell(void *h);
void orc_nbrlist_cells(void *h, int *cell_of_group);    /* cells at the last rebuild */
long orc_nbrlist_ncellpairs(void *h);
void orc_nbrlist_cellpairs(void *h, int *pairs);
void orc_nbrlist_delete(void *h);

/* ElecLJ energy and forces for atom sites (src/eleclj.cpp:140-265, 643-807, 912-976, 1247-1266).
   group: 2*ngroup half-open site ranges.  excl: 2*nexcl site pairs (1-2 and 1-3).
   pairs14: 2*n14 site pairs.  q in internal charge units. */
void *orc_eleclj_new(const orc_config *c, int nsite, int ngroup, const int *group,
                     int nexcl, const int *excl, int n14, const int *pairs14,
                     const int *site_mask, const double *q, const double *sig,
                     const double *eps, const double *rscreen);
/* f is ADDED to (3*nsite); phi, evec, ljf are overwritten when non-null. */
int orc_eleclj_eval(void *h, const double *r, double *f, orc_energy *e,
                    double *phi, double *evec, double *ljf);
double orc_eleclj_eta(void *h);
double orc_eleclj_nlw(void *h);
void *orc_eleclj_nbrlist(void *h);
/* Electrostatic potential of the sites at r at npoint points (3*npoint), written
   to phi[npoint] (ElecLJ::electrostatic_potential_at_gridpoints,
   src/eleclj.cpp:1302-1340, periodic branch). */
int orc_eleclj_phi_at_points(void *h, const double *r, int npoint, const double *pts, double *phi);
void orc_eleclj_delete(void *h);

/* Pair-set semantics (src/pbin.c:41-137): add the 2*nadd pairs in order, sort
   and dedupe the rows, then report each row (cnt[i] entries in rows[i*n ...])
   and the n*n membership matrix. */
int orc_pairset_demo(int n, int nadd, const int *adds, int *cnt, int *rows, int *exists);

#ifdef __cplusplus
}
#endif

#endif

/*
 * mmnb.h — C ABI of libmmnb, the sm_100a implementation of msim's nonbonded
 * force path: real-space Ewald erfc-Coulomb + Lennard-Jones over a GPU-built
 * cell neighbour list, and the P3M / ordinary-Ewald reciprocal space.
 *
 * One handle is one ElecLJ potential (include/eleclj.hpp:303-397 in the
 * reference) bound to one CUDA device and one stream.  Plain C types only:
 * pointers, sizes and int status codes, so any FFI can bind it.
 *
 * What each entry point replaces in the reference:
 *
 *   mmnb_create / mmnb_set_params   ElecLJ::init, types_changed, set_lambda
 *                                   (src/eleclj.cpp:140-265, 273-319, 328-580)
 *                                   and the set-up halves of the C kernels:
 *                                   RSpaceChebyshev_new (include/rspace.h:17),
 *                                   p3m_new + p3m_init (include/pppm.h:12-35),
 *                                   kspace_new (include/kspace.h:11),
 *                                   NeighborList::NeighborList +
 *                                   set_boundary_conditions (include/nbrlist.hpp:15-18)
 *   mmnb_compute                    ElecLJ::add_to_energy_and_forces, i.e.
 *                                   Potential::add_to_energy_and_forces
 *                                   (include/pot.hpp:12, src/eleclj.cpp:785-807),
 *                                   which runs NeighborList::coordinates_changed,
 *                                   RSpaceEwald (include/rspace.h:19-34),
 *                                   p3m_field (include/pppm.h:52-56) or
 *                                   kspace_field (include/kspace.h:14-15),
 *                                   calc_self_phi and the LJ tail
 *   mmnb_scale                      ElecLJ::scale + p3m_scale (src/eleclj.cpp:1268-1280,
 *                                   include/pppm.h:60)
 *   mmnb_destroy                    ElecLJ::cleanup, p3m_delete, kspace_delete
 *
 * Conventions are the reference's: Angstrom, kcal/mol, charges in
 * sqrt(kcal A / mol) (e_to_charge_unit, include/units.h:91-94); vectors are AoS
 * double[3] (cart_t, include/cart.h:9).  Forces are ADDED to the caller's
 * array and the energy is ADDED to *u, as Potential::add_to_energy_and_forces
 * does; the caller zeroes them (src/mdyn.cpp:151-153).
 *
 * Where the reference calls die() or an assertion, these functions return a
 * nonzero status and leave the handle usable; mmnb_last_error() explains.
 */
#ifndef MMNB_H
#define MMNB_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define MMNB_OK 0
#define MMNB_ERR_ARG 1          /* bad argument (sizes, ranges, null pointers) */
#define MMNB_ERR_CUDA 2         /* a CUDA or cuFFT call failed */
#define MMNB_ERR_UNSUPPORTED 3  /* option this build does not provide */
#define MMNB_ERR_CUTOFF 4       /* rspace_cutoff > 0.49 * minimum box diameter,
                                   or smoothing_width >= cutoff (src/eleclj.cpp:168-182) */
#define MMNB_ERR_OVERFLOW 5     /* neighbour rows outgrew their capacity after a retry */
#define MMNB_ERR_STATE 6        /* call out of order (e.g. compute before set_params) */
#define MMNB_ERR_TIMEOUT 7      /* a bounded device-side wait gave up */
#define MMNB_ERR_DEVICE 8       /* a device-side check failed (index or size out of range) */

/* precision forms */
#define MMNB_FP64 0   /* FP64 throughout; matches the reference to ~1e-12 relative */
#define MMNB_MIXED 1  /* FP32 pair and spline math, 64-bit fixed-point force
                         accumulation, FP64 energies, self terms and influence function */

/* boundary conditions: enum bcondtype_t values (include/bcondtype.h:8) */
#define MMNB_CUBIC 1
#define MMNB_ORTHORHOMBIC 2

/* site flags (include/rspace.h:7-8) */
#define MMNB_SITE_HAS_Q 1
#define MMNB_SITE_HAS_LJ 2

typedef struct mmnb_handle mmnb_handle;

/* ElecLJ's hot-path input fields (include/eleclj.hpp:310-328); defaults from
   mmnb_config_init are the reference's (src/eleclj.cpp:13-40). */
typedef struct mmnb_config {
  int precision;                 /* MMNB_FP64 or MMNB_MIXED */
  int bctype;                    /* MMNB_CUBIC or MMNB_ORTHORHOMBIC */
  double box[3];                 /* edge lengths (A); cubic reads box[0] */
  double rspace_cutoff;          /* 0 -> 0.45 * minimum diameter */
  double smoothing_width;        /* 1 */
  double neighbor_list_width;    /* 0 -> 0.2 rc, clipped to 0.499 d - rc */
  double kspace_cutoff;          /* 5 (ordinary Ewald |n| cutoff) */
  double ewald_screening;        /* -1 -> automatic: sqrt(pi kc / (rc d)) for the
                                    k-sum; with P3M the value that minimises the
                                    summed squares of the real-space and mesh error
                                    estimates (src/pppm.c:666-716) */
  int use_p3m;                   /* 0 */
  double p3m_grid_spacing;       /* 0.5 */
  int p3m_assignment_order;      /* 3; 2..7 */
  int p3m_alias_sum_limit;       /* 2 */
  int p3m_ik_differentiate;      /* 0 */
  int include_lj_correction;     /* 1 */
  int geometric_combining_for_sigma; /* 0 */
  int include_rspace;            /* 1 */
  int include_kspace;            /* 1 */
  int include_self;              /* 1 */
  double elec_1_4_scale_factor;  /* 1 */
  double lj_1_4_scale_factor;    /* 1 */
  int rebuild_interval;          /* 0: rebuild on the reference's displacement
                                    criterion (src/nbrlist.cpp:51-77); k > 0: also
                                    force a rebuild every k-th evaluation */
  int device;                    /* CUDA ordinal, -1 = current */
  double p3m_grid_density;       /* -1; > 0: mesh spacing = minimum diameter /
                                    cbrt(density * volume), and p3m_grid_spacing
                                    must keep its default (src/eleclj.cpp:195-200) */
} mmnb_config;

/* Energies of the last evaluation (kcal/mol), as ElecLJ::write reports them
   (src/eleclj.cpp:1026-1150). */
typedef struct mmnb_energy {
  double elec;            /* (q . phi) / 2 */
  double lj;              /* pair LJ + tail correction */
  double lj_correction;   /* tail alone */
  double total;           /* elec + lj: what is added to u */
} mmnb_energy;

/* Fill *c with the reference's defaults. */
int mmnb_config_init(mmnb_config *c);

/* Create a potential for nsite sites in ngroup groups.
   group: 2*ngroup ints, half-open site ranges [a, b) of each group; the first
          site of a group is its anchor (src/eleclj.cpp:654-681, 778-779).
   excl:  2*nexcl site pairs excluded from the pair sum (1-2 and 1-3 pairs,
          src/eleclj.cpp:712-724), either order, duplicates allowed.
   pairs14: 2*n14 site pairs for the scaled 1-4 terms; read only when a 1-4
          scale factor differs from 1 (src/eleclj.cpp:726-747). */
int mmnb_create(const mmnb_config *c, int nsite, int ngroup, const int *group,
                int nexcl, const int *excl, int n14, const int *pairs14,
                mmnb_handle **out);

/* Per-site parameters: mask bits MMNB_SITE_HAS_Q / MMNB_SITE_HAS_LJ, charge
   (internal unit), LJ sigma (A) and epsilon (kcal/mol), short-range
   screening radius (A, 0 = none).  Replaces ElecLJ::set_lambda's per-site
   interpolation output (src/eleclj.cpp:279-308). */
int mmnb_set_params(mmnb_handle *h, const int *site_mask, const double *q,
                    const double *sig, const double *eps, const double *rscreen);

/* One evaluation from HOST arrays.
   r: 3*nsite site positions.  f: 3*nsite, forces ADDED (may be NULL).
   u: energy ADDED (may be NULL).  e, phi (nsite), evec (3*nsite): optional
   outputs of this evaluation (NULL to skip). */
int mmnb_compute(mmnb_handle *h, const double *r, double *f, double *u,
                 mmnb_energy *e, double *phi, double *evec);

/* One evaluation on DEVICE arrays, asynchronous on the handle's stream:
   d_r (3*nsite) positions, d_f (3*nsite) forces ADDED, d_energy (4 doubles,
   mmnb_energy layout) overwritten.  Any of d_f / d_energy may be NULL.
   Launches only; no host synchronisation, so it can be captured in a CUDA graph
   once the handle has done one mmnb_compute (first-call set-up). */
int mmnb_compute_device(mmnb_handle *h, const double *d_r, double *d_f, double *d_energy);

/* Capture one mmnb_compute_device(h, d_r, d_f, d_energy) into a CUDA graph on
   the handle's stream (which must be a non-default stream, see
   mmnb_set_stream); mmnb_graph_launch replays it.  The graph reads d_r and
   writes d_f / d_energy at the addresses given here, and it keeps the
   device-side rebuild test, so replaying it is exactly one more evaluation.
   Call after the handle's first evaluation; capture again after mmnb_scale,
   mmnb_set_params or anything that reallocates (a neighbour-row overflow). */
int mmnb_graph_capture(mmnb_handle *h, const double *d_r, double *d_f, double *d_energy);
int mmnb_graph_launch(mmnb_handle *h);

/* Volume move by factor s: box, eta /= s, Chebyshev table, influence function
   and cell stencil follow (src/eleclj.cpp:1268-1280, src/pppm.c:643-664).
   MMNB_ERR_CUTOFF, with the handle unchanged, when the scaled box would no
   longer hold the cutoff (rc > 0.49 x smallest edge, ElecLJ::init's rule,
   src/eleclj.cpp:168-182) or rc + neighbour-list width would reach half of it. */
int mmnb_scale(mmnb_handle *h, double s);

/* Bind the handle to a CUDA stream (cudaStream_t passed as void*). */
int mmnb_set_stream(mmnb_handle *h, void *stream);

/* Neighbour list of the last rebuild, for parity checks against
   NeighborList (src/nbrlist.cpp:222-251):
   the unordered group pairs {i, j} of the reference's PairBinary, each once,
   written as (i, j) with i < j.  *npairs receives the count; pairs (2*cap ints)
   may be NULL to query the count. */
int mmnb_get_pairlist(mmnb_handle *h, long *npairs, int *pairs, long cap);

/* Cell of each group at the last rebuild, in the reference's numbering
   (ix*n + iy)*n + iz (src/nbrlist.cpp:79-82, 228-234). */
int mmnb_get_cells(mmnb_handle *h, int *cell_of_group, int *ncell_per_dim);

/* Number of list rebuilds so far and number of evaluations. */
int mmnb_get_counters(mmnb_handle *h, long *rebuilds, long *evaluations);

/* Status of the evaluations since the last check, for callers that evaluate
   on device arrays (mmnb_compute_device, mmnb_graph_launch and graphs of their
   own): synchronises the handle's stream.  The reference has no such state --
   its neighbour rows grow on the host as they fill (src/pbin.c:41-50) and its
   errors call die() -- so this reports, after the fact, what the device path
   met:
     MMNB_ERR_OVERFLOW  evaluations (their number in *truncated) ran on
                        neighbour rows cut at their capacity, so pairs were
                        missing; the rows are regrown and the next evaluation
                        rebuilds the list.  Graphs captured before hold the old
                        rows: mmnb_graph_launch refuses them until captured
                        again, and the MD integrators capture again themselves;
     MMNB_ERR_DEVICE    a site coordinate was not finite (NaN or infinite);
     MMNB_OK            neither.
   max_row receives the longest row needed.  Both conditions are cleared.
   mmnb_compute checks them itself (it grows the rows and evaluates again, or
   returns MMNB_ERR_DEVICE without adding to f or u); mmnb_md_run and
   mmnb_md_batch_run return this status for their runs. */
int mmnb_check(mmnb_handle *h, long *truncated, int *max_row);

/* Number of this library's kernels launched on the handle's stream so far
   (library kernels such as cuFFT's are not counted). */
int mmnb_get_launches(mmnb_handle *h, long *launches);

/* Derived settings: rc, neighbour-list width, eta, P3M mesh (0 if unused). */
int mmnb_get_settings(mmnb_handle *h, double *rc, double *nlw, double *eta, int mesh[3]);

/* The dimensionless RMS force error estimates ElecLJ::init reports
   (src/eleclj.cpp:129-138, 225, 233-243): real space 2 / sqrt(rc / V^(1/3))
   exp(-(rc eta)^2) (0 without real space), and reciprocal space -- with P3M the
   mesh estimate p3m_init computes beside the influence function
   (src/pppm.c:313-393), for the k-sum eta l / pi sqrt(8 / kc)
   exp(-(pi kc / (eta l))^2), l = V^(1/3) (0 without k-space). */
int mmnb_get_error_estimates(mmnb_handle *h, double *rspace, double *kspace);

/* Stage timing with CUDA events on the handle's stream.  mmnb_set_timing
   clears the record and turns it on or off; while on, every evaluation
   records one event per stage.  mmnb_get_timing synchronises the stream and
   writes each stage's mean device time per evaluation (ms) into ms[0..nmax)
   and the stage names, comma-separated, into names (size cap); it returns the
   number of stages (negative status on error). */
int mmnb_set_timing(mmnb_handle *h, int on);
int mmnb_get_timing(mmnb_handle *h, double *ms, int nmax, char *names, int cap);

int mmnb_destroy(mmnb_handle *h);

const char *mmnb_last_error(const mmnb_handle *h);
const char *mmnb_status_string(int status);

/* The erfc(eta r)/r table the FP64 pair kernel reads: 512 segments over r^2,
   built with the reference's formula (src/rspace.c:25-37, src/cheby.c:7-45).
   coeff receives 512*7 doubles. */
int mmnb_chebyshev_table(double rc, double eta, double *min, double *max,
                         double *inv_dx, double *coeff);

/* Mesh size P3M chooses along a lattice vector of length a (src/pppm.c:277-292,
   429-431). */
int mmnb_p3m_mesh_size(double a, double grid_spacing);

/* Ordinary Ewald reciprocal-space potential and field, ADDED to d_phi (nsite)
   and d_evec (3*nsite), for callers that cannot allocate device memory — a
   host that has reserved all device memory for its own pool, or a loop that
   must not let an allocation or free synchronise the device.  It allocates
   nothing: positions d_r (3*nsite), charges d_q and both outputs are the
   caller's device arrays, and the only scratch is a fixed array inside the
   library, one per device for the life of the process, holding at most 4096
   wave vectors (|n| <= about 12); a larger kspace_cutoff returns MMNB_ERR_ARG
   with an explanation in mmnb_last_error(NULL).  The first call on a device
   looks up that array's device address; make that first call before any
   stream capture.  All calls on a device share the array and overwrite it, so
   calls that overlap on the GPU race.  bctype MMNB_CUBIC (box[0]) or
   MMNB_ORTHORHOMBIC; stream is a cudaStream_t or NULL.  The launches are
   asynchronous on that stream.  This entry point has no counterpart in the
   reference: it is the computation of kspace_field without kspace_new. */
int mmnb_kspace_field_noalloc(int nsite, const double *d_r, const double *d_q, int bctype,
                              const double box[3], double eta, double kspace_cutoff,
                              double *d_phi, double *d_evec, void *stream);

/* FP32 FMA throughput of a GPU (TFLOP/s), measured by timing independent FMA
   chains over the whole device; the denominator of the pair kernels'
   roofline.  No counterpart in the reference.  device < 0: the current one. */
int mmnb_measure_fp32_peak(int device, double *tflops);

/* ---- launch tuning ---------------------------------------------------------
   No counterpart in the reference (its path is one CPU thread).  Launch
   choices that change no result: tuning[0] = register budget of the
   rigid-water pair kernel as resident warps per SM / 4 (4: 128 registers,
   5: 96), tuning[1] = layout
   of the mixed P3M charge assignment (0: a thread per site, 1: a thread per
   site and mesh x-plane, 2 (default): a lane per site and mesh z-offset, so
   the lanes of a site reduce into consecutive mesh words),
   tuning[2] = P3M mesh work on a second stream beside the pair kernels (1) or
   in line (0), tuning[3] = warps per block of the FP64 rigid-water kernel
   (12, 10 or 8; fewer are launched when its rings and the box's erfc table do
   not fit in shared memory).  mmnb_autotune times each choice over `iters` graph replays of
   an evaluation at r (host array) and keeps the fastest; small systems gain
   most.  It evaluates at r (advancing the rebuild counters); a graph captured
   with mmnb_graph_capture before tuning keeps the old choices. */
int mmnb_autotune(mmnb_handle *h, const double *r, int iters);
int mmnb_get_tuning(mmnb_handle *h, int tuning[4]);
int mmnb_set_tuning(mmnb_handle *h, const int tuning[4]);

/* ---- adjoint --------------------------------------------------------------
   Per-site parameter gradients, for the force-field fits the reference runs
   through WeakCouple::update and BCIFit (src/msimprog.cpp:855-876,
   src/bcifit.cpp:44-123) on the per-type parameters ElecLJ::types_changed maps
   to sites (src/eleclj.cpp:440-503): a type's gradient is the sum of its
   sites' gradients (times dq_site/dq_type where charges are tied).

   mmnb_forward evaluates at r as mmnb_compute does with the site fields
   requested (f and u ADDED when non-NULL, e when non-NULL) and keeps on the device what the gradients of this
   evaluation need: the site potentials and fields.  It replaces the forward
   pass of a fit; the backward does not evaluate again.

   mmnb_site_gradients then returns, for that evaluation, per site i:
     du_dq[i]   = dU/dq_i, the site potential (0 on sites without charge);
     du_dsig[i] = dU/dsigma_i, du_deps[i] = dU/depsilon_i (0 on sites without
                  LJ; LJ tail correction included, differentiated as a smooth
                  function of the sites' sigma and epsilon);
   and, given dl_df = dL/dF (3*nsite) of a loss of the forces the forward
   returned, the same three for L:
     dl_dq[i] = sum_k dl_df_k . dF_k/dq_i, dl_dsig[i], dl_deps[i].
   dL/dq_i = g_i . E_i plus the potential at site i of the dipoles
   p_j = q_j g_j (g = dl_df) and the switch and exclusion terms; the dipoles
   need a second reciprocal-space solve (P3M mesh or Ewald sum), FP64 in both
   precisions.  With the mixed form the gradients carry the forward's field
   error (~1e-5 relative).  Any output may be NULL; with dl_df NULL the dl_*
   outputs are left untouched.  MMNB_ERR_STATE unless the last evaluation of
   the handle was mmnb_forward's (any other evaluation, mmnb_set_params or
   mmnb_scale in between clears it). */
int mmnb_forward(mmnb_handle *h, const double *r, double *f, double *u, mmnb_energy *e);
int mmnb_site_gradients(mmnb_handle *h, const double *dl_df, double *du_dq, double *du_dsig, double *du_deps,
                        double *dl_dq, double *dl_dsig, double *dl_deps);

/* Gradients with respect to uniform scales of all charges, all LJ sigmas and
   all LJ epsilons (each at 1): mmnb_forward at r, then mmnb_site_gradients
   contracted with the site parameters, grad_u[k] = sum_i p_i dU/dp_i.
   grad_u[3]: dU/d(scales).  dl_df (3*nsite, may be NULL) is dL/dF of a loss of
   the forces; grad_l[3] (may be NULL) receives sum_i dl_df_i . dF_i/d(scales). */
int mmnb_backward(mmnb_handle *h, const double *r, const double *dl_df, double *f, double *u,
                  double grad_u[3], double grad_l[3]);

/* ---- virial ----------------------------------------------------------------
   One evaluation at r (forces ADDED to f, energy ADDED to u, breakdown in e;
   each may be NULL) and w = dU/ds at s = 1 along the path of the reference's
   volume moves: MSys::scale (src/msys.cpp:416-421) translates every molecule
   rigidly so its centre of mass is multiplied by s and scales the box, and
   ElecLJ::scale (src/eleclj.cpp:1268-1280) divides eta and, through p3m_scale
   (src/pppm.c:643-664), the influence function by s, keeping rc, the switch and
   the mesh counts -- the path mmnb_scale follows.  The reference has no virial;
   MSimProgram::test_scale (src/msimprog.cpp:379-400) evaluates the energy on
   both sides of one such step.  dU/dV = w / (3 V), so the molecular pressure is
   P = (N_mol k T - w / 3) / V.
   Molecules: nmol half-open site ranges mol[2m], mol[2m+1] covering every site
   once; site_mass (nsite): the masses that define their centres.  FP64 sums on
   the GPU in a fixed order.  MMNB_ERR_UNSUPPORTED for screened charges. */
int mmnb_virial(mmnb_handle *h, const double *r, int nmol, const int *mol, const double *site_mass, double *f,
                double *u, mmnb_energy *e, double *w);

/* ---- potential at points ---------------------------------------------------
   Electrostatic potential of the sites at r (3*nsite, host) at npoint points
   (3*npoint, host), written to phi[npoint] in the units of mmnb_compute's phi
   (the reference's internal potential unit; potential_unit_to_hartree_e,
   include/units.h:106-109, converts it to atomic units for printing, as
   ElecLJ::write_electrostatic_potential_at_gridpoints does).
   Replaces ElecLJ::electrostatic_potential_at_gridpoints
   (src/eleclj.cpp:1302-1340, periodic boxes): real space as
   RSpaceEwaldPhiAtGridpoints (src/rspace.c:892-967, site-point distance cut at
   rc and switched), the ordinary Ewald k-sum over kspace_cutoff wave vectors as
   kspace_phi (src/kspace.c:176-250) whether or not the handle uses P3M for
   forces, and the neutralising term when the sites carry net charge; each
   term follows include_rspace / include_kspace / include_self.  Brute force over
   sites x points, like the reference; allocates and frees its own scratch. */
int mmnb_phi_at_points(mmnb_handle *h, const double *r, int npoint, const double *points, double *phi);

/* ---- molecular dynamics on the device ------------------------------------
   Velocity Verlet with rigid 3-site water, replacing the MD loop of
   MDyn::run (src/mdyn.cpp:142-160: half kick, drift, constrain positions,
   forces, half kick, constrain velocities) and the ConstraintGroup
   SHAKE/RATTLE solves it calls (src/constraint.cpp:295-358), whose converged
   results SETTLE (positions) and a 3 x 3 velocity solve give in closed form.
   Units as the reference's: A, ps, kcal/mol, masses in g/mol / 418.4
   (include/units.h:161-168).  One step is a CUDA graph on the handle's
   stream (forces from mmnb_compute_device of h). */
typedef struct mmnb_md mmnb_md;

/* site_mass: nsite masses (reference mass units).  rigid_water: every group
   is [O, H, H] (sites 3g..3g+2) constrained to O-H = r_oh and H-O-H =
   hoh_angle_deg; 0 integrates without constraints.  dt in ps. */
int mmnb_md_create(mmnb_handle *h, const double *site_mass, double dt, int rigid_water, double r_oh,
                   double hoh_angle_deg, mmnb_md **out);
/* Host positions and velocities (3*nsite each; v may be NULL for zero).
   Velocities are projected onto the constraints and the forces evaluated. */
int mmnb_md_set_state(mmnb_md *md, const double *r, const double *v);
/* nsteps steps; energies (3*nsteps: kinetic, potential, conserved per step)
   may be NULL.  Returns mmnb_check's status for the run: MMNB_ERR_OVERFLOW
   when a neighbour row outgrew its capacity during the run (the rows are
   regrown, so running again from a saved state gives complete rows),
   MMNB_ERR_DEVICE for a non-finite coordinate. */
int mmnb_md_run(mmnb_md *md, int nsteps, double *energies);
int mmnb_md_get_state(mmnb_md *md, double *r, double *v);
const char *mmnb_md_last_error(const mmnb_md *md);
int mmnb_md_destroy(mmnb_md *md);
/* Multiply the velocities by factor (a temperature swap of replica exchange
   rescales them by sqrt(T_new / T_old)). */
int mmnb_md_scale_velocities(mmnb_md *md, double factor);

/* Replica batch: n integrators (each on its own handle and stream, after
   mmnb_md_set_state) advanced together, one CUDA graph launch per step with
   an independent branch per replica, so replicas of uneven size share the
   GPU.  Replaces the one-process-per-replica layout of MDyn's replica
   exchange (src/mdyn.cpp:317-351, one MPI rank per replica); the exchange
   itself (energies from the logs, temperature swaps) is the caller's.
   energies: n host arrays of 3*nsteps (kinetic, potential, conserved per
   step), or NULL; any entry may be NULL. */
typedef struct mmnb_md_batch mmnb_md_batch;
int mmnb_md_batch_create(mmnb_md *const *mds, int n, mmnb_md_batch **out);
int mmnb_md_batch_run(mmnb_md_batch *b, int nsteps, double *const *energies);
const char *mmnb_md_batch_last_error(const mmnb_md_batch *b);
int mmnb_md_batch_destroy(mmnb_md_batch *b);

#ifdef __cplusplus
}
#endif

#endif /* MMNB_H */

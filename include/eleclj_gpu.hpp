/*
 * eleclj_gpu.hpp -- ElecLJ on libmmnb: the msim Potential whose nonbonded
 * force path (real-space Ewald + LJ over the neighbour list, P3M or the Ewald
 * k-sum) runs on the GPU through the C ABI of include/mmnb.h.
 *
 * A maintainer adds this header to the reference tree and constructs an
 * ElecLJGpu wherever an ElecLJ is constructed; MDyn::run, MSimProgram, FEP,
 * CheckGradients and MMin keep calling Potential::add_to_energy_and_forces
 * (include/pot.hpp:12).  ElecLJ::init still does all the host work -- types,
 * sites, groups, exclusions, eta, the P3M mesh choice -- and this class hands
 * the results to the library.
 *
 * Two edits to the reference's include/eleclj.hpp come with it:
 *   - the label `private:` of class ElecLJ (include/eleclj.hpp:361) becomes
 *     `protected:`, so this subclass reads the site arrays (nsite, q, sig, eps,
 *     rscreen, site_mask, r, site, group, excluded, one_four) and the values
 *     init resolved (rc, nlw, eta);
 *   - electrostatic_potential_at_gridpoints (include/eleclj.hpp:357) is
 *     declared virtual, so ESPFit and MSimProgram reach the override below.
 *
 * Status codes from the library replace the reference's die()/insist exits;
 * this class maps a nonzero status back to die() (src/util.c:11-26), so msim
 * behaves as before.  Bond charge increments (ElecLJ::update_q) iterate on the
 * host over the site potentials and are not offered here: init dies if the
 * parameters define any.
 */
#ifndef ELECLJ_GPU_HPP
#define ELECLJ_GPU_HPP

#include <cmath>
#include <vector>

#include "eleclj.hpp"
#include "mmnb.h"
#include "pbin.h"
#include "util.h"

class ElecLJGpu : public ElecLJ
{
public:
  // MMNB_MIXED (FP32 pair math, fixed-point sums) or MMNB_FP64 (the
  // reference's arithmetic, results to ~1e-12)
  int precision;
  // refresh ElecLJ's electric_field() and site potentials on every evaluation
  // (the general pair kernels then run instead of the rigid-water ones)
  bool keep_fields;

  ElecLJGpu() : precision(MMNB_MIXED), keep_fields(false), h(0) { }
  ~ElecLJGpu() { release(); }

  void init(MSys *m)
  {
    ElecLJ::init(m);
    release();
    if (any_bci)
      die("ElecLJGpu::init: bond charge increments are solved on the host; use ElecLJ");
    const BoundaryConditions &bc = *msys->boundary_conditions;
    if (bc.type != cubic && bc.type != orthorhombic)
      die("ElecLJGpu::init: cubic and orthorhombic boundary conditions only");
    mmnb_config c;
    mmnb_config_init(&c);
    c.precision = precision;
    c.bctype = bc.type == cubic ? MMNB_CUBIC : MMNB_ORTHORHOMBIC;
    const Tensor a = bc.lattice_vectors();
    c.box[0] = a.xx;
    c.box[1] = a.yy;
    c.box[2] = a.zz;
    // the values ElecLJ::init resolved (src/eleclj.cpp:164-239)
    c.rspace_cutoff = rc;
    c.smoothing_width = smoothing_width;
    c.neighbor_list_width = nlw;
    c.kspace_cutoff = kspace_cutoff;
    c.ewald_screening = eta;
    c.use_p3m = use_p3m;
    c.p3m_grid_spacing = p3m_grid_density > 0 ? bc.min_diameter() / cbrt(p3m_grid_density * bc.volume())
                                              : p3m_grid_spacing;
    c.p3m_assignment_order = p3m_assignment_order;
    c.p3m_alias_sum_limit = p3m_alias_sum_limit;
    c.p3m_ik_differentiate = p3m_ik_differentiate;
    c.include_lj_correction = include_lj_correction;
    c.geometric_combining_for_sigma = geometric_combining_for_sigma;
    c.include_rspace = include_rspace;
    c.include_kspace = include_kspace;
    c.include_self = include_self;
    c.elec_1_4_scale_factor = elec_1_4_scale_factor;
    c.lj_1_4_scale_factor = lj_1_4_scale_factor;
    const std::vector<int> excl = pair_rows(excluded, nsite), p14 = pair_rows(one_four, nsite);
    std::vector<int> grp(2 * (size_t) ngroup);
    for (int g = 0; g < ngroup; g++) {
      grp[2 * g] = group[g].a;
      grp[2 * g + 1] = group[g].b;
    }
    if (mmnb_create(&c, nsite, ngroup, grp.data(), (int) excl.size() / 2, excl.data(), (int) p14.size() / 2,
                    p14.data(), &h) != MMNB_OK)
      die("ElecLJGpu::init: %s", mmnb_last_error(0));
    set_params();
  }

  // per-site q, sigma, epsilon, screening radius and mask after ElecLJ has
  // (re)computed them (types_changed, set_lambda: src/eleclj.cpp:273-580)
  void set_params()
  {
    if (h && mmnb_set_params(h, (const int *) site_mask, (const double *) q, (const double *) sig,
                             (const double *) eps, (const double *) rscreen) != MMNB_OK)
      die("ElecLJGpu::set_params: %s", mmnb_last_error(h));
  }

  void types_changed()
  {
    ElecLJ::types_changed();
    set_params();
  }

  void types_changed(const MSys &perturbed)
  {
    ElecLJ::types_changed(perturbed);
    set_params();
  }

  void set_lambda(double lambda)
  {
    ElecLJ::set_lambda(lambda);
    set_params();
  }

  // volume move (ElecLJ::scale, src/eleclj.cpp:1268-1280)
  void scale(double s)
  {
    ElecLJ::scale(s);
    if (h && mmnb_scale(h, s) != MMNB_OK)
      die("ElecLJGpu::scale: %s", mmnb_last_error(h));
  }

  // Potential::add_to_energy_and_forces: forces and energy ADDED, as
  // ElecLJ::add_to_energy_and_forces does (src/eleclj.cpp:785-807)
  void add_to_energy_and_forces(double &u, Cartesian *f)
  {
    for (int i = 0; i < nsite; i++)
      r[i] = site[i]->position(msys->atom);
    fs.assign(3 * (size_t) nsite, 0.0);
    mmnb_energy e;
    if (mmnb_compute(h, (const double *) r, fs.data(), &u, &e, keep_fields ? (double *) phi : 0,
                     keep_fields ? (double *) evec : 0) != MMNB_OK)
      die("ElecLJGpu::add_to_energy_and_forces: %s", mmnb_last_error(h));
    for (int i = 0; i < nsite; i++)
      site[i]->apply_force(msys->atom, f, Cartesian(fs[3 * i], fs[3 * i + 1], fs[3 * i + 2]));
    elec_energy = e.elec;
    lj_energy = e.lj;
    lj_correction = e.lj_correction;
  }

  // add_to_energy_and_forces through mmnb_forward: the same energy and forces,
  // and the site potentials and fields stay on the device for site_gradients
  // (the forward pass of a parameter fit; the backward does not evaluate again)
  void forward(double &u, Cartesian *f)
  {
    for (int i = 0; i < nsite; i++)
      r[i] = site[i]->position(msys->atom);
    fs.assign(3 * (size_t) nsite, 0.0);
    mmnb_energy e;
    if (mmnb_forward(h, (const double *) r, fs.data(), &u, &e) != MMNB_OK)
      die("ElecLJGpu::forward: %s", mmnb_last_error(h));
    for (int i = 0; i < nsite; i++)
      site[i]->apply_force(msys->atom, f, Cartesian(fs[3 * i], fs[3 * i + 1], fs[3 * i + 2]));
    elec_energy = e.elec;
    lj_energy = e.lj;
    lj_correction = e.lj_correction;
  }

  // mmnb_site_gradients for the last forward(): per site dU/dq (charge units),
  // dU/dsigma, dU/depsilon and, given dL/dF per SITE (3*nsite, or 0; for sites
  // that are atoms this is dL/dF of the atom), the same three for the loss L.
  // Any output may be 0.
  void site_gradients(const double *dl_df, double *du_dq, double *du_dsig, double *du_deps, double *dl_dq,
                      double *dl_dsig, double *dl_deps)
  {
    if (mmnb_site_gradients(h, dl_df, du_dq, du_dsig, du_deps, dl_dq, dl_dsig, dl_deps) != MMNB_OK)
      die("ElecLJGpu::site_gradients: %s", mmnb_last_error(h));
  }

  // the gradient with respect to one type's parameter, as types_changed maps
  // fixed_charge, sigma and epsilon to the sites of that type
  // (src/eleclj.cpp:440-503): the sum over the sites whose type1 is `type`;
  // multiply a charge sum by e_to_charge_unit(1) for d/d(charge in e)
  double type_sum(const char *type, const double *site_grad) const
  {
    double s = 0;
    for (int i = 0; i < nsite; i++)
      if (site[i]->type1 == Str(type))
        s += site_grad[i];
    return s;
  }

  // ElecLJ::electrostatic_potential_at_gridpoints (src/eleclj.cpp:1302-1340),
  // periodic boxes: the potential at each grid point; p also holds the sites'
  // entries after the points, as the reference's does
  void electrostatic_potential_at_gridpoints(const CVec gp, DVec &p)
  {
    for (int i = 0; i < nsite; i++)
      r[i] = site[i]->position(msys->atom);
    p.resize(gp.size() + nsite);
    p.zero();
    if (mmnb_phi_at_points(h, (const double *) r, gp.size(), (const double *) gp, (double *) p) != MMNB_OK)
      die("ElecLJGpu::electrostatic_potential_at_gridpoints: %s", mmnb_last_error(h));
  }

private:
  mmnb_handle *h;
  std::vector<double> fs;

  // the pairs of a PairBinary over n sites as a flat list of site indices
  // (each unordered pair once, in whichever row PairBinary keeps it:
  // src/pbin.c:6, 41-50)
  static std::vector<int> pair_rows(const struct PairBinary *pb, int n)
  {
    std::vector<int> out;
    if (!pb)
      return out;
    const int *nn = PairBinary_number_of_elements(pb);
    int *const *t = PairBinary_elements(pb);
    for (int i = 0; i < n; i++)
      for (int k = 0; k < nn[i]; k++) {
        out.push_back(i);
        out.push_back(t[i][k]);
      }
    return out;
  }

  void release()
  {
    if (h)
      mmnb_destroy(h);
    h = 0;
  }
};

#endif /* ELECLJ_GPU_HPP */

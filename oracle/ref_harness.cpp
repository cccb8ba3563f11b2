/*
 * Reference harness — TEST INFRASTRUCTURE ONLY.
 *
 * Drives the reference's own, unmodified sources (compiled from where they lie
 * by oracle/Makefile into oracle/_ref/libref.so) through the common oracle
 * interface in oracle/oracle_api.h.  The numerical work is all reference code:
 *   RSpaceChebyshev_new / RSpaceEwald    src/rspace.c:25-37, 382-558
 *   p3m_new / p3m_init / p3m_field       src/pppm.c:313-641 (FFT via oracle/shim)
 *   kspace_new / kspace_field            src/kspace.c:35-174
 *   NeighborList                         src/nbrlist.cpp:9-251
 *   PairBinary                           src/pbin.c
 *   BoundaryConditions                   src/bcond.cpp:22-67, 189-190
 * What this file adds is the ElecLJ orchestration for atom sites, restated
 * from src/eleclj.cpp (that class needs the whole MSys/Atom/HTab/param-file
 * stack, which this harness does not build):
 *   init                     src/eleclj.cpp:140-265 (cutoff, nlw, eta, P3M / Ewald set-up)
 *   init_sites exclusions    src/eleclj.cpp:712-770
 *   set_lambda totA / totB   src/eleclj.cpp:273-308
 *   add_to_energy_and_forces src/eleclj.cpp:785-807
 *   calc_phi_evec_lj         src/eleclj.cpp:912-959
 *   calc_self_phi            src/eleclj.cpp:961-976
 *   recalculate_lj_correction src/eleclj.cpp:1247-1266
 */
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "rspace.h"
#include "cheby.h"
#include "kspace.h"
#include "pppm.h"
#include "pbin.h"
#include "fns.h"
#include "bcond.hpp"
/* The harness reads the list's cell bookkeeping for parity checks; the
   class layout is unchanged by widening access. */
#define private public
#include "nbrlist.hpp"
#undef private

#include "oracle_api.h"

static double sqr(double x) { return x * x; }

static BoundaryConditions *make_bc(int bctype, const double box[3])
{
  if (bctype == cubic)
    return BoundaryConditions::new_cubic(box[0]);
  if (bctype == orthorhombic)
    return BoundaryConditions::new_orthorhombic(Cartesian(box[0], box[1], box[2]));
  return 0;
}

extern "C" {

int orc_chebyshev(double rc, double eta, double *min, double *max, double *inv_dx, double *coeff)
{
  struct Chebyshev *t = RSpaceChebyshev_new(rc, eta, 0, 0);
  *min = t->min;
  *max = t->max;
  *inv_dx = t->inv_dx;
  memcpy(coeff, t->coeff, sizeof(t->coeff));
  free(t);
  return 0;
}

int orc_kspace_field(double kspace_cutoff, int nsite, const double *r, const double *q,
                     const double latv[9], double eta, double *phi, double *evec, int *nk)
{
  /* ElecLJ passes the reciprocal lattice and the volume (src/eleclj.cpp:949-950). */
  const Tensor a = *(const Tensor *) latv;
  const Tensor recip = (2 * M_PI) * a.inverse().transpose();
  const double volume = fabs(a.determinant());
  struct kspace *k = kspace_new(kspace_cutoff, nsite);
  kspace_field(k, (const cart_t *) r, q, (const tensor_t *) &recip, volume, eta, phi, (cart_t *) evec);
  if (nk)
    *nk = kspace_number_of_wavevectors(k);
  kspace_delete(k);
  return 0;
}

void *orc_p3m_new(int nsite, const double latv[9], double grid_spacing, int nalias,
                  int ik_differentiate, int assignment_order, double eta, int ngrid[3], double *chi)
{
  p3m_t p = p3m_new(nsite, latv, grid_spacing, nalias, ik_differentiate, assignment_order, ngrid);
  double c = 0;
  p3m_init(p, eta, &c);
  if (chi)
    *chi = c;
  return p;
}

void orc_p3m_field(void *p, const double *r, const double *q, double *phi, double *evec)
{
  p3m_field((p3m_t) p, r, q, phi, evec);
}

void orc_p3m_delete(void *p)
{
  p3m_delete((p3m_t) p);
}

struct RefNbr {
  NeighborList *nl;
  BoundaryConditions *bc;
  int n;
};

void *orc_nbrlist_new(int ngroup, double cutoff, double width, int bctype, const double box[3])
{
  RefNbr *h = new RefNbr;
  h->n = ngroup;
  h->bc = make_bc(bctype, box);
  h->nl = new NeighborList(ngroup, cutoff, width);
  h->nl->set_boundary_conditions(*h->bc);
  return h;
}

static int nbr_update(NeighborList *nl, int n, const double *gr)
{
  const int was_first = nl->first_time;
  std::vector<double> before(3 * (size_t) n);
  for (int i = 0; i < n; i++) {
    before[3 * i] = nl->last[i].x;
    before[3 * i + 1] = nl->last[i].y;
    before[3 * i + 2] = nl->last[i].z;
  }
  CVec r(n);
  for (int i = 0; i < n; i++)
    r[i] = Cartesian(gr[3 * i], gr[3 * i + 1], gr[3 * i + 2]);
  nl->coordinates_changed(r);
  if (was_first)
    return 1;
  for (int i = 0; i < n; i++)
    if (nl->last[i].x != before[3 * i] || nl->last[i].y != before[3 * i + 1] ||
        nl->last[i].z != before[3 * i + 2])
      return 1;
  return 0;
}

int orc_nbrlist_update(void *hp, const double *gr)
{
  RefNbr *h = (RefNbr *) hp;
  return nbr_update(h->nl, h->n, gr);
}

static long pb_count(const struct PairBinary *p, int n)
{
  const int *nn = PairBinary_number_of_elements(p);
  long s = 0;
  for (int i = 0; i < n; i++)
    s += nn[i];
  return s;
}

static void pb_dump(const struct PairBinary *p, int n, int *out)
{
  const int *nn = PairBinary_number_of_elements(p);
  int *const *t = PairBinary_elements(p);
  long k = 0;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < nn[i]; j++) {
      out[2 * k] = i;
      out[2 * k + 1] = t[i][j];
      k++;
    }
}

long orc_nbrlist_npairs(void *hp)
{
  RefNbr *h = (RefNbr *) hp;
  return pb_count(h->nl->p, h->n);
}

void orc_nbrlist_pairs(void *hp, int *pairs)
{
  RefNbr *h = (RefNbr *) hp;
  pb_dump(h->nl->p, h->n, pairs);
}

int orc_nbrlist_ncell(void *hp)
{
  return ((RefNbr *) hp)->nl->ncell;
}

void orc_nbrlist_cells(void *hp, int *cell_of_group)
{
  RefNbr *h = (RefNbr *) hp;
  NeighborList *nl = h->nl;
  for (int i = 0; i < h->n; i++)
    cell_of_group[i] = -1;
  for (int c = 0; c < nl->ncell3; c++)
    for (int k = nl->cell_head[c]; k != -1; k = nl->cell_list[k])
      cell_of_group[k] = c;
}

long orc_nbrlist_ncellpairs(void *hp)
{
  RefNbr *h = (RefNbr *) hp;
  return pb_count(h->nl->cell, h->nl->ncell3);
}

void orc_nbrlist_cellpairs(void *hp, int *pairs)
{
  RefNbr *h = (RefNbr *) hp;
  pb_dump(h->nl->cell, h->nl->ncell3, pairs);
}

void orc_nbrlist_delete(void *hp)
{
  RefNbr *h = (RefNbr *) hp;
  delete h->nl;
  delete h->bc;
  delete h;
}

struct RefElecLJ {
  orc_config c;
  int nsite, ngroup;
  std::vector<int> group;           /* 2*ngroup */
  std::vector<int> site_mask;
  std::vector<double> q, sig, eps, rscreen;
  BoundaryConditions *bc;
  Tensor latv;
  double rc, nlw, eta, totA, totB;
  bool any_q, any_lj;
  struct PairBinary *excluded, *group_excluded, *one_four;
  struct Chebyshev *cheb;
  struct kspace *kspace;
  p3m_t p3m;
  RefNbr nbr;
  std::vector<double> phi, evec, ljf;
};

void *orc_eleclj_new(const orc_config *c, int nsite, int ngroup, const int *group,
                     int nexcl, const int *excl, int n14, const int *pairs14,
                     const int *site_mask, const double *q, const double *sig,
                     const double *eps, const double *rscreen)
{
  RefElecLJ *h = new RefElecLJ;
  h->c = *c;
  h->nsite = nsite;
  h->ngroup = ngroup;
  h->group.assign(group, group + 2 * ngroup);
  h->site_mask.assign(site_mask, site_mask + nsite);
  h->q.assign(q, q + nsite);
  h->sig.assign(sig, sig + nsite);
  h->eps.assign(eps, eps + nsite);
  h->rscreen.assign(rscreen, rscreen + nsite);
  h->bc = make_bc(c->bctype, c->box);
  if (!h->bc) {
    delete h;
    return 0;
  }
  h->latv = h->bc->lattice_vectors();
  h->any_q = h->any_lj = false;
  for (int i = 0; i < nsite; i++) {
    if (site_mask[i] & SITE_HAS_Q)
      h->any_q = true;
    if (site_mask[i] & SITE_HAS_LJ)
      h->any_lj = true;
  }
  /* src/eleclj.cpp:164-188 */
  const double min_diameter = h->bc->min_diameter();
  h->rc = c->rspace_cutoff;
  if (is_almost_zero(h->rc))
    h->rc = 0.45 * min_diameter;
  if (h->rc > 0.49 * min_diameter || !(h->rc > 0) || c->smoothing_width >= h->rc) {
    delete h->bc;
    delete h;
    return 0;
  }
  h->nlw = c->neighbor_list_width;
  if (is_almost_zero(h->nlw)) {
    h->nlw = 0.2 * h->rc;
    if (h->rc + h->nlw >= 0.5 * min_diameter)
      h->nlw = 0.499 * min_diameter - h->rc;
  }
  h->nbr.n = ngroup;
  h->nbr.bc = h->bc->copy();
  h->nbr.nl = new NeighborList(ngroup, h->rc, h->nlw);
  h->nbr.nl->set_boundary_conditions(*h->bc);
  /* src/eleclj.cpp:189-262 */
  h->eta = c->ewald_screening;
  h->kspace = 0;
  h->p3m = 0;
  h->cheb = 0;
  if (h->any_q) {
    if (c->include_kspace && c->use_p3m) {
      int ngrid[3];
      double kerr = 0;
      h->p3m = p3m_new(nsite, (const double *) &h->latv, c->p3m_grid_spacing, c->p3m_alias_sum_limit,
                       c->p3m_ik_differentiate, c->p3m_assignment_order, ngrid);
      if (h->eta < 0) {
        /* p3m_optimize needs GSL, which the oracle does not provide */
        p3m_delete(h->p3m);
        delete h->nbr.nl;
        delete h->nbr.bc;
        delete h->bc;
        delete h;
        return 0;
      }
      p3m_init(h->p3m, h->eta, &kerr);
    } else {
      if (h->eta < 0)
        h->eta = sqrt((M_PI * c->kspace_cutoff) / (h->rc * min_diameter));
      if (c->include_kspace)
        h->kspace = kspace_new(c->kspace_cutoff, nsite);
    }
    if (c->include_rspace)
      h->cheb = RSpaceChebyshev_new(h->rc, h->eta, 0, 0);
  }
  /* Exclusions and group exclusions, src/eleclj.cpp:712-724, 748-770 */
  h->excluded = PairBinary_new(nsite);
  for (int k = 0; k < nexcl; k++)
    PairBinary_add(h->excluded, excl[2 * k], excl[2 * k + 1]);
  PairBinary_init(h->excluded);
  h->one_four = 0;
  if (!are_approximately_equal(c->elec_1_4_scale_factor, 1) ||
      !are_approximately_equal(c->lj_1_4_scale_factor, 1)) {
    h->one_four = PairBinary_new(nsite);
    for (int k = 0; k < n14; k++)
      PairBinary_add(h->one_four, pairs14[2 * k], pairs14[2 * k + 1]);
    PairBinary_init(h->one_four);
  }
  std::vector<int> group_for_site(nsite, -1);
  for (int g = 0; g < ngroup; g++)
    for (int k = group[2 * g]; k < group[2 * g + 1]; k++)
      group_for_site[k] = g;
  h->group_excluded = PairBinary_new(ngroup);
  {
    const int *nn = PairBinary_number_of_elements(h->excluded);
    int *const *t = PairBinary_elements(h->excluded);
    for (int i = 0; i < nsite; i++)
      for (int k = 0; k < nn[i]; k++) {
        const int ig = group_for_site[i], jg = group_for_site[t[i][k]];
        if (ig != jg)
          PairBinary_add(h->group_excluded, ig, jg);
      }
  }
  PairBinary_init(h->group_excluded);
  /* LJ tail totals, src/eleclj.cpp:283-308: sites are binned by their
     (sigma, epsilon) printed with %12.6g and read back. */
  std::map<std::string, int> se;
  for (int i = 0; i < nsite; i++) {
    if (!(site_mask[i] & SITE_HAS_LJ))
      continue;
    char key[128];
    snprintf(key, 128, "%12.6g %12.6g", sig[i], eps[i]);
    se[key]++;
  }
  h->totA = h->totB = 0;
  for (std::map<std::string, int>::const_iterator ti = se.begin(); ti != se.end(); ++ti) {
    double si, ei;
    sscanf(ti->first.c_str(), "%lf%lf", &si, &ei);
    for (std::map<std::string, int>::const_iterator tj = se.begin(); tj != se.end(); ++tj) {
      double sj, ej;
      sscanf(tj->first.c_str(), "%lf%lf", &sj, &ej);
      const double s6 = pow(c->geometric_combining_for_sigma ? sqrt(si * sj) : 0.5 * (si + sj), 6);
      const double b = 4 * sqrt(ei * ej) * ti->second * tj->second * s6;
      h->totB -= b;
      h->totA += b * s6;
    }
  }
  h->phi.assign(nsite, 0.0);
  h->evec.assign(3 * (size_t) nsite, 0.0);
  h->ljf.assign(3 * (size_t) nsite, 0.0);
  return h;
}

int orc_eleclj_eval(void *hp, const double *r, double *f, orc_energy *e,
                    double *phi_out, double *evec_out, double *ljf_out)
{
  RefElecLJ *h = (RefElecLJ *) hp;
  const orc_config &c = h->c;
  const int nsite = h->nsite, ngroup = h->ngroup;
  /* coordinates_changed, src/eleclj.cpp:773-783 */
  std::vector<double> gr(3 * (size_t) ngroup);
  for (int g = 0; g < ngroup; g++)
    for (int d = 0; d < 3; d++)
      gr[3 * g + d] = r[3 * h->group[2 * g] + d];
  nbr_update(h->nbr.nl, ngroup, gr.data());
  /* calc_phi_evec_lj, src/eleclj.cpp:912-959 */
  std::fill(h->phi.begin(), h->phi.end(), 0.0);
  std::fill(h->evec.begin(), h->evec.end(), 0.0);
  std::fill(h->ljf.begin(), h->ljf.end(), 0.0);
  double lj_energy = 0;
  double *phi = h->phi.data();
  cart_t *evec = (cart_t *) h->evec.data();
  cart_t *ljf = (cart_t *) h->ljf.data();
  if (c.include_rspace)
    RSpaceEwald(nsite, ngroup, (const int(*)[2]) h->group.data(), (const cart_t *) r,
                h->bc->type, (const tensor_t *) &h->latv,
                h->nbr.nl->neighbors(), h->nbr.nl->number_of_neighbors(),
                h->group_excluded, h->excluded,
                sqr(h->rc - c.smoothing_width), sqr(h->rc),
                h->site_mask.data(), h->q.data(), phi, evec, h->eta, h->cheb, h->rscreen.data(),
                h->sig.data(), h->eps.data(), c.geometric_combining_for_sigma,
                &lj_energy, ljf, h->one_four, c.elec_1_4_scale_factor, c.lj_1_4_scale_factor);
  if (h->any_q) {
    if (c.include_kspace) {
      if (h->p3m) {
        p3m_field(h->p3m, r, h->q.data(), phi, (double *) evec);
      } else {
        const Tensor recip = h->bc->reciprocal_lattice_vectors();
        kspace_field(h->kspace, (const cart_t *) r, h->q.data(), (const tensor_t *) &recip,
                     h->bc->volume(), h->eta, phi, evec);
      }
    }
    if (c.include_self) {
      /* calc_self_phi, src/eleclj.cpp:961-976 */
      const double a = h->eta * M_2_SQRTPI;
      double qsum = 0;
      for (int i = 0; i < nsite; i++) {
        qsum += h->q[i];
        phi[i] -= a * h->q[i];
      }
      if (!is_almost_zero(qsum)) {
        const double b = -M_PI / (sqr(h->eta) * h->bc->volume()) * qsum;
        for (int i = 0; i < nsite; i++)
          phi[i] += b;
      }
    }
  }
  /* recalculate_lj_correction, src/eleclj.cpp:1247-1266 */
  double lj_correction = 0;
  if (c.include_lj_correction) {
    const double rhi = h->rc;
    const double rlo = rhi - c.smoothing_width;
    const double rlo2 = rlo * rlo, rlo3 = rlo2 * rlo, rlo4 = rlo3 * rlo;
    const double rlo5 = rlo4 * rlo, rlo6 = rlo5 * rlo, rlo7 = rlo6 * rlo, rlo9 = rlo7 * rlo2;
    const double rhi2 = rhi * rhi, rhi3 = rhi2 * rhi, rhi4 = rhi3 * rhi, rhi5 = rhi4 * rhi;
    const double rhi6 = rhi5 * rhi, rhi7 = rhi6 * rhi;
    const double totA = h->totA, totB = h->totB;
    lj_correction = 2 * M_PI / h->bc->volume() *
      (totA / (9 * rlo9) + totB / (3 * rlo3) -
       (rhi - rlo) / (63 * rhi3 * rlo9 * pow(rhi + rlo, 5)) *
       (3 * totB * rhi3 * rlo6 * (7 * rhi4 + 42 * rhi3 * rlo + 112 * rhi2 * rlo2 + 150 * rhi * rlo3 + 25 * rlo4) +
        totA * (7 * rhi7 + 42 * rhi6 * rlo + 112 * rhi5 * rlo2 +
                182 * rhi4 * rlo3 + 217 * rhi3 * rlo4 + 224 * rhi2 * rlo5 + 192 * rhi * rlo6 + 32 * rlo7)));
    lj_energy += lj_correction;
  }
  /* add_to_energy_and_forces, src/eleclj.cpp:794-805 */
  for (int i = 0; i < nsite; i++)
    for (int d = 0; d < 3; d++)
      f[3 * i + d] += h->q[i] * h->evec[3 * i + d] + h->ljf[3 * i + d];
  double elec = 0;
  if (h->any_q) {
    for (int i = 0; i < nsite; i++)
      elec += h->q[i] * phi[i];
    elec /= 2;
  }
  if (e) {
    e->elec = elec;
    e->lj = lj_energy;
    e->lj_correction = lj_correction;
    e->total = elec + lj_energy;
  }
  if (phi_out)
    memcpy(phi_out, phi, sizeof(double) * nsite);
  if (evec_out)
    memcpy(evec_out, h->evec.data(), sizeof(double) * 3 * nsite);
  if (ljf_out)
    memcpy(ljf_out, h->ljf.data(), sizeof(double) * 3 * nsite);
  return 0;
}

/* ElecLJ::electrostatic_potential_at_gridpoints, periodic branch
   (src/eleclj.cpp:1302-1340), with the reference's own RSpaceEwaldPhiAtGridpoints
   and kspace_new/kspace_phi over points + sites (the points carry no charge). */
int orc_eleclj_phi_at_points(void *hp, const double *r, int npoint, const double *pts, double *phi_out)
{
  RefElecLJ *h = (RefElecLJ *) hp;
  const orc_config &c = h->c;
  const int nsite = h->nsite, ntot = npoint + nsite;
  std::vector<double> p(ntot, 0.0);
  if (c.include_rspace)
    RSpaceEwaldPhiAtGridpoints(nsite, npoint, (const cart_t *) r, (const cart_t *) pts, h->bc->type,
                               (const tensor_t *) &h->latv, sqr(h->rc - c.smoothing_width), sqr(h->rc),
                               h->site_mask.data(), h->q.data(), p.data(), h->eta, h->cheb, h->rscreen.data());
  if (c.include_kspace) {
    std::vector<double> qtot(ntot, 0.0), rtot(3 * (size_t) ntot);
    memcpy(rtot.data(), pts, sizeof(double) * 3 * npoint);
    memcpy(rtot.data() + 3 * (size_t) npoint, r, sizeof(double) * 3 * nsite);
    for (int i = 0; i < nsite; i++)
      qtot[npoint + i] = h->q[i];
    struct kspace *ks = kspace_new(c.kspace_cutoff, ntot);
    const Tensor recip = h->bc->reciprocal_lattice_vectors();
    kspace_phi(ks, (const cart_t *) rtot.data(), qtot.data(), (const tensor_t *) &recip, h->bc->volume(), h->eta,
               p.data());
    kspace_delete(ks);
  }
  if (c.include_self) {
    double qsum = 0;
    for (int i = 0; i < nsite; i++)
      qsum += h->q[i];
    if (!is_almost_zero(qsum)) {
      const double b = -M_PI / (sqr(h->eta) * h->bc->volume()) * qsum;
      for (int i = 0; i < npoint; i++)
        p[i] += b;
    }
  }
  memcpy(phi_out, p.data(), sizeof(double) * npoint);
  return 0;
}

double orc_eleclj_eta(void *hp) { return ((RefElecLJ *) hp)->eta; }
double orc_eleclj_nlw(void *hp) { return ((RefElecLJ *) hp)->nlw; }
void *orc_eleclj_nbrlist(void *hp) { return &((RefElecLJ *) hp)->nbr; }

void orc_eleclj_delete(void *hp)
{
  RefElecLJ *h = (RefElecLJ *) hp;
  if (h->p3m)
    p3m_delete(h->p3m);
  if (h->kspace)
    kspace_delete(h->kspace);
  if (h->cheb)
    free(h->cheb);
  PairBinary_delete(h->excluded);
  PairBinary_delete(h->group_excluded);
  if (h->one_four)
    PairBinary_delete(h->one_four);
  delete h->nbr.nl;
  delete h->nbr.bc;
  delete h->bc;
  delete h;
}

int orc_pairset_demo(int n, int nadd, const int *adds, int *cnt, int *rows, int *exists)
{
  struct PairBinary *p = PairBinary_new(n);
  for (int i = 0; i < nadd; i++)
    PairBinary_add(p, adds[2 * i], adds[2 * i + 1]);
  PairBinary_init(p);
  const int *nn = PairBinary_number_of_elements(p);
  int *const *t = PairBinary_elements(p);
  for (int i = 0; i < n; i++) {
    cnt[i] = nn[i];
    for (int j = 0; j < nn[i] && j < n; j++)
      rows[i * n + j] = t[i][j];
    for (int j = 0; j < n; j++)
      exists[i * n + j] = PairBinary_exists(p, i, j);
  }
  PairBinary_delete(p);
  return 0;
}

} /* extern "C" */

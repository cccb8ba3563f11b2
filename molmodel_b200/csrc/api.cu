// libmmnb C ABI: handle life cycle, host-side set-up that mirrors ElecLJ::init
// (src/eleclj.cpp:140-265), and the per-evaluation launch sequence that
// mirrors ElecLJ::add_to_energy_and_forces (src/eleclj.cpp:785-807).

#include <atomic>

#include "mmnb_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <set>
#include <string>
#include <tuple>
#include <vector>

using namespace mmnb;

namespace {

thread_local std::string g_create_error;

int fail(mmnb_handle *h, int code, const std::string &msg)
{
  if (h)
    h->err = msg;
  else
    g_create_error = msg;
  return code;
}

#define CK(call)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return fail(h, MMNB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));           \
  } while (0)

#define CKFFT(call)                                                                                \
  do {                                                                                             \
    cufftResult r_ = (call);                                                                       \
    if (r_ != CUFFT_SUCCESS)                                                                       \
      return fail(h, MMNB_ERR_CUDA, std::string(#call) + ": cufft error " + std::to_string(r_));   \
  } while (0)

double sq(double x) { return x * x; }

// 64 machine epsilons, the reference's is_almost_zero (src/fns.c:8-31)
bool almost_zero(double x) { return fabs(x) < 64 * 2.220446049250313e-16; }

// Cubic Chebyshev fit of g(r^2) on segment i, the reference's construction
// (src/cheby.c:7-45: 50 nodes, coefficients turned into a power series in the
// position inside the segment), then the derivative coefficients.
template <typename F>
void chebyshev_fit(int i, double r2min, double dx, F g_of_r2, double *o)
{
  const double a = i * dx + r2min, b = (i + 1) * dx + r2min;
  double g[50], c[4];
  const double fac = 2.0 / 50;
  const double bma = 0.5 * (b - a), bpa = 0.5 * (b + a);
  for (int k = 0; k < 50; k++)
    g[k] = g_of_r2(cos(M_PI * (k + 0.5) / 50) * bma + bpa);
  for (int j = 0; j < 4; j++) {
    double s = 0;
    for (int k = 0; k < 50; k++)
      s += g[k] * cos(M_PI * j * (k + 0.5) / 50);
    c[j] = fac * s;
  }
  o[0] = c[0] / 2 - c[1] + c[2] - c[3];
  o[1] = 2 * c[1] - 8 * c[2] + 18 * c[3];
  o[2] = 8 * c[2] - 48 * c[3];
  o[3] = 32 * c[3];
  o[4] = -2 * o[1] / (b - a);
  o[5] = -2 * 2 * o[2] / (b - a);
  o[6] = -2 * 3 * o[3] / (b - a);
}

// Segment i of the reference's erfc(eta r)/r table (src/rspace.c:18-37), same
// formula and operation order: built on the host so segments 0..511 are
// bitwise the ones RSpaceChebyshev_new builds.  Segments past 511 continue the
// same construction beyond the reference's range (the rigid-water FP64 kernel
// reads them for site pairs beyond 1.2 rc^2).
void chebyshev_segment(int i, double r2min, double dx, double eta, double *o)
{
  chebyshev_fit(i, r2min, dx, [eta](double r2) { const double r = sqrt(r2); return erfc(eta * r) / r; }, o);
}

void chebyshev_table(double rhi, double eta, double *mn, double *mx, double *inv_dx, double *coeff7)
{
  const double r2max = 1.2 * sq(rhi);
  const double r2min = r2max > 4 ? 4 : 0.9 * r2max;
  const double dx = (r2max - r2min) / kCheb;
  *mn = r2min;
  *mx = r2max;
  *inv_dx = 1.0 / dx;
  for (int i = 0; i < kCheb; i++)
    chebyshev_segment(i, r2min, dx, eta, coeff7 + 7 * i);
}

// nearest 2^a 3^b 5^c 7^d; ties keep the first found (src/pppm.c:277-292)
int near_2357(double x)
{
  int best = 1;
  double bestdiff = fabs(x - 1);
  for (int p2 = 1; p2 <= x; p2 *= 2)
    for (int p3 = p2; p3 <= x; p3 *= 3)
      for (int p5 = p3; p5 <= x; p5 *= 5)
        for (int p7 = p5; p7 <= x; p7 *= 7) {
          const double diff = fabs(x - p7);
          if (diff < bestdiff) {
            bestdiff = diff;
            best = p7;
          }
        }
  return best;
}

unsigned spread_bits(unsigned v)
{
  v &= 0x3ff;
  v = (v | (v << 16)) & 0x030000ff;
  v = (v | (v << 8)) & 0x0300f00f;
  v = (v | (v << 4)) & 0x030c30c3;
  v = (v | (v << 2)) & 0x09249249;
  return v;
}

template <typename T>
int dalloc(mmnb_handle *h, T **p, size_t n)
{
  h->buf_gen++;
  if (*p) {
    cudaFree(*p);
    *p = nullptr;
  }
  cudaError_t e = cudaMalloc((void **) p, sizeof(T) * (n > 0 ? n : 1));
  if (e != cudaSuccess)
    return fail(h, MMNB_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  return MMNB_OK;
}

template <typename T>
int upload(mmnb_handle *h, T **p, const std::vector<T> &v)
{
  int s = dalloc(h, p, v.size());
  if (s)
    return s;
  if (!v.empty())
    CK(cudaMemcpy(*p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  return MMNB_OK;
}

// per-row sorted unique CSR from a pair list, both directions
void build_csr(int n, const std::vector<std::pair<int, int>> &pairs, std::vector<int> &ptr, std::vector<int> &idx)
{
  std::vector<std::vector<int>> rows(n);
  for (auto &p : pairs) {
    if (p.first == p.second)
      continue;
    rows[p.first].push_back(p.second);
    rows[p.second].push_back(p.first);
  }
  ptr.assign(n + 1, 0);
  idx.clear();
  for (int i = 0; i < n; i++) {
    auto &r = rows[i];
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    ptr[i + 1] = ptr[i] + (int) r.size();
    idx.insert(idx.end(), r.begin(), r.end());
  }
}

// Cell geometry and stencil (src/nbrlist.cpp:9-17, 84-123).  The reference
// pairs cell ia with ib = ia + j (mod n) for every half-space offset j with
// |j_k| <= nmax; as unordered pairs that is the set of wrapped offsets +-j.
// Offsets whose cells cannot hold two anchors closer than cutoff + width are
// dropped (anchors sit within half a cell of their cell's lattice point, so
// along each axis they are at least (|d| - 1) cells apart); the pairs such
// cells would contribute all fail the distance test, so the list is unchanged.
int setup_cells(mmnb_handle *h)
{
  const int n = (int) floor(cbrt(h->ngroup / 2 + 3));
  CellGeom &cg = h->cg;
  cg.n = n;
  for (int d = 0; d < 3; d++)
    cg.lc[d] = h->box.L[d] * (1.0 / n);
  const double cut = h->rc + h->nlw;
  cg.c2 = sq(cut);
  h->ncell3 = n * n * n;
  // reference half stencil
  double maxdiam;
  if (h->cfg.bctype == MMNB_CUBIC)
    maxdiam = sqrt(3.0) * cg.lc[0];
  else
    maxdiam = sqrt(cg.lc[0] * cg.lc[0] + cg.lc[1] * cg.lc[1] + cg.lc[2] * cg.lc[2]);
  const double vol = fabs(cg.lc[0] * cg.lc[1] * cg.lc[2]);
  const double a01 = sqrt(sq(cg.lc[0] * cg.lc[1])), a02 = sqrt(sq(cg.lc[0] * cg.lc[2])),
               a12 = sqrt(sq(cg.lc[1] * cg.lc[2]));
  const double mindiam = vol / std::max(std::max(a01, a02), a12);
  const double c2cell = sq(cut + maxdiam);
  const int nmax = std::min((int) ceil((cut + maxdiam) / mindiam), n / 2 + 1);
  std::set<std::tuple<int, int, int>> full;
  for (int jx = 0; jx <= nmax; jx++)
    for (int jy = (jx == 0 ? 0 : -nmax); jy <= nmax; jy++)
      for (int jz = (jx == 0 && jy == 0 ? 1 : -nmax); jz <= nmax; jz++) {
        double v[3] = {cg.lc[0] * jx, cg.lc[1] * jy, cg.lc[2] * jz};
        for (int d = 0; d < 3; d++)
          v[d] -= cg.lc[d] * floor(v[d] * (1 / cg.lc[d]) + 0.5);
        if (!(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] < c2cell))
          continue;
        for (int sgn = -1; sgn <= 1; sgn += 2) {
          const int dx = ((sgn * jx) % n + n) % n, dy = ((sgn * jy) % n + n) % n, dz = ((sgn * jz) % n + n) % n;
          if (dx || dy || dz)
            full.insert(std::make_tuple(dx, dy, dz));
        }
      }
  const double margin = 1e-6 * std::min(std::min(h->box.L[0], h->box.L[1]), h->box.L[2]) + 1e-12;
  std::vector<std::pair<double, std::tuple<int, int, int>>> kept;
  for (auto &t : full) {
    const int dd[3] = {std::get<0>(t), std::get<1>(t), std::get<2>(t)};
    double lb2 = 0;
    for (int d = 0; d < 3; d++) {
      const int m = std::min(dd[d], n - dd[d]);
      const double gap = std::max(m - 1, 0) * cg.lc[d];
      lb2 += gap * gap;
    }
    if (sqrt(lb2) <= cut + margin)
      kept.push_back(std::make_pair(lb2, t));
  }
  std::stable_sort(kept.begin(), kept.end(),
                   [](const std::pair<double, std::tuple<int, int, int>> &a,
                      const std::pair<double, std::tuple<int, int, int>> &b) { return a.first < b.first; });
  std::vector<int> st;
  st.push_back(0);
  st.push_back(0);
  st.push_back(0);
  for (auto &k : kept) {
    st.push_back(std::get<0>(k.second));
    st.push_back(std::get<1>(k.second));
    st.push_back(std::get<2>(k.second));
  }
  h->nstencil = (int) st.size() / 3;
  int s;
  if ((s = upload(h, &h->d_stencil, st)))
    return s;
  // Morton order of cells
  std::vector<std::pair<unsigned, int>> codes(h->ncell3);
  for (int ix = 0; ix < n; ix++)
    for (int iy = 0; iy < n; iy++)
      for (int iz = 0; iz < n; iz++) {
        const int c = (ix * n + iy) * n + iz;
        codes[c] = std::make_pair(spread_bits(ix) | (spread_bits(iy) << 1) | (spread_bits(iz) << 2), c);
      }
  std::sort(codes.begin(), codes.end());
  std::vector<int> rank(h->ncell3), of_rank(h->ncell3);
  for (int r = 0; r < h->ncell3; r++) {
    of_rank[r] = codes[r].second;
    rank[codes[r].second] = r;
  }
  if ((s = upload(h, &h->d_cell_rank, rank)) || (s = upload(h, &h->d_cell_of_rank, of_rank)))
    return s;
  if ((s = dalloc(h, &h->d_cell_count, h->ncell3)) || (s = dalloc(h, &h->d_cell_start, h->ncell3 + 1)))
    return s;
  h->first = true;
  return MMNB_OK;
}

int alloc_rows(mmnb_handle *h, int cap)
{
  drop_host_graph(h);
  h->rowcap = std::max(1, std::min(cap, h->ngroup));
  int s = dalloc(h, &h->d_nbr, (size_t) h->ngroup * h->rowcap);
  if (!s && h->prune_margin > 0)
    s = dalloc(h, &h->d_pnbr, (size_t) h->ngroup * h->rowcap);
  return s;
}

int initial_rowcap(const mmnb_handle *h)
{
  const double rho = h->ngroup / h->volume;
  const double expect = 4.0 / 3.0 * M_PI * pow(h->rc + h->nlw, 3) * rho + (double) h->ngroup / h->ncell3;
  const int cap = (int) (1.5 * expect) + 48;
  return (cap + 31) / 32 * 32;
}

int setup_cheb(mmnb_handle *h)
{
  std::vector<double> c7(kCheb * 7), c8(kCheb * 8, 0.0);
  chebyshev_table(h->rc, h->eta, &h->cheb_min, &h->cheb_max, &h->cheb_inv_dx, c7.data());
  for (int i = 0; i < kCheb; i++)
    for (int k = 0; k < 7; k++)
      c8[8 * i + k] = c7[7 * i + k];
  int s = upload(h, &h->d_cheb, c8);
  if (s)
    return s;
  // the rigid-water FP64 kernel's copy: the cubic's coefficients only, as two
  // arrays of (c0, c1) and (c2, c3), continued to (rc + 2.5)^2 so every site
  // pair of a water group pair within rc falls inside it
  const double dx = (h->cheb_max - h->cheb_min) / kCheb;
  const double r2ext = sq(h->rc + 2.5);
  h->cheb_w_nseg = std::max(kCheb, std::min(kChebWMax, (int) ceil((r2ext - h->cheb_min) * h->cheb_inv_dx)));
  std::vector<double> w(4 * (size_t) h->cheb_w_nseg);
  for (int i = 0; i < h->cheb_w_nseg; i++) {
    double o[7];
    if (i < kCheb)
      std::copy(c7.begin() + 7 * i, c7.begin() + 7 * i + 7, o);
    else
      chebyshev_segment(i, h->cheb_min, dx, h->eta, o);
    w[2 * i] = o[0];
    w[2 * i + 1] = o[1];
    w[2 * ((size_t) h->cheb_w_nseg + i)] = o[2];
    w[2 * ((size_t) h->cheb_w_nseg + i) + 1] = o[3];
  }
  h->water64_grid = 0;  // the kernel's shared-memory size follows the table
  if ((s = upload(h, &h->d_cheb_w, w)))
    return s;
  // the same fit of (2 eta / sqrt(pi)) exp(-eta^2 r^2) = -eta d/d(eta) of
  // erfc(eta r)/r: since the fit is linear in the sampled values, these cubics
  // are exactly -eta d/d(eta) of the table's cubics (mmnb_virial's eta term)
  std::vector<double> d4(4 * (size_t) kCheb);
  const double eta = h->eta;
  for (int i = 0; i < kCheb; i++) {
    double o[7];
    chebyshev_fit(i, h->cheb_min, dx, [eta](double r2) { return eta * M_2_SQRTPI * exp(-eta * eta * r2); }, o);
    for (int k = 0; k < 4; k++)
      d4[4 * i + k] = o[k];
  }
  return upload(h, &h->d_cheb_d, d4);
}

// reciprocal lattice 2 pi inv(latv)^T of the diagonal box
void recip_diag(const mmnb_handle *h, double rec[3])
{
  for (int d = 0; d < 3; d++)
    rec[d] = 2 * M_PI * (1.0 / h->box.L[d]);
}

// ordinary Ewald wave vectors (src/kspace.c:35-71, 96-103)
int setup_kspace(mmnb_handle *h)
{
  const double kc = h->cfg.kspace_cutoff;
  const double n2max = kc * kc + 1e-8;
  const int nmax = (int) floor(kc);
  struct KI { int x, y, z, n2; };
  std::vector<KI> ks;
  for (int nx = 0; nx <= nmax; nx++)
    for (int ny = (nx == 0 ? 0 : -nmax); ny <= nmax; ny++)
      for (int nz = (nx == 0 && ny == 0 ? 1 : -nmax); nz <= nmax; nz++)
        if (nx * nx + ny * ny + nz * nz <= n2max)
          ks.push_back(KI{nx, ny, nz, nx * nx + ny * ny + nz * nz});
  std::stable_sort(ks.begin(), ks.end(), [](const KI &a, const KI &b) { return a.n2 > b.n2; });
  h->nk = (int) ks.size();
  h->kmax = nmax;
  double rec[3];
  recip_diag(h, rec);
  std::vector<double> kv(3 * ks.size()), ak(ks.size());
  const double c = 0.25 / (h->eta * h->eta), f = 4 * M_PI / h->volume;
  for (size_t k = 0; k < ks.size(); k++) {
    kv[3 * k] = rec[0] * ks[k].x;
    kv[3 * k + 1] = rec[1] * ks[k].y;
    kv[3 * k + 2] = rec[2] * ks[k].z;
    const double k2 = kv[3 * k] * kv[3 * k] + kv[3 * k + 1] * kv[3 * k + 1] + kv[3 * k + 2] * kv[3 * k + 2];
    ak[k] = f * exp(-k2 * c) / k2;
  }
  int s;
  if ((s = upload(h, &h->d_kvecs, kv)) || (s = upload(h, &h->d_ak, ak)) ||
      (s = dalloc(h, &h->d_skc, 2 * ks.size())))
    return s;
  return MMNB_OK;
}

// p3m_optimize (src/pppm.c:666-716): the screening eta that minimises
// chi_r^2 + chi_k^2, with chi_r = 2 / sqrt(rc / V^(1/3)) exp(-(rc eta)^2) the
// real-space error estimate and chi_k the mesh's (p3m_init, here k_green at
// that eta; a negative eta scores 1e8).  The reference runs GSL's one-variable
// simplex (gsl_multimin_fminimizer_nmsimplex) from eta = 0.1 / spacing with a
// step of 0.1 and stops it once the simplex size -- the mean distance of its
// vertices from their centre -- is below 1e-4, or after 100 iterations.  The
// same start, step, size test and iteration limit drive the Nelder-Mead moves
// here as Lagarias, Reeds, M. Wright and P. Wright state them (SIAM J. Optim. 9
// (1998) 112-147: reflection 1, expansion 2, contraction 1/2, shrink 1/2).
// Both end within the size tolerance of the objective's minimum, not on the
// same iterates.  The influence function is then made at the chosen eta (the
// reference leaves the one of the last point its simplex evaluated).
static int p3m_optimize_eta(mmnb_handle *h, double spacing)
{
  const double v13 = pow(h->volume, 1.0 / 3.0);
  cudaError_t err = cudaSuccess;
  auto objective = [&](double eta) {
    if (eta < 0)
      return 1e8;
    const double chi_r = 2 / sqrt(h->rc / v13) * exp(-sq(h->rc * eta));
    double chi_k = 0;
    if (err == cudaSuccess)
      err = launch_p3m_green(h, eta, &chi_k);
    return sq(chi_r) + sq(chi_k);
  };
  double x[2] = {0.1 / spacing, 0.1 / spacing + 0.1};
  double fx[2] = {objective(x[0]), objective(x[1])};
  for (int it = 1; it <= 100 && err == cudaSuccess; it++) {
    const int lo = fx[1] < fx[0] ? 1 : 0, hi = 1 - lo;
    const double c = x[lo];  // centroid of the vertices other than the worst
    const double xr = 2 * c - x[hi], fr = objective(xr);
    bool shrink = false;
    if (fr < fx[lo]) {
      const double xe = 3 * c - 2 * x[hi], fe = objective(xe);
      x[hi] = fe < fr ? xe : xr;
      fx[hi] = fe < fr ? fe : fr;
    } else if (fr < fx[hi]) {
      const double xo = c + 0.5 * (xr - c), fo = objective(xo);
      if (fo <= fr) {
        x[hi] = xo;
        fx[hi] = fo;
      } else {
        shrink = true;
      }
    } else {
      const double xi = c + 0.5 * (x[hi] - c), fi = objective(xi);
      if (fi < fx[hi]) {
        x[hi] = xi;
        fx[hi] = fi;
      } else {
        shrink = true;
      }
    }
    if (shrink) {
      x[hi] = c + 0.5 * (x[hi] - c);
      fx[hi] = objective(x[hi]);
    }
    if (0.5 * fabs(x[1] - x[0]) < 1e-4)
      break;
  }
  if (err != cudaSuccess)
    return fail(h, MMNB_ERR_CUDA, std::string("P3M screening optimisation: ") + cudaGetErrorString(err));
  h->eta = fx[1] < fx[0] ? x[1] : x[0];
  h->eta_optimised = true;
  if (!(h->eta > 0))
    return fail(h, MMNB_ERR_ARG, "P3M screening optimisation did not find a positive eta");
  return MMNB_OK;
}

int setup_p3m(mmnb_handle *h)
{
  const mmnb_config &c = h->cfg;
  if (c.p3m_assignment_order < 2 || c.p3m_assignment_order > kMaxOrder)
    return fail(h, MMNB_ERR_ARG, "p3m_assignment_order must be 2..7");
  if (c.p3m_alias_sum_limit < 1 || c.p3m_alias_sum_limit > 8)
    return fail(h, MMNB_ERR_ARG, "p3m_alias_sum_limit must be 1..8");
  if (!(c.p3m_grid_spacing > 0))
    return fail(h, MMNB_ERR_ARG, "p3m_grid_spacing must be > 0");
  // a grid density, when given, sets the spacing (src/eleclj.cpp:195-200)
  double spacing = c.p3m_grid_spacing;
  if (c.p3m_grid_density > 0) {
    if (!almost_zero(spacing - 0.5))
      return fail(h, MMNB_ERR_ARG, "only one of p3m_grid_spacing, p3m_grid_density should be specified");
    spacing = h->min_diameter / cbrt(c.p3m_grid_density * h->volume);
  }
  for (int d = 0; d < 3; d++)
    h->mesh[d] = near_2357(floor(sqrt(sq(h->box.L[d])) / spacing + 0.5));
  const size_t nr = (size_t) h->mesh[0] * h->mesh[1] * h->mesh[2];
  const size_t nk = (size_t) h->mesh[0] * h->mesh[1] * (h->mesh[2] / 2 + 1);
  int s;
  if ((s = dalloc(h, &h->d_green, nk)) || (s = dalloc(h, &h->d_kvec, 3 * nk)) ||
      (s = dalloc(h, &h->d_chi_part, (nk + 127) / 128)))
    return s;
  if (c.precision == MMNB_MIXED) {
    if ((s = dalloc(h, &h->d_mesh_fx, nr)) || (s = dalloc(h, &h->d_mesh32, nr)) ||
        (s = dalloc(h, &h->d_meshk32, nk)) || (s = dalloc(h, &h->d_green32, nk)))
      return s;
    CK(cudaMemset(h->d_mesh_fx, 0, sizeof(unsigned long long) * nr));
    if (c.p3m_ik_differentiate)
      if ((s = dalloc(h, &h->d_egrid32, 3 * nr)) || (s = dalloc(h, &h->d_egridk32, 3 * nk)))
        return s;
    CKFFT(cufftPlan3d(&h->plan_r2c32, h->mesh[0], h->mesh[1], h->mesh[2], CUFFT_R2C));
    CKFFT(cufftPlan3d(&h->plan_c2r32, h->mesh[0], h->mesh[1], h->mesh[2], CUFFT_C2R));
    CKFFT(cufftSetStream(h->plan_r2c32, h->stream));
    CKFFT(cufftSetStream(h->plan_c2r32, h->stream));
  } else {
    if ((s = dalloc(h, &h->d_mesh, nr * (c.p3m_ik_differentiate ? 1 : 1))) || (s = dalloc(h, &h->d_meshk, nk)))
      return s;
    CKFFT(cufftPlan3d(&h->plan_r2c, h->mesh[0], h->mesh[1], h->mesh[2], CUFFT_D2Z));
    CKFFT(cufftPlan3d(&h->plan_c2r, h->mesh[0], h->mesh[1], h->mesh[2], CUFFT_Z2D));
    CKFFT(cufftSetStream(h->plan_r2c, h->stream));
    CKFFT(cufftSetStream(h->plan_c2r, h->stream));
    if (c.p3m_ik_differentiate)
      if ((s = dalloc(h, &h->d_egrid, 3 * nr)) || (s = dalloc(h, &h->d_egridk, 3 * nk)))
        return s;
  }
  if (h->eta < 0 && (s = p3m_optimize_eta(h, spacing)))
    return s;
  CK(launch_p3m_green(h, h->eta, &h->p3m_chi));
  if (c.precision == MMNB_MIXED)
    CK(launch_green32(h));
  CK(cudaStreamSynchronize(h->stream));
  h->p3m = true;
  return MMNB_OK;
}

void free_all(mmnb_handle *h)
{
  drop_host_graph(h);
  for (cudaEvent_t &ev : h->ev_chunk)
    if (ev) {
      cudaEventDestroy(ev);
      ev = nullptr;
    }
  if (h->ev_eval) {
    cudaEventDestroy(h->ev_eval);
    h->ev_eval = nullptr;
  }
  for (cudaEvent_t &ev : h->ev_in)
    if (ev) {
      cudaEventDestroy(ev);
      ev = nullptr;
    }
  if (h->ev_free) {
    cudaEventDestroy(h->ev_free);
    h->ev_free = nullptr;
  }
  if (h->copy_in) {
    cudaStreamSynchronize(h->copy_in);
    cudaStreamDestroy(h->copy_in);
    h->copy_in = nullptr;
  }
  void *ptrs[] = {h->d_group, h->d_excl_ptr, h->d_excl_idx, h->d_p14_ptr, h->d_p14_idx, h->d_gexcl_ptr,
                  h->d_gexcl_idx, h->d_mask, h->d_q, h->d_sig, h->d_eps, h->d_rscreen, h->d_cheb, h->d_cheb_w, h->d_cheb_d, h->d_lj_row, h->d_lj_row_part,
                  h->d_vir_part, h->d_vir_row, h->d_vir_mol, h->d_vir_molw, h->d_vir_mass,
                  h->d_stencil, h->d_cell_rank, h->d_cell_of_rank, h->d_cell_of_group, h->d_cell_count,
                  h->d_cell_start, h->d_slot, h->d_sorted, h->d_rank, h->d_anchor, h->d_last, h->d_anchor_sorted, h->d_anchor32, h->d_block_sum,
                  h->d_top2, h->d_nbr, h->d_nbr_count, h->d_pnbr, h->d_pcount, h->d_plast, h->d_flags, h->d_sr,
                  h->d_sp, h->d_site_of_slot,
                  h->d_phi, h->d_evec, h->d_ljf, h->d_lj_part, h->d_elec_part, h->d_energy, h->d_r, h->d_f,
                  h->d_mesh, h->d_meshk, h->d_green, h->d_kvec, h->d_egrid, h->d_egridk, h->d_mesh32,
                  h->d_meshk32, h->d_green32, h->d_egrid32, h->d_egridk32, h->d_mesh_fx, h->d_kint, h->d_kvecs, h->d_ak, h->d_skc,
                  h->mx.site, h->mx.par, h->mx.anchor, h->mx.anc32, h->mx.acc, h->mx.acck, h->d_wsum,
                  h->d_bwd, h->d_gmesh, h->d_gmeshk, h->d_chi_part};
  for (void *p : ptrs)
    if (p)
      cudaFree(p);
  if (h->side) {
    cudaStreamSynchronize(h->side);
    cudaStreamDestroy(h->side);
    h->side = nullptr;
  }
  if (h->ev_fork)
    cudaEventDestroy(h->ev_fork);
  if (h->ev_join)
    cudaEventDestroy(h->ev_join);
  h->ev_fork = h->ev_join = nullptr;
  if (h->h_flags)
    cudaFreeHost(h->h_flags);
  if (h->h_f)
    cudaFreeHost(h->h_f);
  if (h->h_out)
    cudaFreeHost(h->h_out);
  if (h->h_status)
    cudaFreeHost(h->h_status);
  if (h->h_bwd)
    cudaFreeHost(h->h_bwd);
  if (h->plan_r2c)
    cufftDestroy(h->plan_r2c);
  if (h->plan_c2r)
    cufftDestroy(h->plan_c2r);
  if (h->plan_r2c32)
    cufftDestroy(h->plan_r2c32);
  if (h->plan_c2r32)
    cufftDestroy(h->plan_c2r32);
  if (h->gplan_r2c)
    cufftDestroy(h->gplan_r2c);
  if (h->gplan_c2r)
    cufftDestroy(h->gplan_c2r);
  for (auto e : h->timing.pool)
    cudaEventDestroy(e);
  if (h->graph_exec)
    cudaGraphExecDestroy(h->graph_exec);
  if (h->graph)
    cudaGraphDestroy(h->graph);
}

}  // namespace

namespace mmnb {

int set_global_error(int code, const std::string &msg)
{
  g_create_error = msg;
  return code;
}

void timing_mark(mmnb_handle *h, const char *name)
{
  Timing &t = h->timing;
  if (!t.on || h->capturing)
    return;
  if (t.used == t.pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess)
      return;
    t.pool.push_back(e);
  }
  cudaEventRecord(t.pool[t.used], h->stream);
  t.names.push_back(name);
  t.used++;
}

// The reference's LJ tail (src/eleclj.cpp:1247-1266) for totals A and B.
double lj_tail_ab(const mmnb_handle *h, double A, double B)
{
  const double rhi = h->rc, rlo = rhi - h->cfg.smoothing_width;
  const double rlo2 = rlo * rlo, rlo3 = rlo2 * rlo, rlo4 = rlo3 * rlo;
  const double rlo5 = rlo4 * rlo, rlo6 = rlo5 * rlo, rlo7 = rlo6 * rlo, rlo9 = rlo7 * rlo2;
  const double rhi2 = rhi * rhi, rhi3 = rhi2 * rhi, rhi4 = rhi3 * rhi, rhi5 = rhi4 * rhi;
  const double rhi6 = rhi5 * rhi, rhi7 = rhi6 * rhi;
  return 2 * M_PI / h->volume *
         (A / (9 * rlo9) + B / (3 * rlo3) -
          (rhi - rlo) / (63 * rhi3 * rlo9 * pow(rhi + rlo, 5)) *
              (3 * B * rhi3 * rlo6 * (7 * rhi4 + 42 * rhi3 * rlo + 112 * rhi2 * rlo2 + 150 * rhi * rlo3 + 25 * rlo4) +
               A * (7 * rhi7 + 42 * rhi6 * rlo + 112 * rhi5 * rlo2 + 182 * rhi4 * rlo3 + 217 * rhi3 * rlo4 +
                    224 * rhi2 * rlo5 + 192 * rhi * rlo6 + 32 * rlo7)));
}

void drop_host_graph(mmnb_handle *h)
{
  if (h->hgraph_exec)
    cudaGraphExecDestroy(h->hgraph_exec);
  if (h->hgraph)
    cudaGraphDestroy(h->hgraph);
  h->hgraph_exec = nullptr;
  h->hgraph = nullptr;
}

}  // namespace mmnb

extern "C" {

int mmnb_config_init(mmnb_config *c)
{
  if (!c)
    return MMNB_ERR_ARG;
  memset(c, 0, sizeof(*c));
  c->precision = MMNB_FP64;
  c->bctype = MMNB_CUBIC;
  c->rspace_cutoff = 0;
  c->smoothing_width = 1;
  c->neighbor_list_width = 0;
  c->kspace_cutoff = 5;
  c->ewald_screening = -1;
  c->use_p3m = 0;
  c->p3m_grid_spacing = 0.5;
  c->p3m_assignment_order = 3;
  c->p3m_alias_sum_limit = 2;
  c->p3m_ik_differentiate = 0;
  c->include_lj_correction = 1;
  c->geometric_combining_for_sigma = 0;
  c->include_rspace = 1;
  c->include_kspace = 1;
  c->include_self = 1;
  c->elec_1_4_scale_factor = 1;
  c->lj_1_4_scale_factor = 1;
  c->rebuild_interval = 0;
  c->device = -1;
  c->p3m_grid_density = -1;
  return MMNB_OK;
}

static int create_impl(mmnb_handle *h, const mmnb_config *c, int nsite, int ngroup, const int *group, int nexcl,
                       const int *excl, int n14, const int *pairs14)
{
  h->cfg = *c;
  if (c->precision != MMNB_FP64 && c->precision != MMNB_MIXED)
    return fail(h, MMNB_ERR_ARG, "precision must be MMNB_FP64 or MMNB_MIXED");
  if (c->bctype != MMNB_CUBIC && c->bctype != MMNB_ORTHORHOMBIC)
    return fail(h, MMNB_ERR_UNSUPPORTED, "only cubic and orthorhombic boundary conditions are supported");
  if (nsite <= 0 || ngroup <= 0 || !group)
    return fail(h, MMNB_ERR_ARG, "nsite and ngroup must be positive and group non-null");
  if ((nexcl > 0 && !excl) || (n14 > 0 && !pairs14) || nexcl < 0 || n14 < 0)
    return fail(h, MMNB_ERR_ARG, "exclusion or 1-4 arrays missing");
  h->nsite = nsite;
  h->ngroup = ngroup;
  // box
  for (int d = 0; d < 3; d++) {
    const double L = c->bctype == MMNB_CUBIC ? c->box[0] : c->box[d];
    if (!(L > 0))
      return fail(h, MMNB_ERR_ARG, "box lengths must be > 0");
    h->box.L[d] = L;
    h->box.invL[d] = 1 / L;
  }
  h->volume = h->box.L[0] * h->box.L[1] * h->box.L[2];
  h->min_diameter = std::min(std::min(h->box.L[0], h->box.L[1]), h->box.L[2]);
  // groups: contiguous, covering every site once
  h->group.assign(group, group + 2 * (size_t) ngroup);
  h->group_of_site.assign(nsite, -1);
  h->maxgs = 1;
  for (int g = 0; g < ngroup; g++) {
    const int a = group[2 * g], b = group[2 * g + 1];
    if (a < 0 || b > nsite || b <= a)
      return fail(h, MMNB_ERR_ARG, "group " + std::to_string(g) + " has an invalid site range");
    h->maxgs = std::max(h->maxgs, b - a);
    for (int s = a; s < b; s++) {
      if (h->group_of_site[s] >= 0)
        return fail(h, MMNB_ERR_ARG, "site " + std::to_string(s) + " belongs to two groups");
      h->group_of_site[s] = g;
    }
  }
  for (int s = 0; s < nsite; s++)
    if (h->group_of_site[s] < 0)
      return fail(h, MMNB_ERR_ARG, "site " + std::to_string(s) + " belongs to no group");
  if (h->maxgs > kMaxGroup)
    return fail(h, MMNB_ERR_UNSUPPORTED, "groups of more than 8 sites are not supported");
  h->G = h->maxgs <= 4 ? h->maxgs : 8;
  // cutoff, skin (src/eleclj.cpp:164-182)
  h->rc = c->rspace_cutoff;
  if (almost_zero(h->rc))
    h->rc = 0.45 * h->min_diameter;
  if (h->rc > 0.49 * h->min_diameter || !(h->rc > 0))
    return fail(h, MMNB_ERR_CUTOFF, "rspace_cutoff must be <= 0.49 * minimum diameter of box");
  if (c->smoothing_width >= h->rc || c->smoothing_width < 0)
    return fail(h, MMNB_ERR_CUTOFF, "smoothing_width must be less than the real-space cutoff");
  h->nlw = c->neighbor_list_width;
  if (almost_zero(h->nlw)) {
    h->nlw = 0.2 * h->rc;
    if (h->rc + h->nlw >= 0.5 * h->min_diameter)
      h->nlw = 0.499 * h->min_diameter - h->rc;
  }
  if (h->nlw < 0)
    return fail(h, MMNB_ERR_ARG, "neighbor_list_width must be >= 0");
  h->rhi2 = sq(h->rc);
  h->rlo2 = sq(h->rc - c->smoothing_width);
  h->inv_sw = h->rhi2 > h->rlo2 ? 1.0 / (h->rhi2 - h->rlo2) : 0.0;
  // Ewald parameter (src/eleclj.cpp:189-239)
  // (with P3M a negative value is resolved by setup_p3m, before the real-space
  // table is made)
  h->eta = c->ewald_screening;
  const bool p3m = c->include_kspace && c->use_p3m;
  if (h->eta < 0 && !p3m)
    h->eta = sqrt((M_PI * c->kspace_cutoff) / (h->rc * h->min_diameter));
  if (!(h->eta > 0) && !(p3m && h->eta < 0))
    return fail(h, MMNB_ERR_ARG, "ewald_screening must be > 0, or negative for the automatic choice");
  // topology tables
  std::vector<std::pair<int, int>> ep, pp;
  for (int k = 0; k < nexcl; k++) {
    const int i = excl[2 * k], j = excl[2 * k + 1];
    if (i < 0 || j < 0 || i >= nsite || j >= nsite)
      return fail(h, MMNB_ERR_ARG, "exclusion pair out of range");
    ep.push_back(std::make_pair(i, j));
  }
  build_csr(nsite, ep, h->excl_ptr, h->excl_idx);
  h->use_14 = !almost_zero(c->elec_1_4_scale_factor - 1) || !almost_zero(c->lj_1_4_scale_factor - 1);
  if (h->use_14)
    for (int k = 0; k < n14; k++) {
      const int i = pairs14[2 * k], j = pairs14[2 * k + 1];
      if (i < 0 || j < 0 || i >= nsite || j >= nsite)
        return fail(h, MMNB_ERR_ARG, "1-4 pair out of range");
      pp.push_back(std::make_pair(i, j));
    }
  build_csr(nsite, pp, h->p14_ptr, h->p14_idx);
  std::vector<std::pair<int, int>> gp;
  for (auto &e : ep) {
    const int gi = h->group_of_site[e.first], gj = h->group_of_site[e.second];
    if (gi != gj)
      gp.push_back(std::make_pair(gi, gj));
  }
  build_csr(ngroup, gp, h->gexcl_ptr, h->gexcl_idx);
  h->any_gexcl = !h->gexcl_idx.empty();
  // device
  if (c->device >= 0)
    CK(cudaSetDevice(c->device));
  CK(cudaGetDevice(&h->dev));
  CK(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
  h->stream = h->own_stream;
  {
    // the mesh work on the side stream at the highest priority: its blocks
    // go first whenever the pair kernels' blocks leave an SM slot (graphs are
    // instantiated with node priorities so captured launches keep it)
    int least = 0, greatest = 0;
    CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    CK(cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, greatest));
  }
  CK(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
  int s;
  std::vector<int> gvec(h->group);
  if ((s = upload(h, &h->d_group, gvec)) || (s = upload(h, &h->d_excl_ptr, h->excl_ptr)) ||
      (s = upload(h, &h->d_excl_idx, h->excl_idx)) || (s = upload(h, &h->d_p14_ptr, h->p14_ptr)) ||
      (s = upload(h, &h->d_p14_idx, h->p14_idx)) || (s = upload(h, &h->d_gexcl_ptr, h->gexcl_ptr)) ||
      (s = upload(h, &h->d_gexcl_idx, h->gexcl_idx)))
    return s;
  if ((s = dalloc(h, &h->d_mask, nsite)) || (s = dalloc(h, &h->d_q, nsite)) || (s = dalloc(h, &h->d_sig, nsite)) ||
      (s = dalloc(h, &h->d_eps, nsite)) || (s = dalloc(h, &h->d_rscreen, nsite)))
    return s;
  if ((s = dalloc(h, &h->d_cell_of_group, ngroup)) || (s = dalloc(h, &h->d_slot, ngroup)) ||
      (s = dalloc(h, &h->d_sorted, ngroup)) || (s = dalloc(h, &h->d_rank, ngroup)) ||
      (s = dalloc(h, &h->d_anchor, 3 * (size_t) ngroup)) || (s = dalloc(h, &h->d_last, 3 * (size_t) ngroup)) ||
      (s = dalloc(h, &h->d_anchor_sorted, 3 * (size_t) ngroup)) || (s = dalloc(h, &h->d_anchor32, ngroup)) ||
      (s = dalloc(h, &h->d_nbr_count, ngroup)) || (s = dalloc(h, &h->d_flags, kFlagCount)))
    return s;
  {
    // one word per block of the cooperative rebuild (at most 2048 threads of
    // 256-thread blocks resident per SM)
    int nsm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->dev));
    h->block_sum_cap = 8 * nsm;
    if ((s = dalloc(h, &h->d_block_sum, (size_t) h->block_sum_cap)))
      return s;
  }
  CK(cudaMemset(h->d_last, 0, sizeof(double) * 3 * ngroup));
  CK(cudaMemset(h->d_flags, 0, sizeof(int) * kFlagCount));
  CK(cudaMallocHost((void **) &h->h_flags, sizeof(int) * kFlagCount));
  h->top2_blocks = std::min(256, div_up(ngroup, 256));
  // per block: the two largest moves since the last build, then since the last prune
  if ((s = dalloc(h, &h->d_top2, 4 * (size_t) h->top2_blocks)))
    return s;
  const size_t nslot = (size_t) ngroup * h->G;
  if ((s = dalloc(h, &h->d_sr, nslot)) || (s = dalloc(h, &h->d_sp, nslot)) ||
      (s = dalloc(h, &h->d_site_of_slot, nslot)))
    return s;
  h->elec_blocks = div_up(nsite, 256);
  h->lj_pair_blocks = pair_blocks(h);
  h->lj_excl_blocks = excl_blocks(h);
  const size_t nlj = (size_t) h->lj_pair_blocks + h->lj_excl_blocks;
  if ((s = dalloc(h, &h->d_phi, nsite)) || (s = dalloc(h, &h->d_evec, 3 * (size_t) nsite)) ||
      (s = dalloc(h, &h->d_ljf, 3 * (size_t) nsite)) || (s = dalloc(h, &h->d_lj_part, nlj)) ||
      (s = dalloc(h, &h->d_lj_row, ngroup)) || (s = dalloc(h, &h->d_vir_part, nlj)) ||
      (s = dalloc(h, &h->d_vir_row, ngroup)) ||
      (s = dalloc(h, &h->d_elec_part, h->elec_blocks)) || (s = dalloc(h, &h->d_lj_row_part, h->elec_blocks)) || (s = dalloc(h, &h->d_energy, 16)) ||
      (s = dalloc(h, &h->d_r, 3 * (size_t) nsite)) || (s = dalloc(h, &h->d_f, 3 * (size_t) nsite)) ||
      (s = dalloc(h, &h->d_wsum, 8)))
    return s;
  CK(cudaMemset(h->d_lj_part, 0, sizeof(double) * nlj));
  CK(cudaMemset(h->d_wsum, 0, sizeof(unsigned long long) * 8));
  if (c->precision == MMNB_MIXED) {
    if ((s = dalloc(h, &h->mx.site, nslot)) || (s = dalloc(h, &h->mx.par, nslot)) ||
        (s = dalloc(h, &h->mx.anchor, ngroup)) || (s = dalloc(h, &h->mx.anc32, ngroup)) ||
        (s = dalloc(h, &h->mx.acc, (size_t) nsite * kAccStride)) ||
        (s = dalloc(h, &h->mx.acck, (size_t) nsite * 4)))
      return s;
    CK(cudaMemset(h->mx.acc, 0, sizeof(long long) * nsite * kAccStride));
  }
  CK(cudaMallocHost((void **) &h->h_f, sizeof(double) * 3 * (size_t) nsite));
  CK(cudaMallocHost((void **) &h->h_out, sizeof(double) * 16));
  CK(cudaHostAlloc((void **) &h->h_status, sizeof(double) * mmnb_handle::kStatusDoubles, cudaHostAllocMapped));
  CK(cudaHostGetDevicePointer((void **) &h->d_status, h->h_status, 0));
  memset(h->h_status, 0, sizeof(double) * mmnb_handle::kStatusDoubles);
  if ((s = setup_cells(h)))
    return s;
  // the rigid-water kernel's rows pruned to rc + width / 3: rebuilt (by that
  // kernel, from the full rows) whenever the two largest anchor moves since
  // the last prune exceed width / 3, so every pair within rc stays listed
  h->prune_margin = (c->precision == MMNB_MIXED && h->nlw >= 0.3) ? h->nlw / 3 : 0.0;
  if (h->prune_margin > 0 &&
      ((s = dalloc(h, &h->d_pcount, ngroup)) || (s = dalloc(h, &h->d_plast, 3 * (size_t) ngroup))))
    return s;
  if ((s = alloc_rows(h, initial_rowcap(h))))
    return s;
  if (c->include_kspace && c->use_p3m && (s = setup_p3m(h)))
    return s;
  if ((s = setup_cheb(h)))
    return s;
  if (c->include_kspace && !c->use_p3m) {
    h->kspace = true;
    if ((s = setup_kspace(h)))
      return s;
  }
  return MMNB_OK;
}

int mmnb_create(const mmnb_config *c, int nsite, int ngroup, const int *group, int nexcl, const int *excl, int n14,
                const int *pairs14, mmnb_handle **out)
{
  if (!c || !out)
    return fail(nullptr, MMNB_ERR_ARG, "null config or output pointer");
  *out = nullptr;
  mmnb_handle *h = new mmnb_handle;
  const int s = create_impl(h, c, nsite, ngroup, group, nexcl, excl, n14, pairs14);
  if (s) {
    g_create_error = h->err;
    free_all(h);
    if (h->own_stream)
      cudaStreamDestroy(h->own_stream);
    delete h;
    return s;
  }
  *out = h;
  return MMNB_OK;
}

static double lj_tail(const mmnb_handle *h) { return lj_tail_ab(h, h->totA, h->totB); }

static void update_energy_constants(mmnb_handle *h, double qsum)
{
  h->lj_correction = lj_tail(h);
  h->neutral_b = almost_zero(qsum) ? 0 : -M_PI / (sq(h->eta) * h->volume) * qsum;
}

int mmnb_set_params(mmnb_handle *h, const int *site_mask, const double *q, const double *sig, const double *eps,
                    const double *rscreen)
{
  if (!h || !site_mask || !q || !sig || !eps)
    return fail(h, MMNB_ERR_ARG, "null parameter array");
  drop_host_graph(h);
  h->buf_gen++;  // the kernels an evaluation launches may change
  const int n = h->nsite;
  std::vector<double> rs(n, 0.0);
  h->any_q = h->any_lj = h->has_rscreen = false;
  h->lj_on_anchors_only = true;
  double qsum = 0;
  for (int i = 0; i < n; i++) {
    if (site_mask[i] & MMNB_SITE_HAS_Q)
      h->any_q = true;
    if (site_mask[i] & MMNB_SITE_HAS_LJ) {
      h->any_lj = true;
      if (h->group[2 * h->group_of_site[i]] != i)
        h->lj_on_anchors_only = false;
      if (!(sig[i] > 0) || eps[i] < 0)
        return fail(h, MMNB_ERR_ARG, "LJ sites need sigma > 0 and epsilon >= 0");
    }
    if (rscreen) {
      if (rscreen[i] < 0)
        return fail(h, MMNB_ERR_ARG, "screening radius must be >= 0");
      rs[i] = rscreen[i];
      if (rscreen[i] > 0)
        h->has_rscreen = true;
    }
    qsum += q[i];
  }
  CK(cudaMemcpy(h->d_mask, site_mask, sizeof(int) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_q, q, sizeof(double) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_sig, sig, sizeof(double) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_eps, eps, sizeof(double) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_rscreen, rs.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
  h->grad_ready = false;
  h->hq.assign(q, q + n);
  h->hsig.assign(sig, sig + n);
  h->heps.assign(eps, eps + n);
  // LJ tail totals over distinct (sigma, epsilon) printed as %12.6g
  // (src/eleclj.cpp:283-308)
  h->cls_sig.clear();
  h->cls_eps.clear();
  h->cls_n.clear();
  h->site_cls.assign(n, -1);
  for (int i = 0; i < n; i++) {
    if (!(site_mask[i] & MMNB_SITE_HAS_LJ))
      continue;
    char key[128];
    double sv, ev;
    snprintf(key, sizeof key, "%12.6g %12.6g", sig[i], eps[i]);
    sscanf(key, "%lf%lf", &sv, &ev);
    size_t a = 0;
    for (; a < h->cls_sig.size(); a++)
      if (h->cls_sig[a] == sv && h->cls_eps[a] == ev)
        break;
    if (a == h->cls_sig.size()) {
      h->cls_sig.push_back(sv);
      h->cls_eps.push_back(ev);
      h->cls_n.push_back(0);
    }
    h->cls_n[a]++;
    h->site_cls[i] = (int) a;
  }
  h->totA = h->totB = 0;
  for (size_t a = 0; a < h->cls_sig.size(); a++)
    for (size_t b = 0; b < h->cls_sig.size(); b++) {
      const double sa = h->cls_sig[a], sb = h->cls_sig[b];
      const double s6 = pow(h->cfg.geometric_combining_for_sigma ? sqrt(sa * sb) : 0.5 * (sa + sb), 6);
      const double bb = 4 * sqrt(h->cls_eps[a] * h->cls_eps[b]) * h->cls_n[a] * h->cls_n[b] * s6;
      h->totB -= bb;
      h->totA += bb * s6;
    }
  update_energy_constants(h, qsum);
  // rigid-water topology: every group [O(q, LJ), H(q), H(q)], nothing else
  h->water = h->G == 3 && !h->has_rscreen && !h->any_gexcl;
  for (int g = 0; g < h->ngroup && h->water; g++) {
    const int a = h->group[2 * g];
    h->water = h->group[2 * g + 1] - a == 3 && site_mask[a] == (MMNB_SITE_HAS_Q | MMNB_SITE_HAS_LJ) &&
               site_mask[a + 1] == MMNB_SITE_HAS_Q && site_mask[a + 2] == MMNB_SITE_HAS_Q;
  }
  h->water_uni = h->water && h->ngroup > 0;
  if (h->water_uni) {
    const int a = h->group[0];
    for (int g = 0; g < h->ngroup && h->water_uni; g++) {
      const int b = h->group[2 * g];
      h->water_uni = q[b] == q[a] && sig[b] == sig[a] && eps[b] == eps[a] && q[b + 1] == q[a + 1] &&
                     q[b + 2] == q[a + 1];
    }
    h->uni_qO = (float) q[a];
    h->uni_qH = (float) q[a + 1];
    h->uni_sig = (float) sig[a];
    h->uni_seps = (float) sqrt(eps[a]);
  }
  h->params_set = true;
  return MMNB_OK;
}

// sites [lo, hi) of the host call's c-th positions piece
static void in_chunk_sites(const mmnb_handle *h, int c, int &lo, int &hi)
{
  const int n = mmnb_handle::kInChunks;
  lo = (int) ((long) h->nsite * c / n);
  hi = (int) ((long) h->nsite * (c + 1) / n);
}

int mmnb_compute_device(mmnb_handle *h, const double *d_r, double *d_f, double *d_energy)
{
  if (!h || !d_r)
    return fail(h, MMNB_ERR_ARG, "null handle or positions");
  h->grad_ready = false;
  if (!h->params_set)
    return fail(h, MMNB_ERR_STATE, "mmnb_set_params has not been called");
  const bool mixed = h->cfg.precision == MMNB_MIXED;
  double *energy = d_energy ? d_energy : h->d_energy;
  timing_mark(h, "start");
  // P3M charge assignment and FFTs depend only on the positions: they run on
  // the side stream while the list and pair kernels run here, and are joined
  // back before k_finalize (FP64 form: before the interpolation, which adds
  // to what the pair kernels wrote).  With stage timing on, the join follows
  // at once so the marks stay serial.
  const bool p3m = h->any_q && h->cfg.include_kspace && h->p3m;
  // the side stream pays off when the pair kernels leave room beside them;
  // mmnb_autotune may put the mesh work in line instead (tune.p3m_side = 0)
  const bool side = p3m && h->tune.p3m_side;
  // the mixed form's FP64 site arrays (written by the exclusion corrections)
  // do not meet the pair kernels either: they go to the side stream too
  const bool excl_side = side && mixed && h->cfg.include_rspace;
  auto zero_site_arrays = [&]() -> cudaError_t {
    cudaError_t e;
    if ((e = cudaMemsetAsync(h->d_phi, 0, sizeof(double) * h->nsite, h->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->d_evec, 0, sizeof(double) * 3 * h->nsite, h->stream)) != cudaSuccess)
      return e;
    return cudaMemsetAsync(h->d_ljf, 0, sizeof(double) * 3 * h->nsite, h->stream);
  };
  // the mixed form's interpolation writes words of its own (k_gather_mixed),
  // so it joins the mesh work; the FP64 interpolation adds into the site
  // arrays the pair kernels write and waits for them
  const int mesh_stages = mixed ? 3 : 1;
  if (side) {
    cudaStream_t main = h->stream;
    CK(cudaEventRecord(h->ev_fork, main));
    CK(cudaStreamWaitEvent(h->side, h->ev_fork, 0));
    h->stream = h->side;
    cudaError_t e = cudaSuccess;
    int stages = mesh_stages;
    if (h->in_chunks) {
      // the host call's positions arrive in pieces: each piece's charges are
      // assigned as it lands (mixed form), the rest follows the last piece
      for (int c = 0; c < mmnb_handle::kInChunks && e == cudaSuccess; c++) {
        e = cudaStreamWaitEvent(h->side, h->ev_in[c], cudaEventWaitExternal);
        int lo, hi;
        in_chunk_sites(h, c, lo, hi);
        if (e == cudaSuccess && mixed)
          e = launch_spread_mixed_range(h, d_r, lo, hi);
      }
      if (mixed)
        stages |= 4;
    }
    if (excl_side && e == cudaSuccess) {
      e = launch_exclusions(h, d_r);
      timing_mark(h, "rspace_excl");
    }
    if (e == cudaSuccess)
      e = mixed ? launch_p3m_mixed(h, d_r, stages) : launch_p3m_fp64(h, d_r, stages);
    h->stream = main;
    CK(e);
    CK(cudaEventRecord(h->ev_join, h->side));
    if (h->timing.on)
      CK(cudaStreamWaitEvent(main, h->ev_join, 0));
  }
  if (h->in_chunks)
    CK(cudaStreamWaitEvent(h->stream, h->ev_in[mmnb_handle::kInChunks - 1], cudaEventWaitExternal));
  if (p3m && !side)
    CK(mixed ? launch_p3m_mixed(h, d_r, mesh_stages) : launch_p3m_fp64(h, d_r, mesh_stages));
  CK(launch_list_check(h, d_r, h->force_rebuild_next));
  CK(launch_list_rebuild(h));
  timing_mark(h, "nbrlist");
  // FP64 site arrays collect the terms the fixed-point sums do not hold; their
  // first writer (FP64 pair kernels, or the mixed form's exclusion
  // corrections) assigns them, so they need clearing only without real space
  if (!h->cfg.include_rspace)
    CK(zero_site_arrays());
  // FP64 rigid water: its own kernel (any request, site fields included)
  const bool water64 = !mixed && h->water && h->cfg.include_rspace;
  if (mixed)
    CK(launch_prep_mixed(h, d_r));
  else if (water64)
    CK(launch_sort_water64(h, d_r));
  else
    CK(launch_sort_sites(h, d_r));
  timing_mark(h, "sort_sites");
  h->used_water = false;
  h->used_water64 = false;
  if (h->cfg.include_rspace) {
    if (mixed && h->water && !h->want_fields) {
      CK(launch_rspace_water(h));
      h->used_water = true;
    } else if (mixed) {
      CK(launch_rspace_mixed(h));
    } else if (water64) {
      CK(launch_rspace_water64(h));
      h->used_water64 = true;
    } else {
      CK(launch_rspace_fp64(h));
    }
    timing_mark(h, "rspace_pair");
    if (!excl_side) {
      CK(launch_exclusions(h, d_r));
      timing_mark(h, "rspace_excl");
    }
  } else {
    CK(cudaMemsetAsync(h->d_lj_part, 0, sizeof(double) * (h->lj_pair_blocks + h->lj_excl_blocks), h->stream));
    if (mixed)
      CK(cudaMemsetAsync(h->mx.acc, 0, sizeof(long long) * h->nsite * kAccStride, h->stream));
  }
  if (p3m) {
    if (side && !h->timing.on)
      CK(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
    if (!mixed)
      CK(launch_p3m_fp64(h, d_r, 2));
    timing_mark(h, "kspace");
  } else if (h->any_q && h->cfg.include_kspace && h->kspace) {
    CK(launch_kspace(h, d_r));
    timing_mark(h, "kspace");
  }
  CK(launch_finalize(h, d_f, energy));
  timing_mark(h, "finalize");
  h->first = false;
  h->force_rebuild_next = 0;
  h->evals++;
  return MMNB_OK;
}

int mmnb_graph_capture(mmnb_handle *h, const double *d_r, double *d_f, double *d_energy)
{
  if (!h || !d_r)
    return fail(h, MMNB_ERR_ARG, "null handle or positions");
  if (h->first)
    return fail(h, MMNB_ERR_STATE, "evaluate once (mmnb_compute) before capturing");
  if (h->stream == nullptr)
    return fail(h, MMNB_ERR_STATE, "capture needs a non-default stream");
  if (h->graph_exec) {
    cudaGraphExecDestroy(h->graph_exec);
    h->graph_exec = nullptr;
  }
  if (h->graph) {
    cudaGraphDestroy(h->graph);
    h->graph = nullptr;
  }
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  h->capturing = true;
  const long ev = h->evals, ln = h->launches;
  const int s = mmnb_compute_device(h, d_r, d_f, d_energy);
  h->capturing = false;
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  h->evals = ev;
  h->launch_per_eval = h->launches - ln;
  h->launches = ln;
  if (s)
    return s;
  if (e != cudaSuccess)
    return fail(h, MMNB_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
  h->graph = g;
  CK(cudaGraphInstantiate(&h->graph_exec, h->graph, cudaGraphInstantiateFlagUseNodePriority));
  h->graph_gen = h->buf_gen;
  return MMNB_OK;
}

int mmnb_graph_launch(mmnb_handle *h)
{
  if (!h || !h->graph_exec)
    return fail(h, MMNB_ERR_STATE, "no captured evaluation");
  if (h->graph_gen != h->buf_gen)
    return fail(h, MMNB_ERR_STATE,
                "device buffers were reallocated since the capture (rows regrown, mmnb_scale, mmnb_set_params): "
                "capture again");
  CK(cudaGraphLaunch(h->graph_exec, h->stream));
  h->grad_ready = false;
  h->evals++;
  h->launches += h->launch_per_eval;
  return MMNB_OK;
}

// f[i] += src[i] over [b, e), split over host threads when the range is large
// f += src over [b, e) on the host cores: the add of each chunk runs while
// the next chunk is in flight, and its memory traffic (two reads and a write
// of the chunk) bounds the host call's tail
static void add_forces(double *f, const double *src, size_t b, size_t e)
{
  const long n = (long) (e - b);
#pragma omp parallel for schedule(static) if (n > (1 << 12))
  for (long i = 0; i < n; i++)
    f[b + i] += src[b + i];
}

// keep: leave the site potentials and fields of this evaluation on the device
// for mmnb_site_gradients (mmnb_forward)
static int compute_host(mmnb_handle *h, const double *r, double *f, double *u, mmnb_energy *e, double *phi,
                        double *evec, bool keep)
{
  if (!h || !r)
    return fail(h, MMNB_ERR_ARG, "null handle or positions");
  h->grad_ready = false;
  const size_t n3 = 3 * (size_t) h->nsite;
  if (!h->ev_eval) {
    CK(cudaEventCreateWithFlags(&h->ev_eval, cudaEventDisableTiming));
    for (cudaEvent_t &ev : h->ev_chunk)
      CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  }
  volatile unsigned long long *ready =
      reinterpret_cast<volatile unsigned long long *>(h->h_status) + mmnb_handle::kStatusReady;
  for (int attempt = 0; attempt < 2; attempt++) {
    *ready = 0ull;  // k_finalize sets it once this evaluation's status is in place
    // after the first call, a plain evaluation replays the handle's own graph
    // (zeroing, list check/rebuild, pair and mesh kernels, finalize)
    const bool graph =
        !h->first && !(phi || evec || keep) && !h->timing.on && !h->force_rebuild_next && !h->want_virial;
    if (graph) {
      // the positions in pieces on the copy stream (once the handle's stream
      // is done with d_r); the graph waits for each piece where it needs it
      if (!h->copy_in) {
        CK(cudaStreamCreateWithFlags(&h->copy_in, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&h->ev_free, cudaEventDisableTiming));
        for (cudaEvent_t &ev : h->ev_in)
          CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      }
      CK(cudaEventRecord(h->ev_free, h->stream));
      CK(cudaStreamWaitEvent(h->copy_in, h->ev_free, 0));
      for (int c = 0; c < mmnb_handle::kInChunks; c++) {
        int lo, hi;
        in_chunk_sites(h, c, lo, hi);
        if (hi > lo)
          CK(cudaMemcpyAsync(h->d_r + 3 * (size_t) lo, r + 3 * (size_t) lo, sizeof(double) * 3 * (hi - lo),
                             cudaMemcpyHostToDevice, h->copy_in));
        CK(cudaEventRecord(h->ev_in[c], h->copy_in));
      }
    } else {
      CK(cudaMemcpyAsync(h->d_r, r, sizeof(double) * n3, cudaMemcpyHostToDevice, h->stream));
    }
    if (graph && !h->hgraph_exec) {
      CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      h->capturing = true;
      h->in_chunks = true;
      const long ev = h->evals, ln = h->launches;
      cudaError_t ce = cudaMemsetAsync(h->d_f, 0, sizeof(double) * n3, h->stream);
      if (ce == cudaSuccess)
        ce = cudaMemsetAsync(h->d_flags + kFlagOverflow, 0, sizeof(int), h->stream);
      h->want_status = true;
      const int s = ce == cudaSuccess ? mmnb_compute_device(h, h->d_r, h->d_f, h->d_energy) : MMNB_ERR_CUDA;
      h->want_status = false;
      h->capturing = false;
      h->in_chunks = false;
      cudaGraph_t g = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(h->stream, &g);
      h->evals = ev;
      h->host_launch_per_eval = h->launches - ln;
      h->launches = ln;
      if (s || ec != cudaSuccess) {
        if (g)
          cudaGraphDestroy(g);
        if (s)
          return s;
        return fail(h, MMNB_ERR_CUDA, std::string("capture of the host call: ") + cudaGetErrorString(ec));
      }
      h->hgraph = g;
      CK(cudaGraphInstantiate(&h->hgraph_exec, g, cudaGraphInstantiateFlagUseNodePriority));
    }
    if (graph) {
      CK(cudaGraphLaunch(h->hgraph_exec, h->stream));
      h->evals++;
      h->launches += h->host_launch_per_eval;
    } else {
      CK(cudaMemsetAsync(h->d_f, 0, sizeof(double) * n3, h->stream));
      CK(cudaMemsetAsync(h->d_flags + kFlagOverflow, 0, sizeof(int), h->stream));
      h->want_fields = phi || evec || keep;
      h->want_status = true;
      const int s = mmnb_compute_device(h, h->d_r, h->d_f, h->d_energy);
      h->want_status = false;
      h->want_fields = false;
      if (s)
        return s;
    }
    // the energies and flags come through the mapped status block (a row
    // overflow means evaluating again); the forces follow in chunks, each
    // added to f while the next one is in flight
    static_assert(4 + (kFlagCount + 1) / 2 <= mmnb_handle::kStatusReady, "status block");
    CK(cudaEventRecord(h->ev_eval, h->stream));
    const int nch = mmnb_handle::kChunks;
    const size_t per = (n3 + nch - 1) / nch;
    for (int c = 0; c < nch; c++) {
      const size_t b = std::min(n3, c * per), en = std::min(n3, b + per);
      if (en > b)
        CK(cudaMemcpyAsync(h->h_f + b, h->d_f + b, sizeof(double) * (en - b), cudaMemcpyDeviceToHost, h->stream));
      CK(cudaEventRecord(h->ev_chunk[c], h->stream));
    }
    if (phi)
      CK(cudaMemcpyAsync(phi, h->d_phi, sizeof(double) * h->nsite, cudaMemcpyDeviceToHost, h->stream));
    if (evec)
      CK(cudaMemcpyAsync(evec, h->d_evec, sizeof(double) * n3, cudaMemcpyDeviceToHost, h->stream));
    // while the device works: drop the staging buffer's lines from the host
    // caches (the last call's adds read them), so that the copies into it do
    // not have to snoop them
    if (f && n3 * sizeof(double) >= (1u << 20))
      evict_host_lines(h->h_f, sizeof(double) * n3);
    // the status block's ready word; the event only tells a failed
    // evaluation apart
    for (unsigned it = 1; *ready == 0ull; it++) {
      if ((it & 255u) != 0)
        continue;
      const cudaError_t q = cudaEventQuery(h->ev_eval);
      if (q == cudaErrorNotReady)
        continue;
      if (q != cudaSuccess)
        return fail(h, MMNB_ERR_CUDA, std::string("evaluation: ") + cudaGetErrorString(q));
      if (*ready == 0ull)
        return fail(h, MMNB_ERR_CUDA, "the evaluation ended without writing its status");
    }
    std::atomic_thread_fence(std::memory_order_acquire);
    memcpy(h->h_out, h->h_status, 4 * sizeof(double));
    memcpy(h->h_flags, h->h_status + 4, sizeof(int) * kFlagCount);
    h->rebuilds = h->h_flags[5];
    if (h->h_flags[kFlagError]) {
      // a device-side check failed (non-finite site coordinates): nothing is
      // added to f or u, the flag is cleared and the handle stays usable
      CK(cudaStreamSynchronize(h->stream));
      CK(cudaMemsetAsync(h->d_flags + kFlagError, 0, sizeof(int), h->stream));
      CK(cudaStreamSynchronize(h->stream));
      return fail(h, MMNB_ERR_DEVICE, "a site coordinate is not finite (NaN or infinite)");
    }
    if (h->h_flags[kFlagOverflow] > 0) {
      // a row outgrew its capacity: grow, force a rebuild, evaluate again (the
      // evaluation on cut rows is not returned, so it is not counted either)
      CK(cudaStreamSynchronize(h->stream));
      h->h_flags[kFlagTruncEvals] -= 1;
      CK(cudaMemcpy(h->d_flags + kFlagTruncEvals, h->h_flags + kFlagTruncEvals, sizeof(int),
                    cudaMemcpyHostToDevice));
      const int need = h->h_flags[kFlagOverflow];
      int st = alloc_rows(h, (need + need / 4 + 63) / 32 * 32);
      if (st)
        return st;
      h->force_rebuild_next = 1;
      h->evals--;
      continue;
    }
    for (int c = 0; c < nch; c++) {
      CK(cudaEventSynchronize(h->ev_chunk[c]));
      const size_t b = std::min(n3, c * per), en = std::min(n3, b + per);
      if (f && en > b)
        add_forces(f, h->h_f, b, en);
    }
    CK(cudaStreamSynchronize(h->stream));
    if (u)
      *u += h->h_out[3];
    if (e) {
      e->elec = h->h_out[0];
      e->lj = h->h_out[1];
      e->lj_correction = h->h_out[2];
      e->total = h->h_out[3];
    }
    h->grad_ready = keep;
    return MMNB_OK;
  }
  return fail(h, MMNB_ERR_OVERFLOW, "neighbour rows overflowed twice");
}

int mmnb_compute(mmnb_handle *h, const double *r, double *f, double *u, mmnb_energy *e, double *phi, double *evec)
{
  return compute_host(h, r, f, u, e, phi, evec, false);
}

int mmnb_forward(mmnb_handle *h, const double *r, double *f, double *u, mmnb_energy *e)
{
  return compute_host(h, r, f, u, e, nullptr, nullptr, true);
}

__global__ void k_scale_green(long nk, double s, double *green, double *kvec)
{
  const long g = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nk)
    return;
  green[g] /= s;
  kvec[3 * g] /= s;
  kvec[3 * g + 1] /= s;
  kvec[3 * g + 2] /= s;
}

int mmnb_scale(mmnb_handle *h, double s)
{
  if (!h || !(s > 0))
    return fail(h, MMNB_ERR_ARG, "scale factor must be > 0");
  {
    // the scaled box must still hold the cutoff (ElecLJ::init's rule,
    // src/eleclj.cpp:168-182) and the listed range within half its smallest
    // edge (minimum image); refused with the handle unchanged
    const double dmin = s * h->min_diameter;
    if (h->rc > 0.49 * dmin)
      return fail(h, MMNB_ERR_CUTOFF, "after scaling by " + std::to_string(s) +
                                          ", rspace_cutoff would exceed 0.49 * minimum diameter of box");
    if (h->rc + h->nlw >= 0.5 * dmin)
      return fail(h, MMNB_ERR_CUTOFF, "after scaling by " + std::to_string(s) +
                                          ", rspace_cutoff + neighbor_list_width would reach half the box");
  }
  drop_host_graph(h);
  h->grad_ready = false;
  for (int d = 0; d < 3; d++) {
    h->box.L[d] *= s;
    h->box.invL[d] = 1 / h->box.L[d];
  }
  h->volume = h->box.L[0] * h->box.L[1] * h->box.L[2];
  h->min_diameter = std::min(std::min(h->box.L[0], h->box.L[1]), h->box.L[2]);
  h->eta *= 1 / s;
  int st;
  if ((st = setup_cheb(h)))
    return st;
  if (h->p3m) {
    const long nk = (long) h->mesh[0] * h->mesh[1] * (h->mesh[2] / 2 + 1);
    k_scale_green<<<div_up(nk, 256), 256, 0, h->stream>>>(nk, s, h->d_green, h->d_kvec);
    CK(cudaGetLastError());
    if (h->cfg.precision == MMNB_MIXED)
      CK(launch_green32(h));
  }
  if (h->kspace && (st = setup_kspace(h)))
    return st;
  if ((st = setup_cells(h)))
    return st;
  // q sum for the neutralising term
  std::vector<double> q(h->nsite);
  CK(cudaMemcpy(q.data(), h->d_q, sizeof(double) * h->nsite, cudaMemcpyDeviceToHost));
  double qsum = 0;
  for (double v : q)
    qsum += v;
  update_energy_constants(h, qsum);
  CK(cudaStreamSynchronize(h->stream));
  return MMNB_OK;
}

int mmnb_set_stream(mmnb_handle *h, void *stream)
{
  if (!h)
    return MMNB_ERR_ARG;
  drop_host_graph(h);
  CK(cudaStreamSynchronize(h->stream));
  h->stream = stream ? (cudaStream_t) stream : h->own_stream;
  if (h->plan_r2c)
    CKFFT(cufftSetStream(h->plan_r2c, h->stream));
  if (h->plan_c2r)
    CKFFT(cufftSetStream(h->plan_c2r, h->stream));
  if (h->plan_r2c32)
    CKFFT(cufftSetStream(h->plan_r2c32, h->stream));
  if (h->plan_c2r32)
    CKFFT(cufftSetStream(h->plan_c2r32, h->stream));
  return MMNB_OK;
}

int mmnb_get_pairlist(mmnb_handle *h, long *npairs, int *pairs, long cap)
{
  if (!h || !npairs)
    return fail(h, MMNB_ERR_ARG, "null argument");
  if (h->evals == 0)
    return fail(h, MMNB_ERR_STATE, "no evaluation yet");
  std::vector<int> cnt(h->ngroup), sorted(h->ngroup), rows((size_t) h->ngroup * h->rowcap);
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaMemcpy(cnt.data(), h->d_nbr_count, sizeof(int) * h->ngroup, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sorted.data(), h->d_sorted, sizeof(int) * h->ngroup, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(rows.data(), h->d_nbr, sizeof(int) * rows.size(), cudaMemcpyDeviceToHost));
  long k = 0;
  for (int p = 0; p < h->ngroup; p++) {
    const int gi = sorted[p];
    for (int e = 0; e < cnt[p]; e++) {
      const int gj = sorted[rows[(size_t) p * h->rowcap + e]];
      if (gi < gj) {
        if (pairs && k < cap) {
          pairs[2 * k] = gi;
          pairs[2 * k + 1] = gj;
        }
        k++;
      }
    }
  }
  *npairs = k;
  return MMNB_OK;
}

int mmnb_get_cells(mmnb_handle *h, int *cell_of_group, int *ncell_per_dim)
{
  if (!h)
    return MMNB_ERR_ARG;
  if (ncell_per_dim)
    *ncell_per_dim = h->cg.n;
  if (cell_of_group) {
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(cell_of_group, h->d_cell_of_group, sizeof(int) * h->ngroup, cudaMemcpyDeviceToHost));
  }
  return MMNB_OK;
}

int mmnb_get_counters(mmnb_handle *h, long *rebuilds, long *evaluations)
{
  if (!h)
    return MMNB_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  int fl[kFlagCount];
  CK(cudaMemcpy(fl, h->d_flags, sizeof(fl), cudaMemcpyDeviceToHost));
  if (rebuilds)
    *rebuilds = fl[5];
  if (evaluations)
    *evaluations = fl[4];
  return MMNB_OK;
}

int mmnb_check(mmnb_handle *h, long *truncated, int *max_row)
{
  if (!h)
    return MMNB_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  int fl[kFlagCount];
  CK(cudaMemcpy(fl, h->d_flags, sizeof(fl), cudaMemcpyDeviceToHost));
  if (truncated)
    *truncated = fl[kFlagTruncEvals];
  if (max_row)
    *max_row = std::max(fl[kFlagMaxRow], fl[kFlagOverflow]);
  // cleared for the next period; the sticky longest-row record stays
  const int zero[2] = {0, 0};
  CK(cudaMemcpy(h->d_flags + kFlagError, zero, sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_flags + kFlagTruncEvals, zero, sizeof(int), cudaMemcpyHostToDevice));
  if (fl[kFlagError])
    return fail(h, MMNB_ERR_DEVICE, "a site coordinate was not finite (NaN or infinite) in an evaluation");
  if (fl[kFlagTruncEvals] > 0) {
    // grow the rows and rebuild at the next evaluation; graphs captured before
    // hold the old rows and are refused until captured again
    const int need = std::max(fl[kFlagOverflow], fl[kFlagMaxRow]);
    int st = alloc_rows(h, (need + need / 4 + 63) / 32 * 32);
    if (st)
      return st;
    CK(cudaMemcpy(h->d_flags + kFlagOverflow, zero, sizeof(int), cudaMemcpyHostToDevice));
    // a device-side request, so a graph captured after this does not carry it
    const int one = 1;
    CK(cudaMemcpy(h->d_flags + kFlagForceRebuild, &one, sizeof(int), cudaMemcpyHostToDevice));
    return fail(h, MMNB_ERR_OVERFLOW,
                std::to_string(fl[kFlagTruncEvals]) + " evaluation(s) ran on neighbour rows cut at their capacity (" +
                    std::to_string(need) + " entries needed); the rows have been regrown and the next evaluation "
                    "rebuilds the list");
  }
  return MMNB_OK;
}

int mmnb_get_launches(mmnb_handle *h, long *launches)
{
  if (!h || !launches)
    return MMNB_ERR_ARG;
  *launches = h->launches;
  return MMNB_OK;
}

int mmnb_get_settings(mmnb_handle *h, double *rc, double *nlw, double *eta, int mesh[3])
{
  if (!h)
    return MMNB_ERR_ARG;
  if (rc)
    *rc = h->rc;
  if (nlw)
    *nlw = h->nlw;
  if (eta)
    *eta = h->eta;
  if (mesh)
    for (int d = 0; d < 3; d++)
      mesh[d] = h->mesh[d];
  return MMNB_OK;
}

int mmnb_get_error_estimates(mmnb_handle *h, double *rspace, double *kspace)
{
  if (!h)
    return MMNB_ERR_ARG;
  const double l = cbrt(h->volume);
  if (rspace)
    *rspace = h->cfg.include_rspace ? 2 / sqrt(h->rc / l) * exp(-sq(h->rc * h->eta)) : 0.0;
  if (kspace) {
    const double kc = h->cfg.kspace_cutoff;
    *kspace = !h->cfg.include_kspace ? 0.0
              : h->p3m               ? h->p3m_chi
                                     : h->eta * l / M_PI * sqrt(8 / kc) * exp(-sq(M_PI * kc / (h->eta * l)));
  }
  return MMNB_OK;
}

int mmnb_set_timing(mmnb_handle *h, int on)
{
  if (!h)
    return MMNB_ERR_ARG;
  CK(cudaStreamSynchronize(h->stream));
  h->timing.on = on != 0;
  h->timing.used = 0;
  h->timing.names.clear();
  return MMNB_OK;
}

int mmnb_get_timing(mmnb_handle *h, double *ms, int nmax, char *names, int cap)
{
  if (!h)
    return -MMNB_ERR_ARG;
  Timing &t = h->timing;
  if (cudaStreamSynchronize(h->stream) != cudaSuccess)
    return -MMNB_ERR_CUDA;
  std::vector<std::string> order;
  std::vector<double> total;
  int nevals = 0;
  for (size_t k = 0; k < t.used; k++) {
    if (t.names[k] == "start") {
      nevals++;
      continue;
    }
    if (k == 0)
      continue;
    float dt = 0;
    cudaEventElapsedTime(&dt, t.pool[k - 1], t.pool[k]);
    size_t i = 0;
    while (i < order.size() && order[i] != t.names[k])
      i++;
    if (i == order.size()) {
      order.push_back(t.names[k]);
      total.push_back(0);
    }
    total[i] += dt;
  }
  std::string all;
  for (size_t i = 0; i < order.size(); i++) {
    if (ms && (int) i < nmax)
      ms[i] = nevals ? total[i] / nevals : 0;
    if (i)
      all += ",";
    all += order[i];
  }
  if (names && cap > 0) {
    strncpy(names, all.c_str(), cap - 1);
    names[cap - 1] = 0;
  }
  return (int) order.size();
}

int mmnb_destroy(mmnb_handle *h)
{
  if (!h)
    return MMNB_OK;
  if (h->stream)
    cudaStreamSynchronize(h->stream);
  free_all(h);
  if (h->own_stream)
    cudaStreamDestroy(h->own_stream);
  delete h;
  return MMNB_OK;
}

const char *mmnb_last_error(const mmnb_handle *h)
{
  return h ? h->err.c_str() : g_create_error.c_str();
}

const char *mmnb_status_string(int status)
{
  switch (status) {
  case MMNB_OK: return "ok";
  case MMNB_ERR_ARG: return "bad argument";
  case MMNB_ERR_CUDA: return "CUDA error";
  case MMNB_ERR_UNSUPPORTED: return "unsupported option";
  case MMNB_ERR_CUTOFF: return "cutoff too large for the box";
  case MMNB_ERR_OVERFLOW: return "neighbour list overflow";
  case MMNB_ERR_STATE: return "call out of order";
  case MMNB_ERR_TIMEOUT: return "device wait timed out";
  case MMNB_ERR_DEVICE: return "device-side check failed";
  default: return "unknown status";
  }
}

int mmnb_chebyshev_table(double rc, double eta, double *min, double *max, double *inv_dx, double *coeff)
{
  if (!min || !max || !inv_dx || !coeff || !(rc > 0) || !(eta > 0))
    return MMNB_ERR_ARG;
  chebyshev_table(rc, eta, min, max, inv_dx, coeff);
  return MMNB_OK;
}

int mmnb_p3m_mesh_size(double a, double grid_spacing)
{
  if (!(a > 0) || !(grid_spacing > 0))
    return 0;
  return near_2357(floor(a / grid_spacing + 0.5));
}

// ---- launch tuning ----------------------------------------------------------------

// average time of `iters` replays of a graph of one evaluation at h->d_r
static int time_evaluation(mmnb_handle *h, int iters, float *ms)
{
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  h->capturing = true;
  const long ev = h->evals, ln = h->launches;
  const int s = mmnb_compute_device(h, h->d_r, h->d_f, h->d_energy);
  h->capturing = false;
  const cudaError_t ec = cudaStreamEndCapture(h->stream, &g);
  h->evals = ev;
  h->launches = ln;
  if (s || ec != cudaSuccess) {
    if (g)
      cudaGraphDestroy(g);
    return s ? s : fail(h, MMNB_ERR_CUDA, cudaGetErrorString(ec));
  }
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t e = cudaGraphInstantiate(&ge, g, cudaGraphInstantiateFlagUseNodePriority);
  if (e == cudaSuccess)
    e = cudaEventCreate(&a);
  if (e == cudaSuccess)
    e = cudaEventCreate(&b);
  for (int k = 0; k < 2 && e == cudaSuccess; k++)
    e = cudaGraphLaunch(ge, h->stream);
  if (e == cudaSuccess)
    e = cudaEventRecord(a, h->stream);
  for (int k = 0; k < iters && e == cudaSuccess; k++)
    e = cudaGraphLaunch(ge, h->stream);
  if (e == cudaSuccess)
    e = cudaEventRecord(b, h->stream);
  if (e == cudaSuccess)
    e = cudaEventSynchronize(b);
  if (e == cudaSuccess)
    e = cudaEventElapsedTime(ms, a, b);
  if (a)
    cudaEventDestroy(a);
  if (b)
    cudaEventDestroy(b);
  if (ge)
    cudaGraphExecDestroy(ge);
  cudaGraphDestroy(g);
  if (e != cudaSuccess)
    return fail(h, MMNB_ERR_CUDA, std::string("tuning: ") + cudaGetErrorString(e));
  *ms /= iters;
  return MMNB_OK;
}

int mmnb_autotune(mmnb_handle *h, const double *r, int iters)
{
  if (!h || !r || iters < 1)
    return fail(h, MMNB_ERR_ARG, "null handle or positions, or iters < 1");
  if (!h->params_set)
    return fail(h, MMNB_ERR_STATE, "mmnb_set_params has not been called");
  int s;
  if (h->first && (s = mmnb_compute(h, r, nullptr, nullptr, nullptr, nullptr, nullptr)))
    return s;
  const size_t n3 = 3 * (size_t) h->nsite;
  CK(cudaMemcpyAsync(h->d_r, r, sizeof(double) * n3, cudaMemcpyHostToDevice, h->stream));
  const bool mixed = h->cfg.precision == MMNB_MIXED;
  const bool p3m = h->p3m && h->any_q && h->cfg.include_kspace;
  // one knob at a time, each over its values, keeping the best so far
  struct Knob {
    int *v;
    int nval;
    int vals[3];
    bool on;
  } knobs[] = {{&h->tune.water_minb, 2, {5, 4}, mixed && h->water},
               {&h->tune.spread_planes, 3, {2, 0, 1}, mixed && p3m},
               {&h->tune.p3m_side, 2, {1, 0}, p3m},
               {&h->tune.water64_warps, 3, {12, 10, 8}, !mixed && h->water && h->cfg.include_rspace}};
  for (Knob &k : knobs) {
    if (!k.on)
      continue;
    int best = *k.v;
    float best_ms = 0;
    for (int c = 0; c < k.nval; c++) {
      *k.v = k.vals[c];
      float ms = 0;
      if ((s = time_evaluation(h, iters, &ms)))
        return s;
      if (c == 0 || ms < best_ms) {
        best_ms = ms;
        best = k.vals[c];
      }
    }
    *k.v = best;
  }
  drop_host_graph(h);
  CK(cudaStreamSynchronize(h->stream));
  return MMNB_OK;
}

int mmnb_get_tuning(mmnb_handle *h, int tuning[4])
{
  if (!h || !tuning)
    return MMNB_ERR_ARG;
  tuning[0] = h->tune.water_minb;
  tuning[1] = h->tune.spread_planes;
  tuning[2] = h->tune.p3m_side;
  tuning[3] = h->tune.water64_warps;
  return MMNB_OK;
}

int mmnb_set_tuning(mmnb_handle *h, const int tuning[4])
{
  if (!h || !tuning || (tuning[0] != 4 && tuning[0] != 5) || tuning[1] < 0 || tuning[1] > 2 ||
      (tuning[2] != 0 && tuning[2] != 1) || (tuning[3] != 8 && tuning[3] != 10 && tuning[3] != 12))
    return fail(h, MMNB_ERR_ARG,
                "tuning values: water blocks 4 or 5, spread layout 0, 1 or 2, P3M side 0 or 1, FP64 water warps "
                "8, 10 or 12");
  h->tune.water_minb = tuning[0];
  h->tune.spread_planes = tuning[1];
  h->tune.p3m_side = tuning[2];
  h->tune.water64_warps = tuning[3];
  drop_host_graph(h);
  return MMNB_OK;
}

}  // extern "C"

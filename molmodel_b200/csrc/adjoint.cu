// Per-site parameter gradients of one evaluation (mmnb_forward, then
// mmnb_site_gradients), for the force-field fits the reference runs on its
// per-type parameters (WeakCouple::update, src/msimprog.cpp:855-876; BCIFit,
// src/bcifit.cpp:44-123; types mapped to sites by ElecLJ::types_changed,
// src/eleclj.cpp:440-503).
//
// Energy.  Every electrostatic term (switched real-space pairs, reciprocal
// space, exclusion and 1-4 corrections, self and neutralising terms) is
// q^T K q / 2 with K symmetric, and the forward's site potential is
// phi = K q, so dU/dq_i = phi_i.  LJ pair energies are S(R) u(r) with
// u = A/r^12 - B/r^6, A = 4 eps_ij sig_ij^12, B = 4 eps_ij sig_ij^6,
// eps_ij = sqrt(eps_i eps_j), sig_ij = sqrt(sig_i sig_j) or (sig_i + sig_j)/2:
// dA/dsig_i = 2 k A, dB/dsig_i = k B with k = 3/sig_i (geometric) or
// 6/(sig_i + sig_j), and dA/deps_i = A/(2 eps_i), likewise B.
//
// Loss of the forces, g = dL/dF.  For a group pair (I, J) inside the cutoff
// the forward puts q_a q_b S b1 d_ab on site a (d_ab = r_a - r_b with the
// anchors' image shift, b1 = -(1/r) d/dr of the pair kernel) and the switch
// force ds R T on the anchors (R the anchor displacement, T the summed
// unswitched pair energies, ds = -2 dS/dR^2), opposite on J's side.  Hence
//   dL/dq_i = g_i . E_i + sum_J [ -S sum_b q_b b1 (g_b . d_ib)
//                                 + ds (g_A - g_B) . R sum_b q_b b0_ib ]
//             + (the same dipole term for exclusion and 1-4 partners)
//             + (the reciprocal-space potential of the dipoles q_j g_j),
// with E_i the forward's field; and for LJ
//   dL/dsig_i = sum_J sum_b [ S du'_ib (g_i - g_b) . d_ib + ds (g_A - g_B) . R u'_ib ]
// where ' is d/dsig_i (d/deps_i alike).  The list is full (each group pair
// in both rows), and every term above acts on the row's own sites, so one
// warp per row writes its sites' sums with plain stores: no atomics, a fixed
// summation order, the same rows and cutoff decisions as the forward.  The
// reciprocal-space dipole solve is in pppm.cu / kspace.cu; the LJ tail
// correction (linear in the class totals A and B) is added on the host.

#include <cmath>
#include <vector>

#include "mmnb_internal.cuh"

namespace mmnb {

constexpr int kGradWarps = 4;
constexpr int kGradThreads = 128;
constexpr int kGradQueue = 64;  // per warp: at most 31 carried over plus 32 new

// per-site output slots of the scratch area (each nsite doubles)
enum GradSlot { kDuDq = 0, kDuDsig, kDuDeps, kDlDq, kDlDsig, kDlDeps, kGradSlots };

struct GradArgs {
  int nsite, ngroup, rowcap, geometric;
  Box box;
  double rlo2, rhi2, inv_sw, eta;
  double cheb_min, cheb_max, cheb_inv_dx;
  const double *cheb;
  // the rigid-water forward's copy of the table: the cubics' (c0, c1) and
  // (c2, c3), continued to (rc + 2.5)^2 (k_grad_pair)
  const double2 *tw0, *tw1;
  double nsegw;
  const double *r, *q, *sig, *eps, *rscreen;
  const double *g;  // dL/dF, 3 per site, or null
  const int *mask, *nbr, *nbr_count, *sorted, *group;
  const int *gexcl_ptr, *gexcl_idx, *excl_ptr, *excl_idx, *p14_ptr, *p14_idx;
  double e14, l14;
  int scale_e14, scale_l14, do14;
  double *out;      // kGradSlots x nsite
};

// LJ pair energy u, force scalar du (force = du d), and their sigma_i
// derivatives us, dus (eps_i derivatives: u / (2 eps_i), du / (2 eps_i))
struct LJd {
  double u, du, us, dus;
};

__device__ __forceinline__ LJd lj_terms(double si, double sj, double ei, double ej, int geometric, double r2)
{
  double sg, kap;
  if (geometric) {
    sg = si * sj;
    kap = 3 / si;
  } else {
    const double hs = 0.5 * (si + sj);
    sg = hs * hs;
    kap = 6 / (si + sj);
  }
  const double s6 = sg * sg * sg;
  const double b = 4 * sqrt(ei * ej) * s6, aa = b * s6;
  const double ir2 = 1.0 / r2, ir6 = ir2 * ir2 * ir2;
  const double a12 = aa * ir6 * ir6, b6 = b * ir6;
  LJd t;
  t.u = a12 - b6;
  t.du = (12 * a12 - 6 * b6) * ir2;
  t.us = kap * (2 * a12 - b6);
  t.dus = kap * (24 * a12 - 6 * b6) * ir2;
  return t;
}

// b0 = erfc(eta r)/r from the table's cubic and b1 = -(2 / dx) d b0/d(segment
// position) from its derivative: the reference stores b1's quadratic as
// exactly that derivative (-2 k c_k / dx, k = 1..3), so half the table is
// read; outside the table the exact functions
__device__ __forceinline__ void ewald_grad_b(const GradArgs &a, double r2, double &b0, double &b1)
{
  const double x = (r2 - a.cheb_min) * a.cheb_inv_dx;
  if (x > 0 && x < a.nsegw) {
    const int i = (int) x;
    const double f = x - i;
    const double2 c01 = __ldg(a.tw0 + i), c23 = __ldg(a.tw1 + i);
    b0 = ((c23.y * f + c23.x) * f + c01.y) * f + c01.x;
    b1 = -2 * a.cheb_inv_dx * ((3 * c23.y * f + 2 * c23.x) * f + c01.y);
  } else {
    const double r = sqrt(r2);
    const double er = a.eta * r;
    b0 = erfc(er) / r;
    b1 = (b0 + a.eta * M_2_SQRTPI * exp(-(er * er))) / r2;
  }
}

__device__ __forceinline__ double3 load3(const double *p, int i)
{
  return make_double3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}

// One warp per row (sorted group p).  Lane l takes row site ia = l / P of the
// group and partner slot l % P (P = 32 / G partners per step), so each lane
// holds one row site's state.  The row's partners within rc are queued in list
// order in a per-warp ring (the anchor test of 32 entries at a time); each step
// evaluates P queued partners against every row site.  The row sites' sums are
// reduced over the warp in a fixed order at the end.
template <int G, bool SCREEN, bool GEXCL>
__global__ void __launch_bounds__(kGradWarps * 32) k_grad_pair(GradArgs a)
{
  constexpr int P = 32 / G;
  constexpr int kMask = kGradQueue - 1;
  const int lane = threadIdx.x & 31;
  const int p = blockIdx.x * kGradWarps + (threadIdx.x >> 5);
  if (p >= a.ngroup)
    return;  // the whole warp
  const int gi = a.sorted[p];
  const int si0 = a.group[2 * gi], ns = a.group[2 * gi + 1] - si0;
  const int ia = lane / P, pk = lane % P;
  const bool act = ia < G && ia < ns;
  // the row's anchor (the minimum image is taken between anchors) and this
  // lane's row site
  const double4 r0 = make_double4(a.r[3 * si0], a.r[3 * si0 + 1], a.r[3 * si0 + 2], 0);
  const double3 g0 = a.g ? load3(a.g, si0) : make_double3(0, 0, 0);
  double4 ri = make_double4(0, 0, 0, 0);
  double3 gv = make_double3(0, 0, 0);
  double sgi = 0, epi = 0, rsi = 0;
  int mi = 0;
  if (act) {
    const int s = si0 + ia;
    ri = make_double4(a.r[3 * s], a.r[3 * s + 1], a.r[3 * s + 2], a.q[s]);
    if (a.g)
      gv = load3(a.g, s);
    sgi = a.sig[s];
    epi = a.eps[s];
    rsi = a.rscreen[s];
    mi = a.mask[s];
  }
  double psi = 0, dus = 0, due = 0, dls = 0, dle = 0;
  const int cnt = a.nbr_count[p];
  const int *row = a.nbr + (size_t) p * a.rowcap;
  __shared__ double qd[kGradWarps][7][kGradQueue];
  __shared__ int qg[kGradWarps][kGradQueue];
  double(*wq)[kGradQueue] = qd[threadIdx.x >> 5];
  int *wg = qg[threadIdx.x >> 5];
  const unsigned below = (1u << lane) - 1;
  // row site ia against the queued partner in ring slot k
  auto partner = [&](int k) {
    const int gj = wg[k];
    const double x = wq[0][k], y = wq[1][k], z = wq[2][k], sx = wq[3][k], sy = wq[4][k], sz = wq[5][k];
    const double r2a = wq[6][k];
    const int sj0 = a.group[2 * gj], nsj = a.group[2 * gj + 1] - sj0;
    double S = 1, ds = 0;
    if (r2a > a.rlo2) {
      const double zz = (r2a - a.rlo2) * a.inv_sw;
      S = ((-6 * zz + 15) * zz - 10) * zz * zz * zz + 1;
      ds = ((60 * zz - 120) * zz + 60) * zz * zz * a.inv_sw;
    }
    double GR = 0;
    if (a.g && ds != 0) {
      const double3 gB = load3(a.g, sj0);
      GR = (g0.x - gB.x) * x + (g0.y - gB.y) * y + (g0.z - gB.z) * z;
    }
    bool gx = false;
    if (GEXCL)
      gx = csr_has(a.gexcl_ptr, a.gexcl_idx, gi, gj);
#pragma unroll
    for (int jb = 0; jb < G; jb++) {
      if (jb >= nsj)
        break;
      const int sj = sj0 + jb;
      const int m = mi & a.mask[sj];
      if (!m)
        continue;
      if (GEXCL && gx && csr_has(a.excl_ptr, a.excl_idx, si0 + ia, sj))
        continue;
      const double xj = a.r[3 * sj], yj = a.r[3 * sj + 1], zj = a.r[3 * sj + 2];
      const double3 gj3 = a.g ? load3(a.g, sj) : make_double3(0, 0, 0);
      double dx, dy, dz, r2;
      if (ia == 0 && jb == 0) {
        dx = x;
        dy = y;
        dz = z;
        r2 = r2a;
      } else {
        dx = (ri.x + sx) - xj;
        dy = (ri.y + sy) - yj;
        dz = (ri.z + sz) - zj;
        r2 = dx * dx + dy * dy + dz * dz;
      }
      if (m & MMNB_SITE_HAS_Q) {
        double b0, b1;
        ewald_grad_b(a, r2, b0, b1);
        if (SCREEN) {
          const double rs = rsi + a.rscreen[sj];
          if (r2 < rs * rs) {
            const double invr = 1.0 / sqrt(r2);
            const double inv3 = 1.0 / (rs * rs * rs);
            b0 += (-0.5 * r2 * inv3 + 1.5 / rs) - invr;
            b1 += inv3 - invr * invr * invr;
          }
        }
        const double gjd = gj3.x * dx + gj3.y * dy + gj3.z * dz;
        psi += a.q[sj] * (ds * GR * b0 - S * b1 * gjd);
      }
      if (m & MMNB_SITE_HAS_LJ) {
        const LJd t = lj_terms(sgi, a.sig[sj], epi, a.eps[sj], a.geometric, r2);
        const double gd = (gv.x - gj3.x) * dx + (gv.y - gj3.y) * dy + (gv.z - gj3.z) * dz;
        dus += S * t.us;
        due += S * t.u;
        dls += S * t.dus * gd + ds * GR * t.us;
        dle += S * t.du * gd + ds * GR * t.u;
      }
    }
  };
  int head = 0, qn = 0;  // ring entries [head, head + qn)
  for (int base = 0; base < cnt; base += 32) {
    const int e = base + lane;
    bool take = false;
    double x = 0, y = 0, z = 0, sx = 0, sy = 0, sz = 0, r2a = 0;
    int gj = 0;
    if (e < cnt) {
      gj = a.sorted[row[e]];
      const int sj0 = a.group[2 * gj];
      const double4 rjA = make_double4(a.r[3 * sj0], a.r[3 * sj0 + 1], a.r[3 * sj0 + 2], 0);
      r2a = anchor_disp(a.box, r0, rjA, x, y, z, sx, sy, sz);
      take = r2a <= a.rhi2;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, take);
    if (take) {
      const int k = (head + qn + __popc(bal & below)) & kMask;
      wq[0][k] = x;
      wq[1][k] = y;
      wq[2][k] = z;
      wq[3][k] = sx;
      wq[4][k] = sy;
      wq[5][k] = sz;
      wq[6][k] = r2a;
      wg[k] = gj;
    }
    qn += __popc(bal);
    __syncwarp();
    for (; qn >= P; qn -= P, head = (head + P) & kMask) {
      if (act)
        partner((head + pk) & kMask);
      __syncwarp();  // the slots are free again only after every lane has read them
    }
  }
  if (act && pk < qn)
    partner((head + pk) & kMask);
  // each row site's sums over its lanes (the other lanes add zero), in a fixed order
  const size_t n = a.nsite;
#pragma unroll
  for (int t = 0; t < G; t++) {
    double v[5] = {ia == t ? psi : 0.0, ia == t ? dus : 0.0, ia == t ? due : 0.0, ia == t ? dls : 0.0,
                   ia == t ? dle : 0.0};
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
      for (int c = 0; c < 5; c++)
        v[c] += __shfl_xor_sync(0xffffffffu, v[c], off);
    if (lane == 0 && t < ns) {
      const int s = si0 + t;
      a.out[kDlDq * n + s] += v[0];
      a.out[kDuDsig * n + s] += v[1];
      a.out[kDuDeps * n + s] += v[2];
      a.out[kDlDsig * n + s] += v[3];
      a.out[kDlDeps * n + s] += v[4];
    }
  }
}

// exclusion corrections and 1-4 pairs, one thread per site over its own
// partners (the forward's k_exclusions_fp64 terms)
__global__ void __launch_bounds__(kGradThreads) k_grad_excl(GradArgs a)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nsite)
    return;
  const int mi = a.mask[i];
  const double xi = a.r[3 * i], yi = a.r[3 * i + 1], zi = a.r[3 * i + 2];
  const double3 gi = a.g ? load3(a.g, i) : make_double3(0, 0, 0);
  double psi = 0, dus = 0, due = 0, dls = 0, dle = 0;
  if ((mi & MMNB_SITE_HAS_Q) && a.g) {
    for (int n = a.excl_ptr[i]; n < a.excl_ptr[i + 1]; n++) {
      const int j = a.excl_idx[n];
      if (!(a.mask[j] & MMNB_SITE_HAS_Q))
        continue;
      double x = xi - a.r[3 * j], y = yi - a.r[3 * j + 1], z = zi - a.r[3 * j + 2];
      min_image_ref(a.box, x, y, z);
      const double r2 = x * x + y * y + z * z;
      const double rm = sqrt(r2);
      const double er = a.eta * rm;
      const double b0 = -erf(er) / rm;
      const double b1 = (b0 + a.eta * M_2_SQRTPI * exp(-(er * er))) / r2;
      const double3 gj = load3(a.g, j);
      psi -= a.q[j] * b1 * (gj.x * x + gj.y * y + gj.z * z);
    }
  }
  if (a.do14) {
    for (int n = a.p14_ptr[i]; n < a.p14_ptr[i + 1]; n++) {
      const int j = a.p14_idx[n];
      const int m = mi & a.mask[j];
      double x = xi - a.r[3 * j], y = yi - a.r[3 * j + 1], z = zi - a.r[3 * j + 2];
      min_image_ref(a.box, x, y, z);
      const double r2 = x * x + y * y + z * z;
      const double3 gj = a.g ? load3(a.g, j) : make_double3(0, 0, 0);
      if ((m & MMNB_SITE_HAS_Q) && a.g) {
        const double rs = a.rscreen[i] + a.rscreen[j];
        double b1;
        if (r2 < rs * rs) {
          b1 = 1.0 / (rs * rs * rs);
        } else {
          const double invr = 1.0 / sqrt(r2);
          b1 = invr * invr * invr;
        }
        if (a.scale_e14)
          b1 *= a.e14;
        psi -= a.q[j] * b1 * (gj.x * x + gj.y * y + gj.z * z);
      }
      if (m & MMNB_SITE_HAS_LJ) {
        const LJd t = lj_terms(a.sig[i], a.sig[j], a.eps[i], a.eps[j], a.geometric, r2);
        const double l = a.scale_l14 ? a.l14 : 1.0;
        const double gd = (gi.x - gj.x) * x + (gi.y - gj.y) * y + (gi.z - gj.z) * z;
        dus += l * t.us;
        due += l * t.u;
        dls += l * t.dus * gd;
        dle += l * t.du * gd;
      }
    }
  }
  const size_t n = a.nsite;
  a.out[kDlDq * n + i] += psi;
  a.out[kDuDsig * n + i] += dus;
  a.out[kDuDeps * n + i] += due;
  a.out[kDlDsig * n + i] += dls;
  a.out[kDlDeps * n + i] += dle;
}

// dU/dq_i = phi_i; dL/dq_i += g_i . E_i; epsilon sums / (2 eps_i); zero on
// sites without the parameter
__global__ void k_grad_finish(int nsite, const int *__restrict__ mask, const double *__restrict__ eps,
                              const double *__restrict__ g, const double *__restrict__ phi,
                              const double *__restrict__ evec, double *__restrict__ out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsite)
    return;
  const size_t n = nsite;
  const int m = mask[i];
  if (m & MMNB_SITE_HAS_Q) {
    out[kDuDq * n + i] = phi[i];
    if (g)
      out[kDlDq * n + i] += g[3 * i] * evec[3 * i] + g[3 * i + 1] * evec[3 * i + 1] + g[3 * i + 2] * evec[3 * i + 2];
  } else {
    out[kDuDq * n + i] = 0;
    out[kDlDq * n + i] = 0;
  }
  if ((m & MMNB_SITE_HAS_LJ) && eps[i] > 0) {
    const double inv = 0.5 / eps[i];
    out[kDuDeps * n + i] *= inv;
    out[kDlDeps * n + i] *= inv;
  } else {
    out[kDuDsig * n + i] = 0;
    out[kDuDeps * n + i] = 0;
    out[kDlDsig * n + i] = 0;
    out[kDlDeps * n + i] = 0;
  }
}

template <int G>
static void launch_grad_pair_g(mmnb_handle *h, const GradArgs &a)
{
  const int blocks = div_up(h->ngroup, kGradWarps);
  if (h->has_rscreen) {
    if (h->any_gexcl)
      k_grad_pair<G, true, true><<<blocks, kGradWarps * 32, 0, h->stream>>>(a);
    else
      k_grad_pair<G, true, false><<<blocks, kGradWarps * 32, 0, h->stream>>>(a);
  } else {
    if (h->any_gexcl)
      k_grad_pair<G, false, true><<<blocks, kGradWarps * 32, 0, h->stream>>>(a);
    else
      k_grad_pair<G, false, false><<<blocks, kGradWarps * 32, 0, h->stream>>>(a);
  }
  h->launches += 1;
}

// FP64 meshes and plans of the dipole solve: the FP64 form's own (the forward
// has finished with them), or, for the mixed form, a set made on first use
static int grad_p3m_scratch(mmnb_handle *h, P3mScratch &s)
{
  const size_t nr = (size_t) h->mesh[0] * h->mesh[1] * h->mesh[2];
  const size_t nk = (size_t) h->mesh[0] * h->mesh[1] * (h->mesh[2] / 2 + 1);
  if (h->plan_r2c) {
    s.r2c = h->plan_r2c;
    s.c2r = h->plan_c2r;
    if (h->cfg.p3m_ik_differentiate) {
      s.spread = h->d_egrid;
      s.spreadk = h->d_egridk;
      s.solvek = h->d_meshk;
      s.solve = h->d_mesh;
    } else {
      s.spread = s.solve = h->d_mesh;
      s.spreadk = h->d_meshk;
    }
    return MMNB_OK;
  }
  // ik: three spread meshes and the summed spectrum's mesh
  const int nm = h->cfg.p3m_ik_differentiate ? 4 : 1;
  if (!h->gplan_r2c) {
    cudaError_t e = cudaMalloc(&h->d_gmesh, sizeof(double) * nr * nm);
    if (e == cudaSuccess)
      e = cudaMalloc(&h->d_gmeshk, sizeof(cufftDoubleComplex) * nk * nm);
    if (e != cudaSuccess) {
      h->err = std::string("gradient mesh: ") + cudaGetErrorString(e);
      return MMNB_ERR_CUDA;
    }
    if (cufftPlan3d(&h->gplan_r2c, h->mesh[0], h->mesh[1], h->mesh[2], CUFFT_D2Z) != CUFFT_SUCCESS ||
        cufftPlan3d(&h->gplan_c2r, h->mesh[0], h->mesh[1], h->mesh[2], CUFFT_Z2D) != CUFFT_SUCCESS) {
      h->err = "gradient mesh: cuFFT plan";
      return MMNB_ERR_CUDA;
    }
  }
  s.r2c = h->gplan_r2c;
  s.c2r = h->gplan_c2r;
  s.spread = h->d_gmesh;
  s.spreadk = h->d_gmeshk;
  if (nm == 4) {
    s.solve = h->d_gmesh + 3 * nr;
    s.solvek = h->d_gmeshk + 3 * nk;
  } else {
    s.solve = h->d_gmesh;
  }
  return MMNB_OK;
}

}  // namespace mmnb

using namespace mmnb;

// dst[0, n) = src[0, n) on the host cores (the staging copies of a call)
static void copy_host(double *dst, const double *src, size_t n)
{
  const long m = (long) n;
#pragma omp parallel for schedule(static) if (m > (1 << 15))
  for (long i = 0; i < m; i++)
    dst[i] = src[i];
}

static int grad_fail(mmnb_handle *h, int code, const std::string &msg)
{
  if (h)
    h->err = msg;
  return code;
}

extern "C" int mmnb_site_gradients(mmnb_handle *h, const double *dl_df, double *du_dq, double *du_dsig,
                                   double *du_deps, double *dl_dq, double *dl_dsig, double *dl_deps)
{
  if (!h)
    return grad_fail(h, MMNB_ERR_ARG, "null handle");
  if (!h->grad_ready)
    return grad_fail(h, MMNB_ERR_STATE,
                     "no evaluation to differentiate: call mmnb_forward first (any other evaluation, "
                     "mmnb_set_params or mmnb_scale since then discards it)");
  const size_t n = h->nsite, n3 = 3 * n;
  const size_t nskd = h->kspace ? 2 * (size_t) h->nk : 0;
  const size_t need = kGradSlots * n + n3 + nskd;
  if (h->bwd_cap < need) {
    if (h->d_bwd)
      cudaFree(h->d_bwd);
    h->d_bwd = nullptr;
    h->bwd_cap = 0;
    if (h->h_bwd)
      cudaFreeHost(h->h_bwd);
    h->h_bwd = nullptr;
    cudaError_t ea = cudaMalloc(&h->d_bwd, need * sizeof(double));
    if (ea == cudaSuccess)
      ea = cudaMallocHost((void **) &h->h_bwd, kGradSlots * n * sizeof(double));
    if (ea != cudaSuccess)
      return grad_fail(h, MMNB_ERR_CUDA, std::string("gradient scratch: ") + cudaGetErrorString(ea));
    h->bwd_cap = need;
  }
  double *d_out = h->d_bwd, *d_g = dl_df ? h->d_bwd + kGradSlots * n : nullptr;
  double *d_skd = h->d_bwd + kGradSlots * n + n3;
  P3mScratch ps;
  const bool p3m = h->any_q && h->cfg.include_kspace && h->p3m && dl_df;
  if (p3m) {
    const int st = grad_p3m_scratch(h, ps);
    if (st)
      return st;
  }
  GradArgs a;
  a.nsite = h->nsite;
  a.ngroup = h->ngroup;
  a.rowcap = h->rowcap;
  a.geometric = h->cfg.geometric_combining_for_sigma;
  a.box = h->box;
  a.rlo2 = h->rlo2;
  a.rhi2 = h->rhi2;
  a.inv_sw = h->inv_sw;
  a.eta = h->eta;
  a.cheb_min = h->cheb_min;
  a.cheb_max = h->cheb_max;
  a.cheb_inv_dx = h->cheb_inv_dx;
  a.cheb = h->d_cheb;
  a.tw0 = reinterpret_cast<const double2 *>(h->d_cheb_w);
  a.tw1 = a.tw0 + h->cheb_w_nseg;
  a.nsegw = h->cheb_w_nseg;
  a.r = h->d_r;  // the forward's positions (host path)
  a.q = h->d_q;
  a.sig = h->d_sig;
  a.eps = h->d_eps;
  a.rscreen = h->d_rscreen;
  a.g = d_g;
  a.mask = h->d_mask;
  a.nbr = h->d_nbr;
  a.nbr_count = h->d_nbr_count;
  a.sorted = h->d_sorted;
  a.group = h->d_group;
  a.gexcl_ptr = h->d_gexcl_ptr;
  a.gexcl_idx = h->d_gexcl_idx;
  a.excl_ptr = h->d_excl_ptr;
  a.excl_idx = h->d_excl_idx;
  a.p14_ptr = h->d_p14_ptr;
  a.p14_idx = h->d_p14_idx;
  // the forward's 1-4 terms: (factor - 1) x the full pair when scaling, the
  // full pair otherwise (interact() as src/rspace.c:522-557 calls it)
  a.e14 = h->cfg.elec_1_4_scale_factor - 1;
  a.l14 = h->cfg.lj_1_4_scale_factor - 1;
  a.scale_e14 = fabs(h->cfg.elec_1_4_scale_factor - 1) > 1e-10;
  a.scale_l14 = fabs(h->cfg.lj_1_4_scale_factor - 1) > 1e-10;
  a.do14 = h->use_14 ? 1 : 0;
  a.out = d_out;
  cudaError_t e = cudaMemsetAsync(d_out, 0, sizeof(double) * kGradSlots * n, h->stream);
  if (e == cudaSuccess && d_g) {
    // through the handle's pinned force staging buffer (idle between host calls)
    copy_host(h->h_f, dl_df, n3);
    e = cudaMemcpyAsync(d_g, h->h_f, n3 * sizeof(double), cudaMemcpyHostToDevice, h->stream);
  }
  if (e == cudaSuccess && h->cfg.include_rspace) {
    switch (h->G) {
    case 1: launch_grad_pair_g<1>(h, a); break;
    case 2: launch_grad_pair_g<2>(h, a); break;
    case 3: launch_grad_pair_g<3>(h, a); break;
    case 4: launch_grad_pair_g<4>(h, a); break;
    default: launch_grad_pair_g<8>(h, a); break;
    }
    k_grad_excl<<<div_up(h->nsite, kGradThreads), kGradThreads, 0, h->stream>>>(a);
    h->launches += 1;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && d_g && h->any_q && h->cfg.include_kspace) {
    if (h->p3m)
      e = launch_p3m_dipole_fp64(h, h->d_r, d_g, ps, d_out + kDlDq * n);
    else if (h->kspace)
      e = launch_kspace_dipole(h, h->d_r, d_g, d_skd, d_out + kDlDq * n);
  }
  if (e == cudaSuccess) {
    k_grad_finish<<<div_up(h->nsite, kGradThreads), kGradThreads, 0, h->stream>>>(h->nsite, h->d_mask, h->d_eps,
                                                                                   d_g, h->d_phi, h->d_evec, d_out);
    h->launches += 1;
    e = cudaGetLastError();
  }
  double *outs[kGradSlots] = {du_dq, du_dsig, du_deps, dl_df ? dl_dq : nullptr, dl_df ? dl_dsig : nullptr,
                              dl_df ? dl_deps : nullptr};
  // the slots are contiguous: one pinned copy back, then to the caller's arrays
  const int nslot = dl_df ? kGradSlots : kDlDq;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h->h_bwd, d_out, nslot * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess)
    return grad_fail(h, MMNB_ERR_CUDA, std::string("site gradients: ") + cudaGetErrorString(e));
  for (int k = 0; k < nslot; k++)
    if (outs[k])
      copy_host(outs[k], h->h_bwd + k * n, n);
  // LJ tail: U_tail = cA totA + cB totB over the classes' (sigma, eps, count);
  // d totA / d sig_i = 2 sum_b n_b dA_ab/dsig_a for site i in class a
  if (h->cfg.include_lj_correction && (du_dsig || du_deps) && !h->cls_sig.empty()) {
    const double cA = lj_tail_ab(h, 1, 0), cB = lj_tail_ab(h, 0, 1);
    const size_t nc = h->cls_sig.size();
    std::vector<double> ts(nc, 0.0), te(nc, 0.0);
    for (size_t ca = 0; ca < nc; ca++)
      for (size_t cb = 0; cb < nc; cb++) {
        const double sa = h->cls_sig[ca], sb = h->cls_sig[cb], ea = h->cls_eps[ca], eb = h->cls_eps[cb];
        const bool geo = h->cfg.geometric_combining_for_sigma != 0;
        const double s6 = pow(geo ? sqrt(sa * sb) : 0.5 * (sa + sb), 6);
        const double kap = geo ? 3 / sa : 6 / (sa + sb);
        const double bb = 4 * sqrt(ea * eb) * s6, aa = bb * s6;
        const double nb = (double) h->cls_n[cb];
        ts[ca] += 2 * nb * (cA * 2 * kap * aa - cB * kap * bb);
        if (ea > 0)
          te[ca] += 2 * nb * (cA * aa - cB * bb) / (2 * ea);
      }
    for (size_t i = 0; i < n; i++) {
      const int c = h->site_cls[i];
      if (c < 0)
        continue;
      if (du_dsig)
        du_dsig[i] += ts[c];
      if (du_deps)
        du_deps[i] += te[c];
    }
  }
  return MMNB_OK;
}

extern "C" int mmnb_backward(mmnb_handle *h, const double *r, const double *dl_df, double *f, double *u,
                             double grad_u[3], double grad_l[3])
{
  if (!h || !r || !grad_u)
    return grad_fail(h, MMNB_ERR_ARG, "null handle, positions or gradient output");
  int s = mmnb_forward(h, r, f, u, nullptr);
  if (s)
    return s;
  const size_t n = h->nsite;
  std::vector<double> g(6 * n, 0.0);
  s = mmnb_site_gradients(h, dl_df, g.data(), g.data() + n, g.data() + 2 * n, g.data() + 3 * n, g.data() + 4 * n,
                          g.data() + 5 * n);
  if (s)
    return s;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (size_t i = 0; i < n; i++) {
    const double p[3] = {h->hq[i], h->hsig[i], h->heps[i]};
    for (int k = 0; k < 6; k++)
      acc[k] += p[k % 3] * g[k * n + i];
  }
  for (int k = 0; k < 3; k++)
    grad_u[k] = acc[k];
  if (grad_l)
    for (int k = 0; k < 3; k++)
      grad_l[k] = dl_df ? acc[3 + k] : 0;
  return MMNB_OK;
}

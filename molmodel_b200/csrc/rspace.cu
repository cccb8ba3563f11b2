// Real-space Ewald + Lennard-Jones, FP64 form.
//
// Replaces RSpaceEwald (src/rspace.c:382-558).  Semantics kept from the
// reference:
//   * cutoff, switching and minimum image are decided per GROUP pair from the
//     two anchor sites; every site pair of the group pair uses the anchors'
//     image shift (src/rspace.c:423-478);
//   * the quintic switch S(z), z = (r^2 - rlo^2)/(rhi^2 - rlo^2), multiplies
//     both Coulomb and LJ terms; the switch derivative times the summed
//     unswitched energy acts on the anchors only (:479-489);
//   * erfc(eta r)/r and its -2 d/d(r^2) come from the reference's own
//     512-segment Chebyshev table inside its range, from erfc/exp outside
//     (:104-156);
//   * excluded site pairs are skipped only inside group pairs that contain an
//     exclusion (group_excluded, :422, 446, 465), and every excluded charged
//     pair gets the -erf(eta r)/r correction (:492-521);
//   * 1-4 pairs get scaled plain Coulomb + LJ (:522-557).
//
// Layout: the neighbour list is full (both directions); one warp owns one
// group row, its 32 lanes stride over the row's partners, and each lane
// accumulates only the row group's sites.  A warp shuffle reduction then
// gives each site its total, written once with plain stores — no atomics, and
// the summation order is fixed, so results are bitwise reproducible.

#include "mmnb_internal.cuh"

namespace mmnb {

struct PairArgs {
  int ngroup, rowcap, geometric;
  Box box;
  double rlo2, rhi2, eta;
  double cheb_min, cheb_max, cheb_inv_dx;
  const double *cheb;
  const double4 *sr;   // x, y, z, q        (sorted, padded)
  const double4 *sp;   // sig, eps, rscreen, mask
  const int *nbr, *nbr_count, *sorted, *group;
  const int *gexcl_ptr, *gexcl_idx, *excl_ptr, *excl_idx;
  double *phi, *evec, *ljf, *lj_part;
};

__device__ __forceinline__ bool csr_has(const int *ptr, const int *idx, int row, int key)
{
  int lo = ptr[row], hi = ptr[row + 1] - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int v = idx[mid];
    if (key < v)
      hi = mid - 1;
    else if (key > v)
      lo = mid + 1;
    else
      return true;
  }
  return false;
}

// b0 = erfc(eta r)/r, b1 = (b0 + 2 eta/sqrt(pi) exp(-eta^2 r^2)) / r^2
__device__ __forceinline__ void ewald_b(const PairArgs &a, double r2, double &b0, double &b1)
{
  if (a.cheb_min < r2 && r2 < a.cheb_max) {
    double x = (r2 - a.cheb_min) * a.cheb_inv_dx;
    const unsigned i = (unsigned) x;
    const double2 *c = reinterpret_cast<const double2 *>(a.cheb + 8 * (size_t) i);
    const double2 c01 = __ldg(c), c23 = __ldg(c + 1), c45 = __ldg(c + 2), c67 = __ldg(c + 3);
    x -= i;
    b0 = ((c23.y * x + c23.x) * x + c01.y) * x + c01.x;
    b1 = (c67.x * x + c45.y) * x + c45.x;
  } else {
    const double r = sqrt(r2);
    const double er = a.eta * r;
    const double e = exp(-(er * er));
    b0 = erfc(er) / r;
    b1 = (b0 + a.eta * M_2_SQRTPI * e) / r2;
  }
}

template <int G, bool SCREEN, bool GEXCL>
__global__ void __launch_bounds__(128) k_pair_fp64(PairArgs a)
{
  const int lane = threadIdx.x & 31;
  const int p = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (p >= a.ngroup)
    return;
  double4 ri[G], pi_[G];
#pragma unroll
  for (int k = 0; k < G; k++) {
    ri[k] = a.sr[(size_t) p * G + k];
    pi_[k] = a.sp[(size_t) p * G + k];
  }
  int mi[G];
#pragma unroll
  for (int k = 0; k < G; k++)
    mi[k] = (int) pi_[k].w;
  const int gi = a.sorted[p];
  const int si0 = a.group[2 * gi];
  double aphi[G], aex[G], aey[G], aez[G], alx[G], aly[G], alz[G];
#pragma unroll
  for (int k = 0; k < G; k++)
    aphi[k] = aex[k] = aey[k] = aez[k] = alx[k] = aly[k] = alz[k] = 0;
  double elj = 0;
  const int cnt = a.nbr_count[p];
  const int *row = a.nbr + (size_t) p * a.rowcap;
  const double negL0 = -a.box.L[0], negL1 = -a.box.L[1], negL2 = -a.box.L[2];
  for (int e = lane; e < cnt; e += 32) {
    const int q = row[e];
    double4 rj[G], pj[G];
#pragma unroll
    for (int k = 0; k < G; k++) {
      rj[k] = a.sr[(size_t) q * G + k];
      pj[k] = a.sp[(size_t) q * G + k];
    }
    // anchor displacement and minimum-image shift, rounded as the reference does
    double x = __dsub_rn(ri[0].x, rj[0].x);
    double y = __dsub_rn(ri[0].y, rj[0].y);
    double z = __dsub_rn(ri[0].z, rj[0].z);
    const double sx = __dmul_rn(negL0, floor(__dadd_rn(__dmul_rn(x, a.box.invL[0]), 0.5)));
    const double sy = __dmul_rn(negL1, floor(__dadd_rn(__dmul_rn(y, a.box.invL[1]), 0.5)));
    const double sz = __dmul_rn(negL2, floor(__dadd_rn(__dmul_rn(z, a.box.invL[2]), 0.5)));
    x = __dadd_rn(x, sx);
    y = __dadd_rn(y, sy);
    z = __dadd_rn(z, sz);
    const double r2a = __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
    if (r2a > a.rhi2)
      continue;
    double s = 1, ds = 0;
    const bool smoothing = r2a > a.rlo2;
    if (smoothing) {
      const double inv = 1.0 / (a.rhi2 - a.rlo2);
      const double zz = (r2a - a.rlo2) * inv;
      s = ((-6 * zz + 15) * zz - 10) * zz * zz * zz + 1;
      ds = ((60 * zz - 120) * zz + 60) * zz * zz * inv;
    }
    bool gx = false;
    int gj = 0;
    if (GEXCL) {
      gj = a.sorted[q];
      gx = csr_has(a.gexcl_ptr, a.gexcl_idx, gi, gj);
    }
    double tmps = 0;
#pragma unroll
    for (int ia = 0; ia < G; ia++) {
#pragma unroll
      for (int jb = 0; jb < G; jb++) {
        const int m = mi[ia] & (int) pj[jb].w;
        if (!m)
          continue;
        if (GEXCL && gx) {
          const int sj = a.group[2 * gj] + jb;
          if (csr_has(a.excl_ptr, a.excl_idx, si0 + ia, sj))
            continue;
        }
        double dx, dy, dz, r2;
        if (ia == 0 && jb == 0) {
          dx = x;
          dy = y;
          dz = z;
          r2 = r2a;
        } else {
          dx = (ri[ia].x + sx) - rj[jb].x;
          dy = (ri[ia].y + sy) - rj[jb].y;
          dz = (ri[ia].z + sz) - rj[jb].z;
          r2 = dx * dx + dy * dy + dz * dz;
        }
        if (m & MMNB_SITE_HAS_Q) {
          double b0, b1;
          ewald_b(a, r2, b0, b1);
          if (SCREEN) {
            const double rs = pi_[ia].z + pj[jb].z;
            if (r2 < rs * rs) {
              const double invr = 1.0 / sqrt(r2);
              const double inv3 = 1.0 / (rs * rs * rs);
              b0 += (-0.5 * r2 * inv3 + 1.5 / rs) - invr;
              b1 += inv3 - invr * invr * invr;
            }
          }
          const double qj = rj[jb].w;
          if (smoothing) {
            tmps += ri[ia].w * qj * b0;
            b0 *= s;
            b1 *= s;
          }
          const double qb1 = qj * b1;
          aphi[ia] += qj * b0;
          aex[ia] += qb1 * dx;
          aey[ia] += qb1 * dy;
          aez[ia] += qb1 * dz;
        }
        if (m & MMNB_SITE_HAS_LJ) {
          const double sg = a.geometric ? pi_[ia].x * pj[jb].x
                                        : (0.5 * (pi_[ia].x + pj[jb].x)) * (0.5 * (pi_[ia].x + pj[jb].x));
          const double s6 = sg * sg * sg;
          const double b = 4 * sqrt(pi_[ia].y * pj[jb].y) * s6;
          const double aa = b * s6;
          const double invr2 = 1.0 / r2;
          const double invr6 = invr2 * invr2 * invr2;
          const double binvr6 = b * invr6;
          const double ainvr12 = aa * invr6 * invr6;
          double du = 12 * ainvr12 * invr2 - 6 * binvr6 * invr2;
          double u = ainvr12 - binvr6;
          if (smoothing) {
            tmps += u;
            u *= s;
            du *= s;
          }
          elj += 0.5 * u;
          alx[ia] += du * dx;
          aly[ia] += du * dy;
          alz[ia] += du * dz;
        }
      }
    }
    if (smoothing) {
      alx[0] += ds * x * tmps;
      aly[0] += ds * y * tmps;
      alz[0] += ds * z * tmps;
    }
  }
  // warp reduction; every lane ends with the totals
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int k = 0; k < G; k++) {
      aphi[k] += __shfl_xor_sync(0xffffffffu, aphi[k], off);
      aex[k] += __shfl_xor_sync(0xffffffffu, aex[k], off);
      aey[k] += __shfl_xor_sync(0xffffffffu, aey[k], off);
      aez[k] += __shfl_xor_sync(0xffffffffu, aez[k], off);
      alx[k] += __shfl_xor_sync(0xffffffffu, alx[k], off);
      aly[k] += __shfl_xor_sync(0xffffffffu, aly[k], off);
      alz[k] += __shfl_xor_sync(0xffffffffu, alz[k], off);
    }
    elj += __shfl_xor_sync(0xffffffffu, elj, off);
  }
  const int ns = a.group[2 * gi + 1] - si0;
#pragma unroll
  for (int k = 0; k < G; k++) {
    if (lane == k && k < ns) {
      const int s = si0 + k;
      a.phi[s] = aphi[k];
      a.evec[3 * s] = aex[k];
      a.evec[3 * s + 1] = aey[k];
      a.evec[3 * s + 2] = aez[k];
      a.ljf[3 * s] = alx[k];
      a.ljf[3 * s + 1] = aly[k];
      a.ljf[3 * s + 2] = alz[k];
    }
  }
  if (lane == 0)
    a.lj_part[p] = elj;
}

// sorted, padded FP64 site data for the pair kernel
__global__ void k_sort_sites(const double *__restrict__ r, const double *__restrict__ q,
                             const double *__restrict__ sig, const double *__restrict__ eps,
                             const double *__restrict__ rscreen, const int *__restrict__ mask,
                             const int *__restrict__ sorted, const int *__restrict__ group, int ngroup, int G,
                             double4 *__restrict__ sr, double4 *__restrict__ sp)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ngroup * G)
    return;
  const int p = s / G, k = s % G;
  const int g = sorted[p];
  const int site = group[2 * g] + k;
  if (site < group[2 * g + 1]) {
    sr[s] = make_double4(r[3 * site], r[3 * site + 1], r[3 * site + 2], q[site]);
    sp[s] = make_double4(sig[site], eps[site], rscreen[site], (double) mask[site]);
  } else {
    sr[s] = make_double4(0, 0, 0, 0);
    sp[s] = make_double4(0, 0, 0, 0);
  }
}

// Per-site exclusion correction and 1-4 terms: each thread owns one site and
// adds the partner terms that act on it (src/rspace.c:219-242, 492-557).
struct ExclArgs {
  int nsite;
  Box box;
  double eta, e14, l14;
  int scale_e14, scale_l14, geometric, do14;
  const double *r, *q, *sig, *eps, *rscreen;
  const int *mask, *excl_ptr, *excl_idx, *p14_ptr, *p14_idx;
  double *phi, *evec, *ljf;
  double *lj14_part;
};

__device__ __forceinline__ void min_image_ref(const Box &b, double &x, double &y, double &z)
{
  x = __dadd_rn(x, __dmul_rn(-b.L[0], floor(__dadd_rn(__dmul_rn(x, b.invL[0]), 0.5))));
  y = __dadd_rn(y, __dmul_rn(-b.L[1], floor(__dadd_rn(__dmul_rn(y, b.invL[1]), 0.5))));
  z = __dadd_rn(z, __dmul_rn(-b.L[2], floor(__dadd_rn(__dmul_rn(z, b.invL[2]), 0.5))));
}

__global__ void k_exclusions_fp64(ExclArgs a)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nsite)
    return;
  const int mi = a.mask[i];
  double phi = 0, ex = 0, ey = 0, ez = 0, lx = 0, ly = 0, lz = 0, elj = 0;
  const double xi = a.r[3 * i], yi = a.r[3 * i + 1], zi = a.r[3 * i + 2];
  if (mi & MMNB_SITE_HAS_Q) {
    for (int n = a.excl_ptr[i]; n < a.excl_ptr[i + 1]; n++) {
      const int j = a.excl_idx[n];
      if (!(a.mask[j] & MMNB_SITE_HAS_Q))
        continue;
      double x = xi - a.r[3 * j], y = yi - a.r[3 * j + 1], z = zi - a.r[3 * j + 2];
      min_image_ref(a.box, x, y, z);
      const double r2 = x * x + y * y + z * z;
      const double rm = sqrt(r2);
      const double er = a.eta * rm;
      const double e = exp(-(er * er));
      const double b0 = -erf(er) / rm;
      const double b1 = (b0 + a.eta * M_2_SQRTPI * e) / r2;
      const double qj = a.q[j];
      phi += qj * b0;
      ex += qj * b1 * x;
      ey += qj * b1 * y;
      ez += qj * b1 * z;
    }
  }
  if (a.do14) {
    for (int n = a.p14_ptr[i]; n < a.p14_ptr[i + 1]; n++) {
      const int j = a.p14_idx[n];
      const int m = mi & a.mask[j];
      double x = xi - a.r[3 * j], y = yi - a.r[3 * j + 1], z = zi - a.r[3 * j + 2];
      min_image_ref(a.box, x, y, z);
      const double r2 = x * x + y * y + z * z;
      if (m & MMNB_SITE_HAS_Q) {
        const double rs = a.rscreen[i] + a.rscreen[j];
        double b0, b1;
        if (r2 < rs * rs) {
          b1 = 1.0 / (rs * rs * rs);
          b0 = -0.5 * r2 * b1 + 1.5 / rs;
        } else {
          const double invr = 1.0 / sqrt(r2);
          b0 = invr;
          b1 = invr * invr * invr;
        }
        if (a.scale_e14) {
          b0 *= a.e14;
          b1 *= a.e14;
        }
        const double qj = a.q[j];
        phi += qj * b0;
        ex += qj * b1 * x;
        ey += qj * b1 * y;
        ez += qj * b1 * z;
      }
      if (m & MMNB_SITE_HAS_LJ) {
        const double sg = a.geometric ? a.sig[i] * a.sig[j]
                                      : (0.5 * (a.sig[i] + a.sig[j])) * (0.5 * (a.sig[i] + a.sig[j]));
        const double s6 = sg * sg * sg;
        const double b = 4 * sqrt(a.eps[i] * a.eps[j]) * s6;
        const double aa = b * s6;
        const double invr2 = 1.0 / r2;
        const double invr6 = invr2 * invr2 * invr2;
        double du = 12 * aa * invr6 * invr6 * invr2 - 6 * b * invr6 * invr2;
        double u = aa * invr6 * invr6 - b * invr6;
        if (a.scale_l14) {
          u *= a.l14;
          du *= a.l14;
        }
        elj += 0.5 * u;
        lx += du * x;
        ly += du * y;
        lz += du * z;
      }
    }
  }
  a.phi[i] += phi;
  a.evec[3 * i] += ex;
  a.evec[3 * i + 1] += ey;
  a.evec[3 * i + 2] += ez;
  if (a.do14) {
    a.ljf[3 * i] += lx;
    a.ljf[3 * i + 1] += ly;
    a.ljf[3 * i + 2] += lz;
    a.lj14_part[i] = elj;
  }
}

cudaError_t launch_sort_sites(mmnb_handle *h, const double *d_r)
{
  const int n = h->ngroup * h->G;
  k_sort_sites<<<div_up(n, 256), 256, 0, h->stream>>>(d_r, h->d_q, h->d_sig, h->d_eps, h->d_rscreen, h->d_mask,
                                                      h->d_sorted, h->d_group, h->ngroup, h->G, h->d_sr, h->d_sp);
  return cudaGetLastError();
}

template <int G>
static void launch_pair_g(mmnb_handle *h, const PairArgs &a)
{
  const int blocks = div_up(h->ngroup, 4);
  if (h->has_rscreen) {
    if (h->any_gexcl)
      k_pair_fp64<G, true, true><<<blocks, 128, 0, h->stream>>>(a);
    else
      k_pair_fp64<G, true, false><<<blocks, 128, 0, h->stream>>>(a);
  } else {
    if (h->any_gexcl)
      k_pair_fp64<G, false, true><<<blocks, 128, 0, h->stream>>>(a);
    else
      k_pair_fp64<G, false, false><<<blocks, 128, 0, h->stream>>>(a);
  }
}

cudaError_t launch_rspace_fp64(mmnb_handle *h)
{
  PairArgs a;
  a.ngroup = h->ngroup;
  a.rowcap = h->rowcap;
  a.geometric = h->cfg.geometric_combining_for_sigma;
  a.box = h->box;
  a.rlo2 = h->rlo2;
  a.rhi2 = h->rhi2;
  a.eta = h->eta;
  a.cheb_min = h->cheb_min;
  a.cheb_max = h->cheb_max;
  a.cheb_inv_dx = h->cheb_inv_dx;
  a.cheb = h->d_cheb;
  a.sr = h->d_sr;
  a.sp = h->d_sp;
  a.nbr = h->d_nbr;
  a.nbr_count = h->d_nbr_count;
  a.sorted = h->d_sorted;
  a.group = h->d_group;
  a.gexcl_ptr = h->d_gexcl_ptr;
  a.gexcl_idx = h->d_gexcl_idx;
  a.excl_ptr = h->d_excl_ptr;
  a.excl_idx = h->d_excl_idx;
  a.phi = h->d_phi;
  a.evec = h->d_evec;
  a.ljf = h->d_ljf;
  a.lj_part = h->d_lj_part;
  switch (h->G) {
  case 1: launch_pair_g<1>(h, a); break;
  case 2: launch_pair_g<2>(h, a); break;
  case 3: launch_pair_g<3>(h, a); break;
  case 4: launch_pair_g<4>(h, a); break;
  default: launch_pair_g<8>(h, a); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_exclusions(mmnb_handle *h, const double *d_r)
{
  ExclArgs a;
  a.nsite = h->nsite;
  a.box = h->box;
  a.eta = h->eta;
  a.e14 = h->cfg.elec_1_4_scale_factor - 1;
  a.l14 = h->cfg.lj_1_4_scale_factor - 1;
  a.scale_e14 = fabs(h->cfg.elec_1_4_scale_factor - 1) > 1e-10;
  a.scale_l14 = fabs(h->cfg.lj_1_4_scale_factor - 1) > 1e-10;
  a.geometric = h->cfg.geometric_combining_for_sigma;
  a.do14 = h->use_14 ? 1 : 0;
  a.r = d_r;
  a.q = h->d_q;
  a.sig = h->d_sig;
  a.eps = h->d_eps;
  a.rscreen = h->d_rscreen;
  a.mask = h->d_mask;
  a.excl_ptr = h->d_excl_ptr;
  a.excl_idx = h->d_excl_idx;
  a.p14_ptr = h->d_p14_ptr;
  a.p14_idx = h->d_p14_idx;
  a.phi = h->d_phi;
  a.evec = h->d_evec;
  a.ljf = h->d_ljf;
  a.lj14_part = h->d_lj_part + h->ngroup;
  k_exclusions_fp64<<<div_up(h->nsite, 256), 256, 0, h->stream>>>(a);
  return cudaGetLastError();
}

}  // namespace mmnb

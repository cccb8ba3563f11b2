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
// group row.  In a first pass over each 32 partners the lanes compute the
// anchor distance and push the partners inside the cutoff into a per-warp
// queue in shared memory (ballot compaction); whenever 32 are queued, all
// lanes evaluate one group pair each, so no lane idles on a pair beyond the
// cutoff.  Each lane accumulates only the row group's sites; a warp shuffle
// reduction gives each site its total, written once with plain stores — no
// atomics and a fixed summation order, so results are bitwise reproducible.

#include "mmnb_internal.cuh"

namespace mmnb {

constexpr int kPairWarps = 4;
constexpr int kQueue = 64;

struct PairArgs {
  int ngroup, rowcap, geometric;
  Box box;
  double rlo2, rhi2, inv_sw, eta;
  double cheb_min, cheb_max, cheb_inv_dx;
  const double *cheb;
  const double4 *sr;   // x, y, z, q          (sorted, padded slots)
  const double4 *sp;   // sig, sqrt(eps), rscreen, mask
  const int *nbr, *nbr_count, *sorted, *group;
  const int *gexcl_ptr, *gexcl_idx, *excl_ptr, *excl_idx;
  double *phi, *evec, *ljf, *lj_part;
  double *vir_part;  // per block: sum of the virial's pair term (mmnb_virial), or null
  const double *cheb_d;  // 512 x 4: cubics of -eta d/d(eta) of the table (mmnb_virial)
  const double2 *tw0, *tw1;  // the table's cubics: (c0, c1) and (c2, c3) per segment
};

// b0 = erfc(eta r)/r, b1 = (b0 + 2 eta/sqrt(pi) exp(-eta^2 r^2)) / r^2; seg and
// f: the table segment and the position in it (seg = -1 outside the table)
__device__ __forceinline__ void ewald_b(const PairArgs &a, double r2, double &b0, double &b1, int &seg, double &f)
{
  ewald_table_half(a.tw0, a.tw1, a.cheb_min, a.cheb_max, a.cheb_inv_dx, a.eta, r2, b0, b1, seg, f);
}

// The table is refitted for each eta, so along the volume-move path its eta
// derivative is the fitted cubic D of -eta d/d(eta) erfc(eta r)/r rather than
// b1 r^2 - b0, the identity the exact function obeys and mmnb_virial's scale
// covariance assumes: the difference, for the virial's pair term
__device__ __forceinline__ double table_eta_term(const PairArgs &a, int seg, double f, double r2, double b0,
                                                 double b1)
{
  const double2 *dc = reinterpret_cast<const double2 *>(a.cheb_d) + 2 * seg;
  const double2 d01 = __ldg(dc), d23 = __ldg(dc + 1);
  return ((d23.y * f + d23.x) * f + d01.y) * f + d01.x - (b1 * r2 - b0);
}

template <int G>
struct PairAcc {
  double phi[G], ex[G], ey[G], ez[G], lx[G], ly[G], lz[G];
  double elj;
  double vir;  // LJ and switch force scalars times r^2 (dU/ds terms the site forces do not carry)
};

// one group pair (row group i, partner slot q) inside the cutoff
template <int G, bool SCREEN, bool GEXCL>
__device__ __forceinline__ void pair_fp64(const PairArgs &a, const double4 (&ri)[G], const double4 (&pi)[G],
                                          const int (&mi)[G], int gi, int si0, int q, double4 sh, PairAcc<G> &acc)
{
  double4 rj[G], pj[G];
#pragma unroll
  for (int k = 0; k < G; k++) {
    rj[k] = a.sr[(size_t) q * G + k];
    pj[k] = a.sp[(size_t) q * G + k];
  }
  const double sx = sh.x, sy = sh.y, sz = sh.z, r2a = sh.w;
  const double x = __dadd_rn(__dsub_rn(ri[0].x, rj[0].x), sx);
  const double y = __dadd_rn(__dsub_rn(ri[0].y, rj[0].y), sy);
  const double z = __dadd_rn(__dsub_rn(ri[0].z, rj[0].z), sz);
  double s = 1, ds = 0;
  const bool smoothing = r2a > a.rlo2;
  if (smoothing) {
    const double zz = (r2a - a.rlo2) * a.inv_sw;
    s = ((-6 * zz + 15) * zz - 10) * zz * zz * zz + 1;
    ds = ((60 * zz - 120) * zz + 60) * zz * zz * a.inv_sw;
  }
  bool gx = false;
  int sj0 = 0;
  if (GEXCL) {
    const int gj = a.sorted[q];
    gx = csr_has(a.gexcl_ptr, a.gexcl_idx, gi, gj);
    sj0 = a.group[2 * gj];
  }
  double tmps = 0;
#pragma unroll
  for (int ia = 0; ia < G; ia++) {
#pragma unroll
    for (int jb = 0; jb < G; jb++) {
      const int m = mi[ia] & __double2int_rz(pj[jb].w);
      if (!m)
        continue;
      if (GEXCL && gx && csr_has(a.excl_ptr, a.excl_idx, si0 + ia, sj0 + jb))
        continue;
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
        double b0, b1, fseg;
        int seg;
        ewald_b(a, r2, b0, b1, seg, fseg);
        if (a.vir_part && seg >= 0)
          acc.vir -= 0.5 * ri[ia].w * rj[jb].w * s * table_eta_term(a, seg, fseg, r2, b0, b1);
        if (SCREEN) {
          const double rs = pi[ia].z + pj[jb].z;
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
        acc.phi[ia] += qj * b0;
        acc.ex[ia] += qb1 * dx;
        acc.ey[ia] += qb1 * dy;
        acc.ez[ia] += qb1 * dz;
      }
      if (m & MMNB_SITE_HAS_LJ) {
        const double sg = a.geometric ? pi[ia].x * pj[jb].x
                                      : (0.5 * (pi[ia].x + pj[jb].x)) * (0.5 * (pi[ia].x + pj[jb].x));
        const double s6 = sg * sg * sg;
        const double b = 4 * (pi[ia].y * pj[jb].y) * s6;
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
        acc.elj += 0.5 * u;
        acc.vir += 0.5 * du * r2;
        acc.lx[ia] += du * dx;
        acc.ly[ia] += du * dy;
        acc.lz[ia] += du * dz;
      }
    }
  }
  if (smoothing) {
    acc.lx[0] += ds * x * tmps;
    acc.ly[0] += ds * y * tmps;
    acc.lz[0] += ds * z * tmps;
    acc.vir += 0.5 * ds * tmps * r2a;
  }
}

template <int G, bool SCREEN, bool GEXCL>
// three resident blocks per SM (168 registers) beat two (200): 586 vs 638 us
// on the 98,304-site water box
__global__ void __launch_bounds__(kPairWarps * 32, 3) k_pair_fp64(PairArgs a)
{
  __shared__ double4 qsh[kPairWarps][kQueue];
  __shared__ int qix[kPairWarps][kQueue];
  __shared__ double wlj[kPairWarps], wvir[kPairWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int p = blockIdx.x * kPairWarps + w;
  PairAcc<G> acc;
#pragma unroll
  for (int k = 0; k < G; k++)
    acc.phi[k] = acc.ex[k] = acc.ey[k] = acc.ez[k] = acc.lx[k] = acc.ly[k] = acc.lz[k] = 0;
  acc.elj = 0;
  acc.vir = 0;
  if (p < a.ngroup) {
    double4 ri[G], pi[G];
    int mi[G];
#pragma unroll
    for (int k = 0; k < G; k++) {
      ri[k] = a.sr[(size_t) p * G + k];
      pi[k] = a.sp[(size_t) p * G + k];
      mi[k] = __double2int_rz(pi[k].w);
    }
    const int gi = a.sorted[p];
    const int si0 = a.group[2 * gi];
    const int cnt = a.nbr_count[p];
    const int *row = a.nbr + (size_t) p * a.rowcap;
    const unsigned below = (1u << lane) - 1;
    int qn = 0;
    for (int base = 0; base < cnt; base += 32) {
      const int e = base + lane;
      bool take = false;
      int q = 0;
      double4 sh = make_double4(0, 0, 0, 0);
      if (e < cnt) {
        q = row[e];
        double x, y, z;
        const double r2a = anchor_disp(a.box, ri[0], a.sr[(size_t) q * G], x, y, z, sh.x, sh.y, sh.z);
        sh.w = r2a;
        take = r2a <= a.rhi2;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, take);
      if (take) {
        const int idx = qn + __popc(bal & below);
        qsh[w][idx] = sh;
        qix[w][idx] = q;
      }
      qn += __popc(bal);
      __syncwarp();
      if (qn >= 32) {
        pair_fp64<G, SCREEN, GEXCL>(a, ri, pi, mi, gi, si0, qix[w][lane], qsh[w][lane], acc);
        __syncwarp();
        if (lane < qn - 32) {
          qsh[w][lane] = qsh[w][lane + 32];
          qix[w][lane] = qix[w][lane + 32];
        }
        __syncwarp();
        qn -= 32;
      }
    }
    if (lane < qn)
      pair_fp64<G, SCREEN, GEXCL>(a, ri, pi, mi, gi, si0, qix[w][lane], qsh[w][lane], acc);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
      for (int k = 0; k < G; k++) {
        acc.phi[k] += __shfl_xor_sync(0xffffffffu, acc.phi[k], off);
        acc.ex[k] += __shfl_xor_sync(0xffffffffu, acc.ex[k], off);
        acc.ey[k] += __shfl_xor_sync(0xffffffffu, acc.ey[k], off);
        acc.ez[k] += __shfl_xor_sync(0xffffffffu, acc.ez[k], off);
        acc.lx[k] += __shfl_xor_sync(0xffffffffu, acc.lx[k], off);
        acc.ly[k] += __shfl_xor_sync(0xffffffffu, acc.ly[k], off);
        acc.lz[k] += __shfl_xor_sync(0xffffffffu, acc.lz[k], off);
      }
      acc.elj += __shfl_xor_sync(0xffffffffu, acc.elj, off);
      acc.vir += __shfl_xor_sync(0xffffffffu, acc.vir, off);
    }
    const int ns = a.group[2 * gi + 1] - si0;
#pragma unroll
    for (int k = 0; k < G; k++) {
      if (lane == k && k < ns) {
        const int s = si0 + k;
        a.phi[s] = acc.phi[k];
        a.evec[3 * s] = acc.ex[k];
        a.evec[3 * s + 1] = acc.ey[k];
        a.evec[3 * s + 2] = acc.ez[k];
        a.ljf[3 * s] = acc.lx[k];
        a.ljf[3 * s + 1] = acc.ly[k];
        a.ljf[3 * s + 2] = acc.lz[k];
      }
    }
  }
  if (lane == 0) {
    wlj[w] = acc.elj;
    wvir[w] = acc.vir;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0, v = 0;
    for (int k = 0; k < kPairWarps; k++) {
      t += wlj[k];
      v += wvir[k];
    }
    a.lj_part[blockIdx.x] = t;
    if (a.vir_part)
      a.vir_part[blockIdx.x] = v;
  }
}

// sorted, padded FP64 site data for the pair kernel
__global__ void k_sort_sites(const double *__restrict__ r, const double *__restrict__ q,
                             const double *__restrict__ sig, const double *__restrict__ eps,
                             const double *__restrict__ rscreen, const int *__restrict__ mask,
                             const int *__restrict__ sorted, const int *__restrict__ group, int ngroup, int G,
                             double4 *__restrict__ sr, double4 *__restrict__ sp, int *__restrict__ flags)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ngroup * G)
    return;
  const int p = s / G, k = s % G;
  const int g = sorted[p];
  const int site = group[2 * g] + k;
  if (site < group[2 * g + 1]) {
    const double x = r[3 * site], y = r[3 * site + 1], z = r[3 * site + 2];
    if (!isfinite(x) || !isfinite(y) || !isfinite(z))
      flags[kFlagError] = MMNB_ERR_DEVICE;
    sr[s] = make_double4(x, y, z, q[site]);
    sp[s] = make_double4(sig[site], sqrt(eps[site]), rscreen[site], (double) mask[site]);
  } else {
    sr[s] = make_double4(0, 0, 0, 0);
    sp[s] = make_double4(0, 0, 0, 0);
  }
}

// Per-site exclusion correction and 1-4 terms: each thread owns one site and
// adds the partner terms that act on it (src/rspace.c:219-242, 492-557).
constexpr int kExclThreads = 256;

struct ExclArgs {
  int nsite;
  Box box;
  double eta, e14, l14;
  int scale_e14, scale_l14, geometric, do14;
  int assign;  // write the site arrays (first writer of the evaluation) instead of adding
  const double *r, *q, *sig, *eps, *rscreen;
  const int *mask, *excl_ptr, *excl_idx, *p14_ptr, *p14_idx;
  double *phi, *evec, *ljf;
  double *lj14_part;
  double *vir14_part;  // per block: the 1-4 LJ force scalars times r^2 / 2 (mmnb_virial), or null
};

__global__ void __launch_bounds__(kExclThreads) k_exclusions_fp64(ExclArgs a)
{
  __shared__ double sl[kExclThreads], sv[kExclThreads];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double elj = 0, vir = 0;
  if (i < a.nsite) {
    const int mi = a.mask[i];
    double phi = 0, ex = 0, ey = 0, ez = 0, lx = 0, ly = 0, lz = 0;
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
          vir += 0.5 * du * r2;
          lx += du * x;
          ly += du * y;
          lz += du * z;
        }
      }
    }
    if (a.assign) {
      // the same bits as adding to zeroed arrays (0 + x, which also turns -0 into +0)
      a.phi[i] = 0.0 + phi;
      a.evec[3 * i] = 0.0 + ex;
      a.evec[3 * i + 1] = 0.0 + ey;
      a.evec[3 * i + 2] = 0.0 + ez;
      a.ljf[3 * i] = 0.0 + lx;
      a.ljf[3 * i + 1] = 0.0 + ly;
      a.ljf[3 * i + 2] = 0.0 + lz;
    } else {
      a.phi[i] += phi;
      a.evec[3 * i] += ex;
      a.evec[3 * i + 1] += ey;
      a.evec[3 * i + 2] += ez;
      if (a.do14) {
        a.ljf[3 * i] += lx;
        a.ljf[3 * i + 1] += ly;
        a.ljf[3 * i + 2] += lz;
      }
    }
  }
  sl[threadIdx.x] = elj;
  sv[threadIdx.x] = vir;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sl[threadIdx.x] += sl[threadIdx.x + s];
      sv[threadIdx.x] += sv[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    a.lj14_part[blockIdx.x] = sl[0];
    if (a.vir14_part)
      a.vir14_part[blockIdx.x] = sv[0];
  }
}

cudaError_t launch_sort_sites(mmnb_handle *h, const double *d_r)
{
  const int n = h->ngroup * h->G;
  k_sort_sites<<<div_up(n, 256), 256, 0, h->stream>>>(d_r, h->d_q, h->d_sig, h->d_eps, h->d_rscreen, h->d_mask,
                                                      h->d_sorted, h->d_group, h->ngroup, h->G, h->d_sr, h->d_sp,
                                                      h->d_flags);
  h->launches += 1;
  return cudaGetLastError();
}

template <int G>
static void launch_pair_g(mmnb_handle *h, const PairArgs &a)
{
  const int blocks = div_up(h->ngroup, kPairWarps);
  const int threads = kPairWarps * 32;
  h->launches += 1;
  if (h->has_rscreen) {
    if (h->any_gexcl)
      k_pair_fp64<G, true, true><<<blocks, threads, 0, h->stream>>>(a);
    else
      k_pair_fp64<G, true, false><<<blocks, threads, 0, h->stream>>>(a);
  } else {
    if (h->any_gexcl)
      k_pair_fp64<G, false, true><<<blocks, threads, 0, h->stream>>>(a);
    else
      k_pair_fp64<G, false, false><<<blocks, threads, 0, h->stream>>>(a);
  }
}

int pair_blocks(const mmnb_handle *h) { return div_up(h->ngroup, kPairWarps); }
int excl_blocks(const mmnb_handle *h) { return div_up(h->nsite, kExclThreads); }

cudaError_t launch_rspace_fp64(mmnb_handle *h)
{
  PairArgs a;
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
  a.vir_part = h->want_virial ? h->d_vir_part : nullptr;
  a.cheb_d = h->d_cheb_d;
  a.tw0 = reinterpret_cast<const double2 *>(h->d_cheb_w);
  a.tw1 = a.tw0 + h->cheb_w_nseg;
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
  // the mixed form's pair kernels leave the FP64 site arrays alone: the
  // exclusion corrections are their first write of an evaluation
  a.assign = h->cfg.precision == MMNB_MIXED ? 1 : 0;
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
  a.lj14_part = h->d_lj_part + h->lj_pair_blocks;
  a.vir14_part = h->want_virial ? h->d_vir_part + h->lj_pair_blocks : nullptr;
  k_exclusions_fp64<<<excl_blocks(h), kExclThreads, 0, h->stream>>>(a);
  h->launches += 1;
  return cudaGetLastError();
}

}  // namespace mmnb

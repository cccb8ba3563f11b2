// Real-space Ewald + Lennard-Jones for rigid 3-site water, FP64 form.
//
// The group-pair semantics of RSpaceEwald (src/rspace.c:413-491), evaluated
// for groups [O(q, LJ), H(q), H(q)] (ElecLJ's groups for water,
// src/eleclj.cpp:654-676):
//   * the anchor (O) displacement, its minimum-image shift and the cutoff test
//     use the reference's rounding (anchor_disp), so the evaluated group pairs
//     are the reference's;
//   * every site pair uses the anchors' image shift; the quintic switch S and
//     dS/dr^2 come from the anchor distance, multiply the Coulomb and LJ terms,
//     and dS times the summed unswitched energy acts on the anchors (:479-489);
//   * b0 = erfc(eta r)/r comes from the reference's 512-segment Chebyshev cubic
//     in r^2 (src/rspace.c:25-37, src/cheby.c:7-45) and b1 = -2 db0/d(r^2) from
//     the derivative of that same cubic -- the reference stores the derivative
//     coefficients (-2 c1, -4 c2, -6 c3)/(b - a) beside the cubic; here they are
//     formed from the cubic's own coefficients and the segment width, which
//     agrees to rounding (the table's b1 is not the exact field term: it differs
//     from it by up to ~1e-5 relative at short range, so the table, not an exact
//     erfc, is what reproduces the reference);
//   * past the table's upper end (r^2 > 1.2 rc^2, which only site pairs of
//     water reach) the table continues with segments of the same construction
//     (the reference evaluates erfc and exp there; the two differ by ~1e-16
//     absolute at those distances), and below its lower end (r^2 < 4) erfc and
//     exp are evaluated directly, as in the reference.
//
// Layout: a persistent grid, one block of up to kW64Warps warps per SM slot; each
// warp takes the next row group from a counter and walks its list 32 entries
// at a time (anchor test per lane, ballot compaction into a 128-slot ring of
// anchor displacements, cp.async of the partner's 96-byte record into the same
// slot), evaluating 32 queued group pairs at a time.  The table's two halves,
// (c0, c1) and (c2, c3) per segment, sit in shared memory as two arrays of
// 16-byte entries, so a warp's random segment reads spread over all banks.
// Row totals are summed over the lanes in a fixed order (transpose through
// shared memory), so results do not depend on which warp or SM took the row.

#include "mmnb_internal.cuh"

namespace mmnb {

#ifndef MMNB_W64_BLOCKS
#define MMNB_W64_BLOCKS 1
#endif
// warps per block the kernel is compiled for (its register budget: 12 warps
// of 384 threads leave 170 registers a thread); a launch may use fewer when
// the rings and the table do not fit in shared memory
#ifndef MMNB_W64_WARPS
#define MMNB_W64_WARPS 12
#endif
constexpr int kW64Warps = MMNB_W64_WARPS;
// a batch of 32 is queued before the oldest 32 are evaluated, so the ring
// holds up to 63 + 32 entries
constexpr int kW64Ring = 128;
constexpr int kW64Acc = 17;  // phi (3), field (9), LJ + switch force on O (3), LJ energy, virial term

struct Water64Args {
  int ngroup, rowcap, geometric, nseg;
  Box box;
  double rlo2, rhi2, inv_sw, eta;
  double cmin, inv_dx, dscale, nsegd;  // dscale = -2 / segment width
  const double2 *table;                // [nseg] (c0, c1), then [nseg] (c2, c3)
  const double4 *anchor;               // sorted groups: anchor (x, y, z, -)
  const double4 *rec;                  // sorted groups: 3 x double4, layout in k_sort_water64
  const int *nbr, *nbr_count, *sorted, *group;
  unsigned long long *counter;         // next row; zeroed by k_sort_water64
  double *phi, *evec, *ljf, *lj_row;
  double *vir_row;                     // per row: the virial's pair term (mmnb_virial), or null
  const double *cheb_d;                // 512 x 4: cubics of -eta d/d(eta) of the table (mmnb_virial)
};

// b0 = erfc(eta r)/r and b1 = (b0 + 2 eta/sqrt(pi) exp(-eta^2 r^2)) / r^2;
// seg and f: the table segment and the position in it, seg = -1 outside the table
__device__ __forceinline__ void ewald_w64(const Water64Args &a, const double2 *t0, const double2 *t1, double r2,
                                          double &b0, double &b1, int &seg, double &f)
{
  const double x = (r2 - a.cmin) * a.inv_dx;
  if (x > 0 && x < a.nsegd) {
    // floor(x) exactly: x + 2^52 rounded down holds floor(x) in its low word
    const double t = __dadd_rd(x, 4503599627370496.0);
    const int i = __double2loint(t);
    f = x - (t - 4503599627370496.0);
    seg = i;
    const double2 c01 = t0[i], c23 = t1[i];
    b0 = ((c23.y * f + c23.x) * f + c01.y) * f + c01.x;
    b1 = a.dscale * ((3 * c23.y * f + 2 * c23.x) * f + c01.y);
  } else {
    seg = -1;
    f = 0;
    const double r = sqrt(r2);
    const double er = a.eta * r;
    b0 = erfc(er) / r;
    b1 = (b0 + a.eta * M_2_SQRTPI * exp(-(er * er))) / r2;
  }
}

// one site pair: d = displacement, qj = partner charge, qjs = qj S.
// VIR: the site pair's part of the virial that scale covariance misses --
// the table is refitted for each eta, so its eta derivative is the fitted
// cubic D of -eta d/d(eta) erfc(eta r)/r, not b1 r^2 - b0 (the identity the
// exact function obeys); qis = q_i S, added to the virial term with the
// factor -1/2 (the full list sees each pair twice)
template <bool VIR>
__device__ __forceinline__ void site_w64(const Water64Args &a, const double2 *t0, const double2 *t1, double dx,
                                         double dy, double dz, double r2, double qj, double qjs, double &ph,
                                         double &ex, double &ey, double &ez, double &tq, double qis, double &vir)
{
  double b0, b1, f;
  int seg;
  ewald_w64(a, t0, t1, r2, b0, b1, seg, f);
  tq += qj * b0;
  ph += qjs * b0;
  const double fb = qjs * b1;
  ex += fb * dx;
  ey += fb * dy;
  ez += fb * dz;
  if (VIR && seg >= 0 && seg < kCheb) {
    const double2 *dc = reinterpret_cast<const double2 *>(a.cheb_d) + 2 * seg;
    const double2 d01 = __ldg(dc), d23 = __ldg(dc + 1);
    const double dd = ((d23.y * f + d23.x) * f + d01.y) * f + d01.x;
    vir -= 0.5 * qis * qj * (dd - (b1 * r2 - b0));
  }
}

__device__ __forceinline__ void cp16(void *dst, const void *src)
{
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"((unsigned) __cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}

template <bool VIR>
__global__ void __launch_bounds__(kW64Warps * 32, MMNB_W64_BLOCKS) k_pair_water64(Water64Args a)
{
  extern __shared__ __align__(16) unsigned char smem[];
  // per warp: ring of (anchor displacement, r^2) and the partner's record
  double4 *ring = reinterpret_cast<double4 *>(smem);  // [warps][4][kW64Ring]
  double2 *tc01 = reinterpret_cast<double2 *>(smem + sizeof(double4) * 4 * kW64Ring * (blockDim.x >> 5));
  const double2 *tc23 = tc01 + a.nseg;
  for (int i = threadIdx.x; i < 2 * a.nseg; i += blockDim.x)
    tc01[i] = a.table[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double4 *qa = ring + (size_t) w * 4 * kW64Ring, *q0 = qa + kW64Ring, *q1 = q0 + kW64Ring, *q2 = q1 + kW64Ring;
  const unsigned below = (1u << lane) - 1;
  for (;;) {
    int p = 0;
    if (lane == 0)
      p = (int) atomicAdd(a.counter, 1ull);
    p = __shfl_sync(0xffffffffu, p, 0);
    if (p >= a.ngroup)
      break;
    const double4 ai = a.anchor[p];
    const double4 r0 = a.rec[3 * (size_t) p], r1 = a.rec[3 * (size_t) p + 1], r2 = a.rec[3 * (size_t) p + 2];
    // record: (h1x, h1y, h1z, h2x), (h2y, h2z, qO, qH1), (qH2, sigma, sqrt(eps), -)
    const double h1x = r0.x, h1y = r0.y, h1z = r0.z, h2x = r0.w, h2y = r1.x, h2z = r1.y;
    const double qO = r1.z, qH1 = r1.w, qH2 = r2.x, sgO = r2.y, seO = r2.z;
    double acc[kW64Acc];
#pragma unroll
    for (int c = 0; c < kW64Acc; c++)
      acc[c] = 0;
    auto compute = [&](int k) {
      const double4 da = qa[k], j0 = q0[k], j1 = q1[k], j2 = q2[k];
      const double j1x = j0.x, j1y = j0.y, j1z = j0.z, j2x = j0.w, j2y = j1.x, j2z = j1.y;
      const double qjO = j1.z, qj1 = j1.w, qj2 = j2.x, sgj = j2.y, sej = j2.z;
      const double r2a = da.w;
      // switch (zero width inside rc - width: s = 1 and ds = 0 exactly there)
      const double zz = fmax(r2a - a.rlo2, 0.0) * a.inv_sw;
      const double s = ((-6 * zz + 15) * zz - 10) * zz * zz * zz + 1;
      const double ds = ((60 * zz - 120) * zz + 60) * zz * zz * a.inv_sw;
      const double qjOs = qjO * s, qj1s = qj1 * s, qj2s = qj2 * s;
      const double qOs = qO * s, qH1s = qH1 * s, qH2s = qH2 * s;
      double tO = 0, t1 = 0, t2 = 0;
      // row O
      site_w64<VIR>(a, tc01, tc23, da.x, da.y, da.z, r2a, qjO, qjOs, acc[0], acc[3], acc[4], acc[5], tO, qOs, acc[16]);
      {
        const double dx = da.x - j1x, dy = da.y - j1y, dz = da.z - j1z;
        site_w64<VIR>(a, tc01, tc23, dx, dy, dz, dx * dx + dy * dy + dz * dz, qj1, qj1s, acc[0], acc[3], acc[4], acc[5], tO, qOs, acc[16]);
      }
      {
        const double dx = da.x - j2x, dy = da.y - j2y, dz = da.z - j2z;
        site_w64<VIR>(a, tc01, tc23, dx, dy, dz, dx * dx + dy * dy + dz * dz, qj2, qj2s, acc[0], acc[3], acc[4], acc[5], tO, qOs, acc[16]);
      }
      // row H1
      {
        const double cx = da.x + h1x, cy = da.y + h1y, cz = da.z + h1z;
        site_w64<VIR>(a, tc01, tc23, cx, cy, cz, cx * cx + cy * cy + cz * cz, qjO, qjOs, acc[1], acc[6], acc[7], acc[8], t1, qH1s, acc[16]);
        double dx = cx - j1x, dy = cy - j1y, dz = cz - j1z;
        site_w64<VIR>(a, tc01, tc23, dx, dy, dz, dx * dx + dy * dy + dz * dz, qj1, qj1s, acc[1], acc[6], acc[7], acc[8], t1, qH1s, acc[16]);
        dx = cx - j2x;
        dy = cy - j2y;
        dz = cz - j2z;
        site_w64<VIR>(a, tc01, tc23, dx, dy, dz, dx * dx + dy * dy + dz * dz, qj2, qj2s, acc[1], acc[6], acc[7], acc[8], t1, qH1s, acc[16]);
      }
      // row H2
      {
        const double cx = da.x + h2x, cy = da.y + h2y, cz = da.z + h2z;
        site_w64<VIR>(a, tc01, tc23, cx, cy, cz, cx * cx + cy * cy + cz * cz, qjO, qjOs, acc[2], acc[9], acc[10], acc[11], t2, qH2s, acc[16]);
        double dx = cx - j1x, dy = cy - j1y, dz = cz - j1z;
        site_w64<VIR>(a, tc01, tc23, dx, dy, dz, dx * dx + dy * dy + dz * dz, qj1, qj1s, acc[2], acc[9], acc[10], acc[11], t2, qH2s, acc[16]);
        dx = cx - j2x;
        dy = cy - j2y;
        dz = cz - j2z;
        site_w64<VIR>(a, tc01, tc23, dx, dy, dz, dx * dx + dy * dy + dz * dz, qj2, qj2s, acc[2], acc[9], acc[10], acc[11], t2, qH2s, acc[16]);
      }
      // O-O Lennard-Jones (src/rspace.c:258-297)
      const double sg = a.geometric ? sgO * sgj : (0.5 * (sgO + sgj)) * (0.5 * (sgO + sgj));
      const double s6 = sg * sg * sg;
      const double b = 4 * (seO * sej) * s6;
      const double aa = b * s6;
      const double invr2 = 1.0 / r2a;
      const double invr6 = invr2 * invr2 * invr2;
      const double binvr6 = b * invr6;
      const double ainvr12 = aa * invr6 * invr6;
      const double du = 12 * ainvr12 * invr2 - 6 * binvr6 * invr2;
      const double u = ainvr12 - binvr6;
      const double tmps = qO * tO + qH1 * t1 + qH2 * t2 + u;
      acc[15] += 0.5 * (u * s);
      const double g = du * s + ds * tmps;
      acc[12] += g * da.x;
      acc[13] += g * da.y;
      acc[14] += g * da.z;
      // the part of dU/ds (box scaling) the site forces do not carry: the LJ and
      // switch force scalar times R^2 (each pair is seen from both rows: half)
      acc[16] += 0.5 * g * r2a;
    };
    const int cnt = a.nbr_count[p];
    const int *row = a.nbr + (size_t) p * a.rowcap;
    // entries past the row end read the row's own group (a valid address)
    int jc = lane < cnt ? row[lane] : p;
    int jn = lane + 32 < cnt ? row[lane + 32] : p;
    double4 ac = a.anchor[jc];
    int head = 0, qn = 0;
    for (int base = 0; base < cnt; base += 32) {
      const int e2 = base + 64 + lane;
      const int jnn = e2 < cnt ? row[e2] : p;
      const double4 an = a.anchor[jn];
      double x, y, z, sx, sy, sz;
      const double r2a = anchor_disp(a.box, ai, ac, x, y, z, sx, sy, sz);
      const bool take = base + lane < cnt && r2a <= a.rhi2;
      const unsigned bal = __ballot_sync(0xffffffffu, take);
      if (take) {
        const int slot = (head + qn + __popc(bal & below)) & (kW64Ring - 1);
        qa[slot] = make_double4(x, y, z, r2a);
        const double4 *src = a.rec + 3 * (size_t) jc;
        cp16(&q0[slot], src);
        cp16(reinterpret_cast<double2 *>(&q0[slot]) + 1, reinterpret_cast<const double2 *>(src) + 1);
        cp16(&q1[slot], src + 1);
        cp16(reinterpret_cast<double2 *>(&q1[slot]) + 1, reinterpret_cast<const double2 *>(src + 1) + 1);
        cp16(&q2[slot], src + 2);
        cp16(reinterpret_cast<double2 *>(&q2[slot]) + 1, reinterpret_cast<const double2 *>(src + 2) + 1);
      }
      asm volatile("cp.async.commit_group;\n" ::: "memory");
      const bool run = qn >= 32;
      qn += __popc(bal);
      if (run) {
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        __syncwarp();
        compute((head + lane) & (kW64Ring - 1));
        __syncwarp();
        head = (head + 32) & (kW64Ring - 1);
        qn -= 32;
      }
      jc = jn;
      jn = jnn;
      ac = an;
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncwarp();
    for (; qn > 0; qn -= 32, head = (head + 32) & (kW64Ring - 1))
      if (lane < qn)
        compute((head + lane) & (kW64Ring - 1));
    // row totals: lanes' values transposed through the warp's ring, each of
    // lanes 0..15 adds one column over the 32 lanes in lane order
    __syncwarp();
    double(*red)[kW64Acc + 1] = reinterpret_cast<double(*)[kW64Acc + 1]>(qa);
    static_assert(32 * (kW64Acc + 1) * sizeof(double) <= 4 * kW64Ring * sizeof(double4), "ring too small");
#pragma unroll
    for (int c = 0; c < kW64Acc; c++)
      red[lane][c] = acc[c];
    __syncwarp();
    const int si0 = a.group[2 * a.sorted[p]];
    if (lane < kW64Acc) {
      double t = 0;
      for (int l = 0; l < 32; l++)
        t += red[l][lane];
      if (lane < 3)
        a.phi[si0 + lane] = t;
      else if (lane < 12)
        a.evec[3 * si0 + (lane - 3)] = t;
      else if (lane < 15)
        a.ljf[3 * si0 + (lane - 12)] = t;
      else if (lane == 15)
        a.lj_row[p] = t;
      else if (a.vir_row)
        a.vir_row[p] = t;
    } else if (lane < kW64Acc + 6) {
      // the H sites carry no LJ force
      a.ljf[3 * si0 + 3 + (lane - kW64Acc)] = 0;
    }
    __syncwarp();  // the ring is the next row's again only after every lane has read it
  }
}

// Per step: sorted FP64 anchors and the 96-byte records of the partner side,
// (h1x, h1y, h1z, h2x), (h2y, h2z, qO, qH1), (qH2, sigma_O, sqrt(eps_O), 0) with
// the H positions taken from the anchor O; the row counter is cleared and a
// non-finite coordinate is flagged.
__global__ void k_sort_water64(const double *__restrict__ r, const double *__restrict__ q,
                               const double *__restrict__ sig, const double *__restrict__ eps,
                               const int *__restrict__ sorted, const int *__restrict__ group, int ngroup,
                               double4 *__restrict__ anchor, double4 *__restrict__ rec,
                               unsigned long long *__restrict__ counter, int *__restrict__ flags)
{
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0)
    *counter = 0ull;
  if (p >= ngroup)
    return;
  const int a0 = group[2 * sorted[p]];
  const double ax = r[3 * a0], ay = r[3 * a0 + 1], az = r[3 * a0 + 2];
  const double *h1 = r + 3 * (a0 + 1), *h2 = r + 3 * (a0 + 2);
  if (!isfinite(ax + ay + az + h1[0] + h1[1] + h1[2] + h2[0] + h2[1] + h2[2]))
    flags[kFlagError] = MMNB_ERR_DEVICE;
  anchor[p] = make_double4(ax, ay, az, 0.0);
  rec[3 * (size_t) p] = make_double4(h1[0] - ax, h1[1] - ay, h1[2] - az, h2[0] - ax);
  rec[3 * (size_t) p + 1] = make_double4(h2[1] - ay, h2[2] - az, q[a0], q[a0 + 1]);
  rec[3 * (size_t) p + 2] = make_double4(q[a0 + 2], sig[a0], sqrt(eps[a0]), 0.0);
}

static size_t water64_smem(const mmnb_handle *h, int warps)
{
  return sizeof(double4) * 4 * kW64Ring * warps + sizeof(double2) * 2 * (size_t) h->cheb_w_nseg;
}

cudaError_t launch_sort_water64(mmnb_handle *h, const double *d_r)
{
  k_sort_water64<<<div_up(h->ngroup, 256), 256, 0, h->stream>>>(
      d_r, h->d_q, h->d_sig, h->d_eps, h->d_sorted, h->d_group, h->ngroup, h->d_sp, h->d_sr, h->d_wsum + 3,
      h->d_flags);
  h->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_rspace_water64(mmnb_handle *h)
{
  cudaError_t e;
  int optin = 0;
  if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->dev)) != cudaSuccess)
    return e;
  // the tuned warps per block, fewer if the rings and this box's table do not
  // fit (the table grows with rc: 12 warps below ~22 KB of table)
  int warps = std::min(h->tune.water64_warps, kW64Warps);
  while (warps > 4 && water64_smem(h, warps) > (size_t) optin)
    warps -= 2;
  if (h->water64_grid == 0 || warps != h->water64_warps) {
    int nsm = 0;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->dev)) != cudaSuccess)
      return e;
    const size_t smem = water64_smem(h, warps);
    if ((e = cudaFuncSetAttribute(k_pair_water64<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)) !=
            cudaSuccess ||
        (e = cudaFuncSetAttribute(k_pair_water64<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)) !=
            cudaSuccess)
      return e;
    int per_sm = 0, per_sm_v = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pair_water64<false>, warps * 32, smem)) !=
            cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_v, k_pair_water64<true>, warps * 32, smem)) !=
            cudaSuccess)
      return e;
    per_sm = std::min(per_sm, per_sm_v);
    if (per_sm < 1)
      return cudaErrorLaunchOutOfResources;
    h->water64_grid = std::min(per_sm * nsm, div_up(h->ngroup, warps));
    h->water64_smem = smem;
    h->water64_warps = warps;
  }
  Water64Args a;
  a.ngroup = h->ngroup;
  a.rowcap = h->rowcap;
  a.geometric = h->cfg.geometric_combining_for_sigma;
  a.nseg = h->cheb_w_nseg;
  a.box = h->box;
  a.rlo2 = h->rlo2;
  a.rhi2 = h->rhi2;
  a.inv_sw = h->inv_sw;
  a.eta = h->eta;
  a.cmin = h->cheb_min;
  a.inv_dx = h->cheb_inv_dx;
  a.dscale = -2 * h->cheb_inv_dx;
  a.nsegd = (double) h->cheb_w_nseg;
  a.table = reinterpret_cast<const double2 *>(h->d_cheb_w);
  a.anchor = h->d_sp;
  a.rec = h->d_sr;
  a.nbr = h->d_nbr;
  a.nbr_count = h->d_nbr_count;
  a.sorted = h->d_sorted;
  a.group = h->d_group;
  a.counter = h->d_wsum + 3;
  a.phi = h->d_phi;
  a.evec = h->d_evec;
  a.ljf = h->d_ljf;
  a.lj_row = h->d_lj_row;
  a.vir_row = h->want_virial ? h->d_vir_row : nullptr;
  a.cheb_d = h->d_cheb_d;
  if (h->want_virial)
    k_pair_water64<true><<<h->water64_grid, h->water64_warps * 32, h->water64_smem, h->stream>>>(a);
  else
    k_pair_water64<false><<<h->water64_grid, h->water64_warps * 32, h->water64_smem, h->stream>>>(a);
  h->launches += 1;
  return cudaGetLastError();
}

}  // namespace mmnb

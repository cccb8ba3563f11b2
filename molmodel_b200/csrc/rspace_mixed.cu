// Real-space Ewald + Lennard-Jones, mixed-precision form.
//
// Same group-pair semantics as the FP64 form (RSpaceEwald, src/rspace.c:413-491):
// the cutoff test and minimum image use the FP64 anchor positions with the
// reference's rounding, so the set of evaluated group pairs is the FP64 set.
// Everything after that is FP32:
//   * site positions enter as FP32 offsets from their group's anchor, so a
//     site-pair displacement is (anchor displacement, FP64 -> FP32) plus the
//     difference of two small offsets: relative precision ~1e-7 at any box
//     size, although the unwrapped coordinates themselves can be large;
//   * erfc(eta r) = t P(t) exp(-eta^2 r^2) with t = 1/(1 + p eta r): the
//     form of Hastings' approximation with a degree-7 P refitted for
//     relative accuracy (below), exp(-eta^2 r^2) shared with the field term
//     b1 = (b0 + 2 eta/sqrt(pi) exp(-eta^2 r^2)) / r^2;
//   * the switch and LJ terms are the FP64 form's formulas in FP32.
// Each group pair's contribution to each row site (potential, field, LJ
// force) is summed in FP32 and then converted to 64-bit fixed point
// (2^32 units per unit) before it is added: integer addition is associative,
// so the totals do not depend on the list order, on which lane took which
// pair, or on the reduction order — the forces are bitwise deterministic.
//
// Work layout as in the FP64 form: full list, one warp per row group, a
// ballot-compacted shared-memory queue of in-cutoff partners so every lane
// evaluates a group pair, and a shared-memory transpose to reduce the lanes'
// fixed-point totals.

#include "mmnb_internal.cuh"

namespace mmnb {

constexpr int kMxWarps = 4;
constexpr int kMxQueue = 64;
constexpr int kNacc = 7;  // phi, E (3), LJ force (3)

// erfc(x) ~= t P(t) exp(-x^2), t = 1/(1 + p x): Hastings' form (Abramowitz &
// Stegun 7.1.26) with P refitted for relative accuracy (<= 4e-7 for all x >= 0,
// FP32 Horner included); molmodel_b200/csrc/fit_erfc.py derives the table.
constexpr float kErfcP = 0.3275911f;
constexpr float kE0 = 0.185182706f, kE1 = 0.179008603f, kE2 = 0.215395942f, kE3 = -0.00290450454f,
                kE4 = 0.502499402f, kE5 = -0.455885917f, kE6 = 0.524125457f, kE7 = -0.147421896f;

__device__ __forceinline__ float ex2_approx(float x)
{
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// r^2 of two distinct sites is a normal number, so the flush-to-zero form
// (no denormal fix-up around the MUFU op) gives rsqrtf's result
__device__ __forceinline__ float rsqrt_approx(float x)
{
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ float rcp_approx(float x)
{
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// b0 = erfc(eta r)/r and b1 = (b0 + c2 exp(-eta^2 r^2))/r^2 from r^2 and 1/r;
// nel2 = -eta^2 log2(e)
__device__ __forceinline__ void ewald_f32(float r2, float rinv, float eta, float nel2, float c2, float &b0,
                                          float &b1)
{
  const float x = eta * (r2 * rinv);
  const float t = rcp_approx(fmaf(kErfcP, x, 1.f));
  float p = fmaf(kE7, t, kE6);
  p = fmaf(p, t, kE5);
  p = fmaf(p, t, kE4);
  p = fmaf(p, t, kE3);
  p = fmaf(p, t, kE2);
  p = fmaf(p, t, kE1);
  p = fmaf(p, t, kE0);
  const float e = ex2_approx(r2 * nel2);
  b0 = t * p * e * rinv;
  b1 = fmaf(c2, e, b0) * (rinv * rinv);
}

struct MixedArgs {
  int ngroup, rowcap, geometric;
  Box box;
  double rhi2;
  float rlo2, inv_sw, eta, c2, nel2;  // c2 = 2 eta / sqrt(pi), nel2 = -eta^2 log2(e)
  const float4 *site;           // offset from anchor, charge
  const float4 *par;            // sigma, sqrt(eps), rscreen, mask bits
  const double4 *anchor;
  const int *nbr, *nbr_count, *sorted, *group;
  const int *gexcl_ptr, *gexcl_idx, *excl_ptr, *excl_idx;
  long long *acc;               // per site, kAccStride
  double *lj_part;
  double *vir_part;             // per block: the virial's pair term (mmnb_virial), or null
};

__device__ __forceinline__ long long to_fx(float v) { return __float2ll_rn(v * 4294967296.0f); }

// one group pair inside the cutoff: FP32 sums, then fixed point
template <int G, bool SCREEN, bool GEXCL, bool ANCHOR_LJ>
__device__ __forceinline__ void pair_mixed(const MixedArgs &a, const float4 (&oi)[G], const float4 (&pi)[G], int gi,
                                           int si0, int q, float4 da, long long (&fx)[G][kNacc], long long &fe,
                                           long long &fv)
{
  float4 oj[G], pj[G];
#pragma unroll
  for (int k = 0; k < G; k++) {
    oj[k] = a.site[(size_t) q * G + k];
    pj[k] = a.par[(size_t) q * G + k];
  }
  const float r2a = da.w;
  float s = 1.f, ds = 0.f;
  const bool smoothing = r2a > a.rlo2;
  if (smoothing) {
    const float z = (r2a - a.rlo2) * a.inv_sw;
    s = fmaf(fmaf(fmaf(-6.f, z, 15.f), z, -10.f), z * z * z, 1.f);
    ds = fmaf(fmaf(60.f, z, -120.f), z, 60.f) * z * z * a.inv_sw;
  }
  bool gx = false;
  int sj0 = 0;
  if (GEXCL) {
    const int gj = a.sorted[q];
    gx = csr_has(a.gexcl_ptr, a.gexcl_idx, gi, gj);
    sj0 = a.group[2 * gj];
  }
  float ph[G], ex[G], ey[G], ez[G], lx[G], ly[G], lz[G];
#pragma unroll
  for (int k = 0; k < G; k++)
    ph[k] = ex[k] = ey[k] = ez[k] = lx[k] = ly[k] = lz[k] = 0.f;
  float tmps = 0.f, u_sum = 0.f, xv = 0.f;
#pragma unroll
  for (int ia = 0; ia < G; ia++) {
    const int mi = __float_as_int(pi[ia].w);
    const float cx = da.x + oi[ia].x, cy = da.y + oi[ia].y, cz = da.z + oi[ia].z;
    float tq = 0.f;  // sum_j q_j b0 before switching, for the switch derivative
#pragma unroll
    for (int jb = 0; jb < G; jb++) {
      const int m = mi & __float_as_int(pj[jb].w);
      if (!m)
        continue;
      if (GEXCL && gx && csr_has(a.excl_ptr, a.excl_idx, si0 + ia, sj0 + jb))
        continue;
      const float dx = cx - oj[jb].x, dy = cy - oj[jb].y, dz = cz - oj[jb].z;
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      const float rinv = rsqrt_approx(r2);
      if (m & MMNB_SITE_HAS_Q) {
        float b0, b1;
        ewald_f32(r2, rinv, a.eta, a.nel2, a.c2, b0, b1);
        if (SCREEN) {
          const float rs = pi[ia].z + pj[jb].z;
          if (r2 < rs * rs) {
            const float inv3 = 1.f / (rs * rs * rs);
            b0 += fmaf(-0.5f * r2, inv3, 1.5f / rs) - rinv;
            b1 += inv3 - rinv * rinv * rinv;
          }
        }
        const float qj = oj[jb].w;
        tq = fmaf(qj, b0, tq);
        const float qs = qj * s;
        ph[ia] = fmaf(qs, b0, ph[ia]);
        const float f = qs * b1;
        ex[ia] = fmaf(f, dx, ex[ia]);
        ey[ia] = fmaf(f, dy, ey[ia]);
        ez[ia] = fmaf(f, dz, ez[ia]);
      }
      if (m & MMNB_SITE_HAS_LJ) {
        const float sg = a.geometric ? pi[ia].x * pj[jb].x : 0.5f * (pi[ia].x + pj[jb].x) * 0.5f * (pi[ia].x + pj[jb].x);
        const float s6 = sg * sg * sg;
        const float b = 4.f * pi[ia].y * pj[jb].y * s6;
        const float aa = b * s6;
        const float ir2 = rinv * rinv;
        const float ir6 = ir2 * ir2 * ir2;
        const float bi6 = b * ir6;
        const float ai12 = aa * ir6 * ir6;
        const float du = (12.f * ai12 - 6.f * bi6) * ir2 * s;
        const float u = ai12 - bi6;
        tmps += u;
        u_sum = fmaf(u, s, u_sum);
        xv = fmaf(du, r2, xv);
        lx[ia] = fmaf(du, dx, lx[ia]);
        ly[ia] = fmaf(du, dy, ly[ia]);
        lz[ia] = fmaf(du, dz, lz[ia]);
      }
    }
    tmps = fmaf(oi[ia].w, tq, tmps);
  }
  if (smoothing) {
    const float g = ds * tmps;
    lx[0] = fmaf(g, da.x, lx[0]);
    ly[0] = fmaf(g, da.y, ly[0]);
    lz[0] = fmaf(g, da.z, lz[0]);
    xv = fmaf(g, r2a, xv);
  }
#pragma unroll
  for (int k = 0; k < G; k++) {
    fx[k][0] += to_fx(ph[k]);
    fx[k][1] += to_fx(ex[k]);
    fx[k][2] += to_fx(ey[k]);
    fx[k][3] += to_fx(ez[k]);
    if (!ANCHOR_LJ || k == 0) {
      fx[k][4] += to_fx(lx[k]);
      fx[k][5] += to_fx(ly[k]);
      fx[k][6] += to_fx(lz[k]);
    }
  }
  fe += to_fx(0.5f * u_sum);
  if (a.vir_part)
    fv += to_fx(0.5f * xv);
}

template <int G, bool SCREEN, bool GEXCL, bool ANCHOR_LJ>
__global__ void __launch_bounds__(kMxWarps * 32) k_pair_mixed(MixedArgs a)
{
  __shared__ float4 qda[kMxWarps][kMxQueue];
  __shared__ int qix[kMxWarps][kMxQueue];
  constexpr int kCols = G * kNacc + 2;  // site values, LJ energy, virial term
  constexpr bool kTranspose = G <= 4;
  __shared__ long long red[kTranspose ? kMxWarps : 1][kTranspose ? 32 : 1][kTranspose ? kCols : 1];
  __shared__ long long wlj[kMxWarps], wvir[kMxWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int p = blockIdx.x * kMxWarps + w;
  long long fx[G][kNacc];
#pragma unroll
  for (int k = 0; k < G; k++)
#pragma unroll
    for (int c = 0; c < kNacc; c++)
      fx[k][c] = 0;
  long long fe = 0, fv = 0;
  int gi = 0, si0 = 0, ns = 0;
  if (p < a.ngroup) {
    float4 oi[G], pi[G];
#pragma unroll
    for (int k = 0; k < G; k++) {
      oi[k] = a.site[(size_t) p * G + k];
      pi[k] = a.par[(size_t) p * G + k];
    }
    const double4 ai = a.anchor[p];
    gi = a.sorted[p];
    si0 = a.group[2 * gi];
    ns = a.group[2 * gi + 1] - si0;
    const int cnt = a.nbr_count[p];
    const int *row = a.nbr + (size_t) p * a.rowcap;
    const unsigned below = (1u << lane) - 1;
    int qn = 0;
    for (int base = 0; base < cnt; base += 32) {
      const int e = base + lane;
      bool take = false;
      int q = 0;
      float4 da = make_float4(0.f, 0.f, 0.f, 0.f);
      if (e < cnt) {
        q = row[e];
        double x, y, z, sx, sy, sz;
        const double r2a = anchor_disp(a.box, ai, a.anchor[q], x, y, z, sx, sy, sz);
        take = r2a <= a.rhi2;
        da = make_float4((float) x, (float) y, (float) z, (float) r2a);
      }
      const unsigned bal = __ballot_sync(0xffffffffu, take);
      if (take) {
        const int idx = qn + __popc(bal & below);
        qda[w][idx] = da;
        qix[w][idx] = q;
      }
      qn += __popc(bal);
      __syncwarp();
      if (qn >= 32) {
        pair_mixed<G, SCREEN, GEXCL, ANCHOR_LJ>(a, oi, pi, gi, si0, qix[w][lane], qda[w][lane], fx, fe, fv);
        __syncwarp();
        if (lane < qn - 32) {
          qda[w][lane] = qda[w][lane + 32];
          qix[w][lane] = qix[w][lane + 32];
        }
        __syncwarp();
        qn -= 32;
      }
    }
    if (lane < qn)
      pair_mixed<G, SCREEN, GEXCL, ANCHOR_LJ>(a, oi, pi, gi, si0, qix[w][lane], qda[w][lane], fx, fe, fv);
  }
  if constexpr (kTranspose) {
    // transpose reduction: lane c sums column c over the 32 lanes
#pragma unroll
    for (int k = 0; k < G; k++)
#pragma unroll
      for (int c = 0; c < kNacc; c++)
        red[w][lane][k * kNacc + c] = fx[k][c];
    red[w][lane][G * kNacc] = fe;
    red[w][lane][G * kNacc + 1] = fv;
    __syncwarp();
    for (int c = lane; c < kCols; c += 32) {
      long long t = 0;
      for (int l = 0; l < 32; l++)
        t += red[w][l][c];
      if (c == G * kNacc) {
        wlj[w] = t;
      } else if (c == G * kNacc + 1) {
        wvir[w] = t;
      } else if (p < a.ngroup) {
        const int k = c / kNacc, comp = c % kNacc;
        if (k < ns)
          a.acc[(size_t) (si0 + k) * kAccStride + comp] = t;
      }
    }
  } else {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
      for (int k = 0; k < G; k++)
#pragma unroll
        for (int c = 0; c < kNacc; c++)
          fx[k][c] += __shfl_xor_sync(0xffffffffu, fx[k][c], off);
      fe += __shfl_xor_sync(0xffffffffu, fe, off);
      fv += __shfl_xor_sync(0xffffffffu, fv, off);
    }
    if (lane == 0) {
      wlj[w] = fe;
      wvir[w] = fv;
    }
    if (p < a.ngroup)
#pragma unroll
      for (int k = 0; k < G; k++)
        if (lane == k && k < ns)
#pragma unroll
          for (int c = 0; c < kNacc; c++)
            a.acc[(size_t) (si0 + k) * kAccStride + c] = fx[k][c];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0, v = 0;
    for (int k = 0; k < kMxWarps; k++) {
      t += wlj[k];
      v += wvir[k];
    }
    a.lj_part[blockIdx.x] = (double) t * kFxInv;
    if (a.vir_part)
      a.vir_part[blockIdx.x] = (double) v * kFxInv;
  }
}

// ---- rigid-water fast path ------------------------------------------------------
//
// Every group is [O, H, H] with O carrying charge and LJ and the H sites
// charge only (the site layout of ElecLJ's groups for 3-site water,
// src/eleclj.cpp:654-676).  The nine site pairs and the one LJ pair of a
// group pair are straight-line code.  A warp owns one row group and walks its
// list 64 entries at a time: each lane tests two partners' anchor distances
// (FP32, from cell-relative anchors; the next 64 anchors are requested one
// step ahead, list indices two steps ahead), and for an accepted partner
// writes the anchor displacement to a 128-slot shared-memory ring and starts
// asynchronous copies (cp.async) of the partner's record (48 bytes, or the
// 24 bytes of H offsets when every water has the same parameters) into the
// same ring slot.  When 32 entries are queued every lane evaluates one group
// pair from shared memory.  Per group
// pair the kernel forms the FORCE on each row site (q E, plus LJ and switch
// terms on O) and the pair energies, and converts those 11 values to fixed
// point.
//
// The site-pair arithmetic runs two site pairs per instruction (sm_100's
// packed FP32 add/mul/fma on register pairs): the nine site pairs of a group
// pair are four packed pairs and one single one,
//   O  x (H1, H2)          partner H sites against the row O,
//   (H1, H2) x O           the row H sites against the partner O,
//   (H1, H2) x (H1, H2)    each row H against the partner H of its own index,
//   (H2, H1) x (H1, H2)    each row H against the other partner H,
//   O  x O,
// so the partner record is laid out in pairs: (h1x, h2x, h1y, h2y),
// (h1z, h2z, q1, q2), (qO, qO, sigma, sqrt(epsilon)), with the H offsets
// taken from the anchor O.  The multiply, add and fma of a packed pair round
// each half exactly as the single instructions do.

constexpr int kWaterRing = 128;
// Warps (rows) per block of the rigid-water kernel: one, so a block retires as
// soon as its row is done and its slot takes the next row (rows differ in
// length; with four warps per block the finished warps idle until the block's
// longest row ends)
constexpr int kWaterWarps = 1;

struct WaterArgs {
  int ngroup, rowcap, geometric;
  Box box;
  double rhi2;
  float rlo2, inv_sw, pe, c2, nel2;  // pe = p eta (erfc argument scale)
  const float4 *site;     // 3 packed slots per sorted group (above)
  const double4 *anchor;  // FP64 anchors (sorted groups): the prune bookkeeping
  const float4 *anc32;    // cell-relative FP32 anchors (sorted groups, k_prep_mixed)
  int ncell, nhalf;       // list cells per dimension, ncell / 2
  float edge[3];          // cell edge, FP32 (the value the offsets were formed with)
  float Lf[3], halfL[3];  // box edges and half edges, FP32
  float rhi2f, rp2f;      // rc^2 and (rc + prune margin)^2, FP32
  float uqO, uqH, usig, useps;  // uniform water: O and H charges, O sigma and sqrt(epsilon)
  const int *nbr, *nbr_count, *sorted, *group;
  long long *acc;         // per site: slots 4..6 receive the force, 0..3 are cleared
  unsigned long long *wsum;  // fixed-point Coulomb and LJ pair energies and, with the virial,
                             // the virial's pair term (wsum[4]); zeroed by the prep kernel
  // pruned rows (null: none): read when flags[kFlagPruneFull] is 0; made from
  // the full rows (pairs with r^2 <= rp2) when it is 1
  int *pnbr, *pcount;
  double *plast;          // sorted anchors at the last prune
  int *flags;
  double rp2;
};

// a pair of FP32 values in one 64-bit register pair (the operand of the packed
// f32x2 instructions)
struct f2 {
  unsigned long long v;
};

__device__ __forceinline__ f2 f2_pack(float lo, float hi)
{
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ f2 f2_dup(float x) { return f2_pack(x, x); }
__device__ __forceinline__ float f2_lo(f2 a)
{
  float lo;
  asm("{\n .reg .f32 t;\n mov.b64 {%0, t}, %1;\n}" : "=f"(lo) : "l"(a.v));
  return lo;
}
__device__ __forceinline__ float f2_hi(f2 a)
{
  float hi;
  asm("{\n .reg .f32 t;\n mov.b64 {t, %0}, %1;\n}" : "=f"(hi) : "l"(a.v));
  return hi;
}
__device__ __forceinline__ f2 add2(f2 a, f2 b)
{
  f2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b)
{
  f2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b)
{
  f2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c)
{
  f2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}
__device__ __forceinline__ f2 f2_of(unsigned long long v) { return f2{v}; }

// erfc polynomial coefficients as packed constants
struct ErfcConst2 {
  f2 e[8];
};

// One site pair of a water group pair: adds q_j b1 S d to the row site's field
// sum (qbs = q_j S) and q_j b0 to its unswitched potential sum (qb = q_j).
// b0 = erfc(eta r)/r, b1 = (b0 + c2 exp(-eta^2 r^2))/r^2.
__device__ __forceinline__ void water_site(float dx, float dy, float dz, float qb, float qbs, const WaterArgs &a,
                                           float &ex, float &ey, float &ez, float &tq, float &rinv_out)
{
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  const float rinv = rsqrt_approx(r2);
  const float t = rcp_approx(fmaf(a.pe, r2 * rinv, 1.f));
  float p = fmaf(kE7, t, kE6);
  p = fmaf(p, t, kE5);
  p = fmaf(p, t, kE4);
  p = fmaf(p, t, kE3);
  p = fmaf(p, t, kE2);
  p = fmaf(p, t, kE1);
  p = fmaf(p, t, kE0);
  const float e = ex2_approx(r2 * a.nel2);
  const float b0 = (t * p) * (e * rinv);
  tq = fmaf(qb, b0, tq);
  const float f = fmaf(a.c2, e, b0) * (rinv * rinv) * qbs;
  ex = fmaf(f, dx, ex);
  ey = fmaf(f, dy, ey);
  ez = fmaf(f, dz, ez);
  rinv_out = rinv;
}

// The same for two site pairs at once (the halves of each packed value are
// independent site pairs): the arithmetic of water_site, half by half.
struct WaterConst2 {
  f2 pe, one, nel2, c2;
};

__device__ __forceinline__ void water_site2(f2 dx, f2 dy, f2 dz, f2 qb, f2 qbs, const WaterConst2 &c,
                                            const ErfcConst2 &k, f2 &ex, f2 &ey, f2 &ez, f2 &tq)
{
  const f2 r2 = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
  const f2 rinv = f2_pack(rsqrt_approx(f2_lo(r2)), rsqrt_approx(f2_hi(r2)));
  const f2 targ = fma2(c.pe, mul2(r2, rinv), c.one);
  const f2 t = f2_pack(rcp_approx(f2_lo(targ)), rcp_approx(f2_hi(targ)));
  f2 p = fma2(k.e[7], t, k.e[6]);
  p = fma2(p, t, k.e[5]);
  p = fma2(p, t, k.e[4]);
  p = fma2(p, t, k.e[3]);
  p = fma2(p, t, k.e[2]);
  p = fma2(p, t, k.e[1]);
  p = fma2(p, t, k.e[0]);
  const f2 earg = mul2(r2, c.nel2);
  const f2 e = f2_pack(ex2_approx(f2_lo(earg)), ex2_approx(f2_hi(earg)));
  const f2 b0 = mul2(mul2(t, p), mul2(e, rinv));
  tq = fma2(qb, b0, tq);
  const f2 f = mul2(mul2(fma2(c.c2, e, b0), mul2(rinv, rinv)), qbs);
  ex = fma2(f, dx, ex);
  ey = fma2(f, dy, ey);
  ez = fma2(f, dz, ez);
}

// Minimum-image anchor displacement with contracted FP64 arithmetic (fewer
// instructions than the reference-rounded form the FP64 kernels use).  The
// decision it feeds only matters at r = rc, where the switch and its
// derivative are zero, so the pair set may differ from the FP64 form's only
// by pairs that contribute nothing.
__device__ __forceinline__ double anchor_disp_fast(const Box &b, double4 ri, double4 rj, double &x, double &y,
                                                   double &z)
{
  x = ri.x - rj.x;
  y = ri.y - rj.y;
  z = ri.z - rj.z;
  x = fma(-b.L[0], rint(x * b.invL[0]), x);
  y = fma(-b.L[1], rint(y * b.invL[1]), y);
  z = fma(-b.L[2], rint(z * b.invL[2]), z);
  return fma(x, x, fma(y, y, z * z));
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"((unsigned) __cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}

__device__ __forceinline__ void cp_async8(void *dst, const void *src)
{
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned) __cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Anchor displacement (row minus partner) from the cell-relative FP32 anchors:
// the integer cell difference wrapped to [-n/2, n/2] (exact), times the cell
// edge, plus the offset difference, and one FP32 minimum-image correction,
// which only pairs near half the box reach.  The offsets and the cell edge
// are below ~5 A, so the result is within ~1e-6 A of the exact minimum-image
// displacement for every pair a row can list (the FP64 form tests the cutoff
// on the reference's rounding; here, as in the other mixed kernels, the pair
// set may differ from it only by pairs at the cutoff, where the switch and its
// derivative vanish).
__device__ __forceinline__ float3 cell_disp(const WaterArgs &a, float4 ai, float4 aj)
{
  const int ci = __float_as_int(ai.w), cj = __float_as_int(aj.w);
  const int dc[3] = {(ci & 1023) - (cj & 1023), ((ci >> 10) & 1023) - ((cj >> 10) & 1023),
                     ((ci >> 20) & 1023) - ((cj >> 20) & 1023)};
  const float dof[3] = {ai.x - aj.x, ai.y - aj.y, ai.z - aj.z};
  float v[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    int d = dc[k];
    d -= d > a.nhalf ? a.ncell : 0;
    d += d < -a.nhalf ? a.ncell : 0;
    // float(d) without a conversion instruction: 1.5 * 2^23 + d is exact
    const float df = __int_as_float(d + 0x4B400000) - 12582912.0f;
    float x = fmaf(df, a.edge[k], dof[k]);
    x -= x > a.halfL[k] ? a.Lf[k] : 0.f;
    x += x < -a.halfL[k] ? a.Lf[k] : 0.f;
    v[k] = x;
  }
  return make_float3(v[0], v[1], v[2]);
}

// The row group's own constants in the rigid-water kernels: H offsets and
// charges, O charge and LJ parameters, the FP64 anchor, packed constants.
struct WaterRow {
  f2 h12x, h12y, h12z, h21x, h21y, h21z;
  float qO, qH1, qH2;
  float2 ljo;
  float qO32, qH1_32, qH2_32;  // charges times the fixed-point scale
  WaterConst2 c2;
  ErfcConst2 ke;
  float4 ai;  // cell-relative FP32 anchor
};

// UNI: every water has the same parameters (taken from the arguments)
template <bool UNI>
__device__ __forceinline__ WaterRow water_row_consts(const WaterArgs &a, int p)
{
  constexpr float kTwo32 = 4294967296.0f;
  WaterRow w;
  const float4 r0 = a.site[3 * (size_t) p], r1 = a.site[3 * (size_t) p + 1];
  const float4 r2 = UNI ? make_float4(a.uqO, a.uqO, a.usig, a.useps) : a.site[3 * (size_t) p + 2];
  w.ai = a.anc32[p];
  w.h12x = f2_pack(r0.x, r0.y);
  w.h12y = f2_pack(r0.z, r0.w);
  w.h12z = f2_pack(r1.x, r1.y);
  w.h21x = f2_pack(r0.y, r0.x);
  w.h21y = f2_pack(r0.w, r0.z);
  w.h21z = f2_pack(r1.y, r1.x);
  w.qO = r2.x;
  w.qH1 = UNI ? a.uqH : r1.z;
  w.qH2 = UNI ? a.uqH : r1.w;
  w.ljo = make_float2(r2.z, r2.w);
  // the converted values come out of the last product directly
  w.qO32 = w.qO * kTwo32;
  w.qH1_32 = w.qH1 * kTwo32;
  w.qH2_32 = w.qH2 * kTwo32;
  w.c2.pe = f2_dup(a.pe);
  w.c2.one = f2_dup(1.f);
  w.c2.nel2 = f2_dup(a.nel2);
  w.c2.c2 = f2_dup(a.c2);
  w.ke.e[0] = f2_dup(kE0);
  w.ke.e[1] = f2_dup(kE1);
  w.ke.e[2] = f2_dup(kE2);
  w.ke.e[3] = f2_dup(kE3);
  w.ke.e[4] = f2_dup(kE4);
  w.ke.e[5] = f2_dup(kE5);
  w.ke.e[6] = f2_dup(kE6);
  w.ke.e[7] = f2_dup(kE7);
  return w;
}

// One group pair inside the cutoff: da = anchor displacement (xyz) and its
// r^2, j0, j1, j2 = the partner's three packed slots.  Adds the row sites'
// fixed-point force words, the pair energies and (VIR) the virial term to fx.
// With UNI the partner's charges and LJ parameters are the arguments' and
// only j0 and the first half of j1 (the H offsets) are read.
template <bool VIR, bool UNI>
__device__ __forceinline__ void water_pair(const WaterArgs &a, const WaterRow &w, float4 da, ulonglong2 j0,
                                           ulonglong2 j1, float4 j2, long long (&fx)[VIR ? 12 : 11])
{
  constexpr float kTwo32 = 4294967296.0f, kTwo31 = 2147483648.0f;
  if (UNI)
    j2 = make_float4(a.uqO, a.uqO, a.usig, a.useps);
  const f2 jx = f2_of(j0.x), jy = f2_of(j0.y), jz = f2_of(j1.x), qj = UNI ? f2_dup(a.uqH) : f2_of(j1.y);
  const float qjO = j2.x;
  // switch S(z) and dS/dr^2 (zero inside rc - width), branch-free
  const float z = fmaxf(da.w - a.rlo2, 0.f) * a.inv_sw;
  const float zz = z * z;
  const float s = fmaf(fmaf(fmaf(-6.f, z, 15.f), z, -10.f), zz * z, 1.f);
  const float ds = fmaf(fmaf(60.f, z, -120.f), z, 60.f) * zz * a.inv_sw;
  const f2 s2 = f2_dup(s);
  const f2 qbs = mul2(qj, s2);
  const f2 q0d = f2_pack(j2.x, j2.y);
  const f2 q0s = mul2(q0d, s2);
  const f2 dx = f2_dup(da.x), dy = f2_dup(da.y), dz = f2_dup(da.z);
  // row O against partner O (single) and partner H1, H2 (packed)
  float eOx = 0.f, eOy = 0.f, eOz = 0.f, tO = 0.f, rOO;
  water_site(da.x, da.y, da.z, qjO, qjO * s, a, eOx, eOy, eOz, tO, rOO);
  f2 aOx = f2_dup(0.f), aOy = aOx, aOz = aOx, aOt = aOx;
  water_site2(sub2(dx, jx), sub2(dy, jy), sub2(dz, jz), qj, qbs, w.c2, w.ke, aOx, aOy, aOz, aOt);
  // rows H1, H2 against partner O, then against partner H1, H2 in order
  const f2 cx = add2(dx, w.h12x), cy = add2(dy, w.h12y), cz = add2(dz, w.h12z);
  f2 hx = f2_dup(0.f), hy = hx, hz = hx, ht = hx;
  water_site2(cx, cy, cz, q0d, q0s, w.c2, w.ke, hx, hy, hz, ht);
  water_site2(sub2(cx, jx), sub2(cy, jy), sub2(cz, jz), qj, qbs, w.c2, w.ke, hx, hy, hz, ht);
  // rows H2, H1 against partner H1, H2
  f2 vx = f2_dup(0.f), vy = vx, vz = vx, vt = vx;
  water_site2(sub2(add2(dx, w.h21x), jx), sub2(add2(dy, w.h21y), jy), sub2(add2(dz, w.h21z), jz), qj, qbs, w.c2,
              w.ke, vx, vy, vz, vt);
  eOx += f2_lo(aOx) + f2_hi(aOx);
  eOy += f2_lo(aOy) + f2_hi(aOy);
  eOz += f2_lo(aOz) + f2_hi(aOz);
  tO += f2_lo(aOt) + f2_hi(aOt);
  const float e1x = f2_lo(hx) + f2_hi(vx), e1y = f2_lo(hy) + f2_hi(vy), e1z = f2_lo(hz) + f2_hi(vz);
  const float e2x = f2_hi(hx) + f2_lo(vx), e2y = f2_hi(hy) + f2_lo(vy), e2z = f2_hi(hz) + f2_lo(vz);
  const float t1 = f2_lo(ht) + f2_hi(vt), t2 = f2_hi(ht) + f2_lo(vt);
  // O-O Lennard-Jones
  const float sj = j2.z, ej = j2.w;
  const float sg = a.geometric ? w.ljo.x * sj : 0.5f * (w.ljo.x + sj);
  const float sq = a.geometric ? sg : sg * sg;
  const float s6 = sq * sq * sq;
  const float b = 4.f * w.ljo.y * ej * s6;
  const float ir2 = rOO * rOO;
  const float ir6 = ir2 * ir2 * ir2;
  const float bi6 = b * ir6;
  const float ai12 = b * s6 * ir6 * ir6;
  const float u = ai12 - bi6;
  const float du = (12.f * ai12 - 6.f * bi6) * ir2 * s;
  // unswitched Coulomb energy of the group pair; its switched half is the
  // row's energy share and, with u, it scales the switch derivative
  const float tq = fmaf(w.qO, tO, fmaf(w.qH1, t1, w.qH2 * t2));
  const float g = ds * (tq + u);
  const float fo32 = (du + g) * kTwo32;
  const float s31 = s * kTwo31;
  fx[0] += __float2ll_rn(fmaf(w.qO32, eOx, fo32 * da.x));
  fx[1] += __float2ll_rn(fmaf(w.qO32, eOy, fo32 * da.y));
  fx[2] += __float2ll_rn(fmaf(w.qO32, eOz, fo32 * da.z));
  fx[3] += __float2ll_rn(w.qH1_32 * e1x);
  fx[4] += __float2ll_rn(w.qH1_32 * e1y);
  fx[5] += __float2ll_rn(w.qH1_32 * e1z);
  fx[6] += __float2ll_rn(w.qH2_32 * e2x);
  fx[7] += __float2ll_rn(w.qH2_32 * e2y);
  fx[8] += __float2ll_rn(w.qH2_32 * e2z);
  fx[9] += __float2ll_rn(tq * s31);
  fx[10] += __float2ll_rn(u * s31);
  if constexpr (VIR)
    fx[11] += __float2ll_rn(0.5f * fo32 * da.w);  // each pair is seen from both rows
}

// One row group p, partners queued through the warp's ring: walks the row's
// list (full rows, making the pruned ones, or the pruned rows) 64 entries per
// step, two per lane, with the next step's 64 anchors already requested and
// the list indices a step further ahead (a row has only a few steps, so each
// step's load latency is what the walk waits on); each lane tests its
// partners' anchor distances, an accepted partner's displacement goes to the
// ring and its record is copied there (cp.async); 32 queued pairs are
// evaluated at a time, one per lane.  qa, q0, q1, q2: the warp's ring.
// Returns the row's first site.
template <bool VIR, bool UNI>
__device__ __forceinline__ int water_row(const WaterArgs &a, int p, int lane, float4 *qa, float4 *q0, float4 *q1,
                                         float4 *q2, long long (&fx)[VIR ? 12 : 11])
{
  constexpr int kMask = kWaterRing - 1;
  const WaterRow w = water_row_consts<UNI>(a, p);
  const int si0 = a.group[2 * a.sorted[p]];
  // full rows (and make the pruned ones), or the pruned rows
  const bool make = a.pnbr && a.flags[kFlagPruneFull];
  const bool use_pruned = a.pnbr && !make;
  const int cnt = use_pruned ? a.pcount[p] : a.nbr_count[p];
  const int *row = (use_pruned ? a.pnbr : a.nbr) + (size_t) p * a.rowcap;
  int *prow = make ? a.pnbr + (size_t) p * a.rowcap : nullptr;
  int pn = 0;
  const unsigned below = (1u << lane) - 1;
  auto compute = [&](int k) {
    water_pair<VIR, UNI>(a, w, qa[k], *reinterpret_cast<const ulonglong2 *>(&q0[k]),
                         *reinterpret_cast<const ulonglong2 *>(&q1[k]), UNI ? make_float4(0.f, 0.f, 0.f, 0.f) : q2[k],
                         fx);
  };
  // Entries past the row end read the row's own group (a valid address);
  // they are never accepted.
  int jc0 = lane < cnt ? row[lane] : p, jc1 = lane + 32 < cnt ? row[lane + 32] : p;
  int jn0 = lane + 64 < cnt ? row[lane + 64] : p, jn1 = lane + 96 < cnt ? row[lane + 96] : p;
  float4 ac0 = a.anc32[jc0], ac1 = a.anc32[jc1];
  int head = 0, qn = 0;  // ring entries [head, head + qn)
  for (int base2 = 0; base2 < cnt; base2 += 64) {
    const int e2 = base2 + 128 + lane;
    const int jnn0 = e2 < cnt ? row[e2] : p, jnn1 = e2 + 32 < cnt ? row[e2 + 32] : p;
    const float4 an0 = a.anc32[jn0], an1 = a.anc32[jn1];
#pragma unroll
    for (int hh = 0; hh < 2; hh++) {
      const int base = base2 + 32 * hh;
      const int jc = hh ? jc1 : jc0;
      const float4 ac = hh ? ac1 : ac0;
      const float3 d = cell_disp(a, w.ai, ac);
      const float r2 = fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z));
      const bool take = base + lane < cnt && r2 <= a.rhi2f;
      if (make) {
        const bool keep = base + lane < cnt && r2 <= a.rp2f;
        const unsigned kb = __ballot_sync(0xffffffffu, keep);
        if (keep)
          prow[pn + __popc(kb & below)] = jc;
        pn += __popc(kb);
      }
      const unsigned bal = __ballot_sync(0xffffffffu, take);
      if (take) {
        const int slot = (head + qn + __popc(bal & below)) & kMask;
        qa[slot] = make_float4(d.x, d.y, d.z, r2);
        const float4 *src = a.site + 3 * (size_t) jc;
        cp_async16(&q0[slot], src);
        if (UNI) {
          cp_async8(&q1[slot], src + 1);  // the H z offsets; the charges are the arguments'
        } else {
          cp_async16(&q1[slot], src + 1);
          cp_async16(&q2[slot], src + 2);
        }
      }
      cp_async_commit();
      // entries of earlier batches are evaluated one batch after their copies
      // were started, so the copies are normally complete by then
      const bool run = qn >= 32;
      qn += __popc(bal);
      if (run) {
        cp_async_wait_prev();
        __syncwarp();
        compute((head + lane) & kMask);
        __syncwarp();  // the slots are free again only after every lane has read them
        head = (head + 32) & kMask;
        qn -= 32;
      }
    }
    jc0 = jn0;
    jc1 = jn1;
    jn0 = jnn0;
    jn1 = jnn1;
    ac0 = an0;
    ac1 = an1;
  }
  cp_async_wait_all();
  __syncwarp();
  for (; qn > 0; qn -= 32, head = (head + 32) & kMask)
    if (lane < qn)
      compute((head + lane) & kMask);
  if (make && lane == 0) {
    // the anchors at this prune (FP64: the list check measures moves from them)
    const double4 ai = a.anchor[p];
    a.pcount[p] = pn;
    a.plast[3 * p] = ai.x;
    a.plast[3 * p + 1] = ai.y;
    a.plast[3 * p + 2] = ai.z;
  }
  return si0;
}

// The lanes' fixed-point totals of a finished row by a butterfly
// reduce-scatter over the warp (no shared memory): the 16 columns (the totals,
// padded) halve at each of four exchange steps, each lane keeping the half
// its lane bit selects, and a last exchange completes the sum, so the lane
// pair (2c, 2c+1) holds the total of column c.  Integer sums: the same bits as
// any other order.  The nine force words go to acc, the potential and field
// words of the three sites are cleared (P3M adds to them), and every lane gets
// the row's Coulomb and LJ pair energies and virial term.
template <bool VIR>
__device__ __forceinline__ void water_row_store_shfl(const WaterArgs &a, int si0, int lane,
                                                     const long long (&fx)[VIR ? 12 : 11], long long &te,
                                                     long long &tl, long long &tv)
{
  constexpr int kCols = VIR ? 12 : 11;
  long long v[16];
#pragma unroll
  for (int c = 0; c < 16; c++)
    v[c] = c < kCols ? fx[c] : 0;
#pragma unroll
  for (int half = 8; half >= 1; half >>= 1) {
    const bool up = lane & (2 * half);
#pragma unroll
    for (int k = 0; k < half; k++) {
      const long long keep = up ? v[k + half] : v[k];
      const long long send = up ? v[k] : v[k + half];
      v[k] = keep + __shfl_xor_sync(0xffffffffu, send, 2 * half);
    }
  }
  const long long t = v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
  const int c = (lane >> 1) & 15;
  if (!(lane & 1)) {
    if (c < 9)
      a.acc[(size_t) (si0 + c / 3) * kAccStride + 4 + c % 3] = t;
  } else if (c < 12) {
    a.acc[(size_t) (si0 + c / 4) * kAccStride + c % 4] = 0;
  }
  te = __shfl_sync(0xffffffffu, t, 2 * 9);
  tl = __shfl_sync(0xffffffffu, t, 2 * 10);
  tv = VIR ? __shfl_sync(0xffffffffu, t, 2 * 11) : 0;
}

// MINB: resident warps per SM / 4 the register budget is cut for (4: 128
// registers, 5: 96); mmnb_autotune picks per handle
// VIR: also the part of dU/ds (box scaling) the site forces do not carry, the
// anchor force scalar times R^2 per group pair (mmnb_virial)
template <int MINB, bool VIR, bool UNI>
__global__ void __launch_bounds__(kWaterWarps * 32, MINB * kMxWarps / kWaterWarps) k_pair_water(WaterArgs a)
{
  // per warp: ring of anchor displacement (xyz, r^2) and the partner's three
  // packed slots
  __shared__ float4 ring[kWaterWarps][4][kWaterRing];
  __shared__ long long wsum[kWaterWarps][3];
  constexpr int kCols = VIR ? 12 : 11;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int p = blockIdx.x * kWaterWarps + w;
  long long te = 0, tl = 0, tv = 0;
  if (p < a.ngroup) {
    long long fx[kCols];
#pragma unroll
    for (int c = 0; c < kCols; c++)
      fx[c] = 0;
    const int si0 = water_row<VIR, UNI>(a, p, lane, ring[w][0], ring[w][1], ring[w][2], ring[w][3], fx);
    water_row_store_shfl<VIR>(a, si0, lane, fx, te, tl, tv);
  }
  if (a.pnbr && a.flags[kFlagPruneFull] && blockIdx.x == 0 && threadIdx.x == 0)
    a.flags[kFlagPruneValid] = 1;
  if (lane == 0) {
    wsum[w][0] = te;
    wsum[w][1] = tl;
    wsum[w][2] = tv;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kWaterWarps; k++) {
      te += wsum[k][0];
      tl += wsum[k][1];
      tv += wsum[k][2];
    }
    // integer sums: the totals do not depend on the order blocks finish in
    atomicAdd(a.wsum, (unsigned long long) te);
    atomicAdd(a.wsum + 1, (unsigned long long) tl);
    if (VIR)
      atomicAdd(a.wsum + 4, (unsigned long long) tv);
  }
}

cudaError_t launch_rspace_water(mmnb_handle *h)
{
  WaterArgs a;
  a.ngroup = h->ngroup;
  a.rowcap = h->rowcap;
  a.geometric = h->cfg.geometric_combining_for_sigma;
  a.box = h->box;
  a.rhi2 = h->rhi2;
  a.rlo2 = (float) h->rlo2;
  a.inv_sw = (float) h->inv_sw;
  a.pe = (float) (h->eta * kErfcP);
  a.c2 = (float) (h->eta * M_2_SQRTPI);
  a.nel2 = (float) (-h->eta * h->eta * M_LOG2E);
  a.site = h->mx.site;
  a.anchor = h->mx.anchor;
  a.nbr = h->d_nbr;
  a.nbr_count = h->d_nbr_count;
  a.sorted = h->d_sorted;
  a.group = h->d_group;
  a.acc = h->mx.acc;
  a.wsum = h->d_wsum;
  a.pnbr = h->prune_margin > 0 ? h->d_pnbr : nullptr;
  a.pcount = h->d_pcount;
  a.plast = h->d_plast;
  a.flags = h->d_flags;
  a.rp2 = (h->rc + h->prune_margin) * (h->rc + h->prune_margin);
  a.anc32 = h->mx.anc32;
  a.ncell = h->cg.n;
  a.nhalf = h->cg.n / 2;
  for (int d = 0; d < 3; d++) {
    a.edge[d] = (float) h->cg.lc[d];
    a.Lf[d] = (float) h->box.L[d];
    a.halfL[d] = (float) (0.5 * h->box.L[d]);
  }
  a.rhi2f = (float) a.rhi2;
  a.rp2f = (float) a.rp2;
  a.uqO = h->uni_qO;
  a.uqH = h->uni_qH;
  a.usig = h->uni_sig;
  a.useps = h->uni_seps;
  h->launches += 1;
  const int blocks = div_up(h->ngroup, kWaterWarps);
  const bool uni = h->water_uni;
  if (h->want_virial && uni)
    k_pair_water<4, true, true><<<blocks, kWaterWarps * 32, 0, h->stream>>>(a);
  else if (h->want_virial)
    k_pair_water<4, true, false><<<blocks, kWaterWarps * 32, 0, h->stream>>>(a);
  else if (h->tune.water_minb == 5 && uni)
    k_pair_water<5, false, true><<<blocks, kWaterWarps * 32, 0, h->stream>>>(a);
  else if (h->tune.water_minb == 5)
    k_pair_water<5, false, false><<<blocks, kWaterWarps * 32, 0, h->stream>>>(a);
  else if (uni)
    k_pair_water<4, false, true><<<blocks, kWaterWarps * 32, 0, h->stream>>>(a);
  else
    k_pair_water<4, false, false><<<blocks, kWaterWarps * 32, 0, h->stream>>>(a);
  return cudaGetLastError();
}

// Per step: sorted FP32 slots and the FP64 anchors.  General layout (any
// groups, k_pair_mixed): per group G slots of (offset from anchor, charge) and
// (sigma, sqrt(epsilon), rscreen, mask), padded with empty slots.  Rigid-water
// layout (k_pair_water): per group three packed slots, (h1x, h2x, h1y, h2y),
// (h1z, h2z, q1, q2), (qO, qO, sigma_O, sqrt(epsilon_O)).
__global__ void k_prep_mixed(const double *__restrict__ r, const double *__restrict__ q,
                             const double *__restrict__ sig, const double *__restrict__ eps,
                             const double *__restrict__ rscreen, const int *__restrict__ mask,
                             const int *__restrict__ sorted, const int *__restrict__ group, int ngroup, int G,
                             int water, float4 *__restrict__ site, float4 *__restrict__ par,
                             double4 *__restrict__ anchor, unsigned long long *__restrict__ wsum,
                             int *__restrict__ flags, float4 *__restrict__ anc32, Box box, int ncell,
                             double3 edge, double3 inv_edge)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < 2)
    wsum[s] = 0ull;
  if (s == 2)
    wsum[4] = 0ull;
  if (s >= ngroup * G)
    return;
  const int p = s / G, k = s % G;
  const int g = sorted[p];
  const int a0 = group[2 * g];
  const double ax = r[3 * a0], ay = r[3 * a0 + 1], az = r[3 * a0 + 2];
  if (k == 0)
    anchor[p] = make_double4(ax, ay, az, 0.0);
  // a non-finite coordinate is flagged (the host reports it); every index
  // below stays in range whatever the coordinates
  if (a0 + k < group[2 * g + 1] &&
      !isfinite(r[3 * (a0 + k)] + r[3 * (a0 + k) + 1] + r[3 * (a0 + k) + 2]))
    flags[kFlagError] = MMNB_ERR_DEVICE;
  if (water) {
    if (k == 0) {
      // the anchor wrapped into the box, its list cell (edge as the kernel
      // holds it, in FP32) and its offset from that cell's corner
      // (any cell near the anchor serves: the offset is taken from the cell
      // chosen, so the cell index needs no exact division)
      const double av[3] = {ax, ay, az}, ev[3] = {edge.x, edge.y, edge.z}, iv[3] = {inv_edge.x, inv_edge.y, inv_edge.z};
      float o[3];
      int code = 0;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const double wv = av[d] - box.L[d] * floor(av[d] * box.invL[d]);
        int c = (int) floor(wv * iv[d]);
        c = min(max(c, 0), ncell - 1);
        o[d] = (float) (wv - c * ev[d]);
        code |= c << (10 * d);
      }
      anc32[p] = make_float4(o[0], o[1], o[2], __int_as_float(code));
    }
    // G == 3: slot k of group p from the two H sites (a0 + 1, a0 + 2) and O
    const int h1 = a0 + 1, h2 = a0 + 2;
    float4 v;
    if (k == 0)
      v = make_float4((float) (r[3 * h1] - ax), (float) (r[3 * h2] - ax), (float) (r[3 * h1 + 1] - ay),
                      (float) (r[3 * h2 + 1] - ay));
    else if (k == 1)
      v = make_float4((float) (r[3 * h1 + 2] - az), (float) (r[3 * h2 + 2] - az), (float) q[h1], (float) q[h2]);
    else
      v = make_float4((float) q[a0], (float) q[a0], (float) sig[a0], (float) sqrt(eps[a0]));
    site[s] = v;
    return;
  }
  const int st = a0 + k;
  if (st < group[2 * g + 1]) {
    const float ox = (float) (r[3 * st] - ax), oy = (float) (r[3 * st + 1] - ay), oz = (float) (r[3 * st + 2] - az);
    site[s] = make_float4(ox, oy, oz, (float) q[st]);
    par[s] = make_float4((float) sig[st], (float) sqrt(eps[st]), (float) rscreen[st], __int_as_float(mask[st]));
  } else {
    site[s] = make_float4(0.f, 0.f, 0.f, 0.f);
    par[s] = make_float4(0.f, 0.f, 0.f, __int_as_float(0));
  }
}

cudaError_t launch_prep_mixed(mmnb_handle *h, const double *d_r)
{
  const int n = h->ngroup * h->G;
  const int water = h->water && !h->want_fields && h->cfg.include_rspace;
  const double3 edge = make_double3((float) h->cg.lc[0], (float) h->cg.lc[1], (float) h->cg.lc[2]);
  const double3 inv_edge = make_double3(1.0 / edge.x, 1.0 / edge.y, 1.0 / edge.z);
  k_prep_mixed<<<div_up(n, 256), 256, 0, h->stream>>>(d_r, h->d_q, h->d_sig, h->d_eps, h->d_rscreen, h->d_mask,
                                                      h->d_sorted, h->d_group, h->ngroup, h->G, water, h->mx.site,
                                                      h->mx.par, h->mx.anchor, h->d_wsum, h->d_flags, h->mx.anc32,
                                                      h->box, h->cg.n, edge, inv_edge);
  h->launches += 1;
  return cudaGetLastError();
}

template <int G, bool ANCHOR_LJ>
static void launch_mixed_g(mmnb_handle *h, const MixedArgs &a)
{
  const int blocks = pair_blocks(h);
  const int threads = kMxWarps * 32;
  h->launches += 1;
  if (h->has_rscreen) {
    if (h->any_gexcl)
      k_pair_mixed<G, true, true, ANCHOR_LJ><<<blocks, threads, 0, h->stream>>>(a);
    else
      k_pair_mixed<G, true, false, ANCHOR_LJ><<<blocks, threads, 0, h->stream>>>(a);
  } else {
    if (h->any_gexcl)
      k_pair_mixed<G, false, true, ANCHOR_LJ><<<blocks, threads, 0, h->stream>>>(a);
    else
      k_pair_mixed<G, false, false, ANCHOR_LJ><<<blocks, threads, 0, h->stream>>>(a);
  }
}

cudaError_t launch_rspace_mixed(mmnb_handle *h)
{
  MixedArgs a;
  a.ngroup = h->ngroup;
  a.rowcap = h->rowcap;
  a.geometric = h->cfg.geometric_combining_for_sigma;
  a.box = h->box;
  a.rhi2 = h->rhi2;
  a.rlo2 = (float) h->rlo2;
  a.inv_sw = (float) h->inv_sw;
  a.eta = (float) h->eta;
  a.c2 = (float) (h->eta * M_2_SQRTPI);
  a.nel2 = (float) (-h->eta * h->eta * M_LOG2E);
  a.site = h->mx.site;
  a.par = h->mx.par;
  a.anchor = h->mx.anchor;
  a.nbr = h->d_nbr;
  a.nbr_count = h->d_nbr_count;
  a.sorted = h->d_sorted;
  a.group = h->d_group;
  a.gexcl_ptr = h->d_gexcl_ptr;
  a.gexcl_idx = h->d_gexcl_idx;
  a.excl_ptr = h->d_excl_ptr;
  a.excl_idx = h->d_excl_idx;
  a.acc = h->mx.acc;
  a.lj_part = h->d_lj_part;
  a.vir_part = h->want_virial ? h->d_vir_part : nullptr;
  const bool alj = h->lj_on_anchors_only;
  switch (h->G) {
  case 1: launch_mixed_g<1, false>(h, a); break;
  case 2: alj ? launch_mixed_g<2, true>(h, a) : launch_mixed_g<2, false>(h, a); break;
  case 3: alj ? launch_mixed_g<3, true>(h, a) : launch_mixed_g<3, false>(h, a); break;
  case 4: alj ? launch_mixed_g<4, true>(h, a) : launch_mixed_g<4, false>(h, a); break;
  default: launch_mixed_g<8, false>(h, a); break;
  }
  return cudaGetLastError();
}

}  // namespace mmnb

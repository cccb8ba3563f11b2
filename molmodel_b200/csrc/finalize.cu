// Self terms, force assembly and energies (src/eleclj.cpp:794-805, 961-976).
//
// Per site: phi -= (2 eta / sqrt(pi)) q, plus the neutralising background
// -pi/(eta^2 V) sum(q) when the system is charged; F += q E + F_LJ (AtomSite
// projection, include/eleclj.hpp:68-71).  Energies: elec = (q . phi)/2 and
// LJ = pair sum + tail.  Each block writes its partial sum; the last block to
// finish (a counter taken after a fence) adds the partials in index order, so
// the FP64 energies are bitwise reproducible without a second launch.

#include "mmnb_internal.cuh"

namespace mmnb {

constexpr int kFinThreads = 256;

struct FinArgs {
  int nsite, do_self;
  int keep_fields;       // write phi, E and the LJ force back (the caller asked for the site fields)
  double self_a, neutral_b;
  const double *q;
  const long long *acc;  // mixed form: fixed-point potential, field and LJ force per site
  const long long *acck; // mixed P3M: fixed-point interpolated potential and field per site
  double *phi, *evec, *ljf, *f, *elec_part;
  // energy reduction
  const double *lj_part;              // per-block LJ partials [lj_lo, lj_hi)
  int lj_lo, lj_hi, any_q;
  const double *lj_row;               // FP64 water kernel: per-row LJ energies [0, nrow), or null
  int nrow;
  double *lj_row_part;                // per block: its slice of lj_row
  const unsigned long long *wsum;     // water kernel's fixed-point pair energies, or null
  unsigned long long *counter;        // finished-block counter, left at 0
  int *flags;                         // list flags: counts evaluations finished on cut rows
  double *status;                     // or null: the host call's mapped status block
                                      // (energies, flags, ready word)
  double tail;
  double *energy;
};

// sum over the block in a fixed order: lanes by a shuffle tree, then the
// warps' sums in warp order (sh: one slot per warp plus one)
__device__ __forceinline__ double block_sum(double v, double *sh)
{
  constexpr int kWarps = kFinThreads / 32;
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0)
    sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < kWarps; w++)
      t += sh[w];
    sh[kWarps] = t;
  }
  __syncthreads();
  const double t = sh[kWarps];
  __syncthreads();  // sh may be reused at once
  return t;
}

__global__ void __launch_bounds__(kFinThreads) k_finalize(FinArgs a)
{
  __shared__ double se[kFinThreads / 32 + 1];
  __shared__ bool last;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0;
  if (i < a.nsite) {
    const double qi = a.q[i];
    double p = a.phi[i];
    double ev[3], lf[3];
    for (int d = 0; d < 3; d++) {
      ev[d] = a.evec[3 * i + d];
      lf[d] = a.ljf[3 * i + d];
    }
    if (a.acc) {
      // fold the fixed-point sums into the FP64 site values (one site's words
      // are 64 contiguous bytes: four 16-byte loads)
      const longlong2 *o2 = reinterpret_cast<const longlong2 *>(a.acc + (size_t) i * kAccStride);
      const longlong2 w01 = o2[0], w23 = o2[1], w45 = o2[2], w67 = o2[3];
      const long long o[7] = {w01.x, w01.y, w23.x, w23.y, w45.x, w45.y, w67.x};
      long long k[4] = {0, 0, 0, 0};
      if (a.acck) {
        const longlong4 v = reinterpret_cast<const longlong4 *>(a.acck)[i];
        k[0] = v.x;
        k[1] = v.y;
        k[2] = v.z;
        k[3] = v.w;
      }
      p += (double) (o[0] + k[0]) * kFxInv;
      for (int d = 0; d < 3; d++) {
        ev[d] += (double) (o[1 + d] + k[1 + d]) * kFxInv;
        lf[d] += (double) o[4 + d] * kFxInv;
      }
    }
    if (a.do_self) {
      p -= a.self_a * qi;
      p += a.neutral_b;
    }
    e = qi * p;
    if (a.keep_fields) {
      a.phi[i] = p;
      for (int d = 0; d < 3; d++) {
        a.evec[3 * i + d] = ev[d];
        a.ljf[3 * i + d] = lf[d];
      }
    }
    if (a.f) {
      a.f[3 * i] += qi * ev[0] + lf[0];
      a.f[3 * i + 1] += qi * ev[1] + lf[1];
      a.f[3 * i + 2] += qi * ev[2] + lf[2];
    }
  }
  const double bs = block_sum(e, se);
  double rs = 0;
  if (a.lj_row) {
    // this block's slice of the per-row LJ energies (fixed slices, fixed order)
    const int per = (a.nrow + gridDim.x - 1) / gridDim.x;
    const int lo = blockIdx.x * per, hi = min(a.nrow, lo + per);
    for (int k = lo + threadIdx.x; k < hi; k += blockDim.x)
      rs += a.lj_row[k];
    rs = block_sum(rs, se);
  }
  if (threadIdx.x == 0) {
    a.elec_part[blockIdx.x] = bs;
    if (a.lj_row)
      a.lj_row_part[blockIdx.x] = rs;
    __threadfence();
    last = atomicAdd(a.counter, 1ull) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last)
    return;
  __threadfence();
  double el = 0, lj = 0;
  for (int k = threadIdx.x; k < (int) gridDim.x; k += blockDim.x)
    el += a.elec_part[k];
  for (int k = a.lj_lo + threadIdx.x; k < a.lj_hi; k += blockDim.x)
    lj += a.lj_part[k];
  if (a.lj_row)
    for (int k = threadIdx.x; k < (int) gridDim.x; k += blockDim.x)
      lj += a.lj_row_part[k];
  el = block_sum(el, se);
  lj = block_sum(lj, se);
  if (threadIdx.x == 0) {
    if (a.wsum) {
      // the water kernel's real-space Coulomb energy is a pair sum (not in phi)
      el += 2 * ((double) (long long) a.wsum[0] * kFxInv);
      lj += (double) (long long) a.wsum[1] * kFxInv;
    }
    const double elec = a.any_q ? el / 2 : 0;
    const double ljt = lj + a.tail;
    a.energy[0] = elec;
    a.energy[1] = ljt;
    a.energy[2] = a.tail;
    a.energy[3] = elec + ljt;
    *a.counter = 0ull;
    if (a.flags[kFlagListTrunc])
      a.flags[kFlagTruncEvals] += 1;
    if (a.status) {
      // over the bus to the waiting host: the block first, the ready word last
      volatile double *st = a.status;
      st[0] = elec;
      st[1] = ljt;
      st[2] = a.tail;
      st[3] = elec + ljt;
      volatile int *fl = reinterpret_cast<volatile int *>(a.status + 4);
      for (int k = 0; k < kFlagCount; k++)
        fl[k] = a.flags[k];
      __threadfence_system();
      reinterpret_cast<volatile unsigned long long *>(a.status)[mmnb_handle::kStatusReady] = 1ull;
    }
  }
}

cudaError_t launch_finalize(mmnb_handle *h, double *d_f, double *d_energy)
{
  FinArgs a;
  a.nsite = h->nsite;
  a.do_self = (h->any_q && h->cfg.include_self) ? 1 : 0;
  a.keep_fields = h->want_fields ? 1 : 0;
  a.self_a = h->eta * M_2_SQRTPI;
  // neutralising background for a charged system (src/eleclj.cpp:965-975)
  a.neutral_b = h->neutral_b;
  a.q = h->d_q;
  a.acc = h->cfg.precision == MMNB_MIXED ? h->mx.acc : nullptr;
  a.acck = (a.acc && h->any_q && h->cfg.include_kspace && h->p3m) ? h->mx.acck : nullptr;
  a.phi = h->d_phi;
  a.evec = h->d_evec;
  a.ljf = h->d_ljf;
  a.f = d_f;
  a.elec_part = h->d_elec_part;
  a.lj_part = h->d_lj_part;
  // the water kernel leaves its LJ energy in the fixed-point word, not in the
  // pair partials
  a.lj_lo = (h->used_water || h->used_water64) ? h->lj_pair_blocks : 0;
  a.lj_row = h->used_water64 ? h->d_lj_row : nullptr;
  a.nrow = h->ngroup;
  a.lj_row_part = h->d_lj_row_part;
  a.lj_hi = h->lj_pair_blocks + h->lj_excl_blocks;
  a.any_q = h->any_q ? 1 : 0;
  a.wsum = h->used_water ? h->d_wsum : nullptr;
  a.counter = h->d_wsum + 2;
  a.flags = h->d_flags;
  a.tail = h->cfg.include_lj_correction ? h->lj_correction : 0.0;
  a.energy = d_energy;
  a.status = h->want_status ? h->d_status : nullptr;
  k_finalize<<<h->elec_blocks, kFinThreads, 0, h->stream>>>(a);
  h->launches += 1;
  return cudaGetLastError();
}

}  // namespace mmnb

// Self terms, force assembly and energies (src/eleclj.cpp:794-805, 961-976).
//
// Per site: phi -= (2 eta / sqrt(pi)) q, plus the neutralising background
// -pi/(eta^2 V) sum(q) when the system is charged; F += q E + F_LJ (AtomSite
// projection, include/eleclj.hpp:68-71).  Energies: elec = (q . phi)/2 and
// LJ = pair sum + tail, reduced in a fixed order (per-block partials, then one
// block), so the FP64 energies are bitwise reproducible.

#include "mmnb_internal.cuh"

namespace mmnb {

constexpr int kFinThreads = 256;
constexpr int kEnergyThreads = 1024;

struct FinArgs {
  int nsite, do_self;
  double self_a, neutral_b;
  const double *q;
  const long long *acc;  // mixed form: fixed-point potential, field and LJ force per site
  double *phi, *evec, *ljf, *f, *elec_part;
};

__global__ void k_finalize(FinArgs a)
{
  __shared__ double se[kFinThreads];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0;
  if (i < a.nsite) {
    const double qi = a.q[i];
    double p = a.phi[i];
    if (a.acc) {
      // fold the fixed-point sums into the FP64 site arrays
      const long long *o = a.acc + (size_t) i * kAccStride;
      p += (double) o[0] * kFxInv;
      for (int d = 0; d < 3; d++) {
        a.evec[3 * i + d] += (double) o[1 + d] * kFxInv;
        a.ljf[3 * i + d] += (double) o[4 + d] * kFxInv;
      }
    }
    if (a.do_self) {
      p -= a.self_a * qi;
      p += a.neutral_b;
    }
    a.phi[i] = p;
    e = qi * p;
    if (a.f) {
      a.f[3 * i] += qi * a.evec[3 * i] + a.ljf[3 * i];
      a.f[3 * i + 1] += qi * a.evec[3 * i + 1] + a.ljf[3 * i + 1];
      a.f[3 * i + 2] += qi * a.evec[3 * i + 2] + a.ljf[3 * i + 2];
    }
  }
  se[threadIdx.x] = e;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      se[threadIdx.x] += se[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    a.elec_part[blockIdx.x] = se[0];
}

// elec = (q . phi)/2 over the site potentials, plus the real-space Coulomb
// energy summed directly by the rigid-water kernel (nep partials, already in
// final units; 0 when another pair kernel filled the site potentials)
__global__ void __launch_bounds__(kEnergyThreads) k_energy(int nelec, const double *__restrict__ elec_part, int nlj,
                                                           const double *__restrict__ lj_part, int nep,
                                                           const double *__restrict__ ep_part, double tail, int any_q,
                                                           double *__restrict__ energy)
{
  __shared__ double se[kEnergyThreads], sl[kEnergyThreads];
  double e = 0, l = 0;
  for (int i = threadIdx.x; i < nelec; i += blockDim.x)
    e += elec_part[i];
  for (int i = threadIdx.x; i < nep; i += blockDim.x)
    e += 2 * ep_part[i];
  for (int i = threadIdx.x; i < nlj; i += blockDim.x)
    l += lj_part[i];
  se[threadIdx.x] = e;
  sl[threadIdx.x] = l;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      se[threadIdx.x] += se[threadIdx.x + s];
      sl[threadIdx.x] += sl[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double elec = any_q ? se[0] / 2 : 0;
    const double lj = sl[0] + tail;
    energy[0] = elec;
    energy[1] = lj;
    energy[2] = tail;
    energy[3] = elec + lj;
  }
}

cudaError_t launch_finalize(mmnb_handle *h, double *d_f, double *d_energy)
{
  FinArgs a;
  a.nsite = h->nsite;
  a.do_self = (h->any_q && h->cfg.include_self) ? 1 : 0;
  a.self_a = h->eta * M_2_SQRTPI;
  // neutralising background for a charged system (src/eleclj.cpp:965-975)
  a.neutral_b = h->neutral_b;
  a.q = h->d_q;
  a.acc = h->cfg.precision == MMNB_MIXED ? h->mx.acc : nullptr;
  a.phi = h->d_phi;
  a.evec = h->d_evec;
  a.ljf = h->d_ljf;
  a.f = d_f;
  a.elec_part = h->d_elec_part;
  k_finalize<<<h->elec_blocks, kFinThreads, 0, h->stream>>>(a);
  const int nlj = h->lj_pair_blocks + h->lj_excl_blocks;
  k_energy<<<1, kEnergyThreads, 0, h->stream>>>(h->elec_blocks, h->d_elec_part, nlj, h->d_lj_part,
                                                 h->used_water ? h->lj_pair_blocks : 0, h->d_ep_part,
                                             h->cfg.include_lj_correction ? h->lj_correction : 0.0,
                                             h->any_q ? 1 : 0, d_energy);
  h->launches += 2;
  return cudaGetLastError();
}

}  // namespace mmnb

// Ordinary Ewald reciprocal sum (replaces kspace_new / kspace_field,
// src/kspace.c:35-174), used when use_p3m is off.
//
// Wave vectors are the half space of integer n with |n|^2 <= kc^2 + 1e-8,
// k = 2 pi inv(L)^T n, a_k = (4 pi / V) exp(-k^2 / 4 eta^2) / k^2.  The
// structure factor S(k) = sum_i q_i exp(i k.r_i) is reduced by one block per k
// (fixed-order tree, deterministic), then one thread per site sums
// phi_i += 2 a_k Re(S(k) exp(-i k.r_i)) and E_i += 2 a_k k Im(...).

#include "mmnb_internal.cuh"

namespace mmnb {

constexpr int kKThreads = 256;

__global__ void k_kspace_structure(int nsite, int nk, const double *__restrict__ r, const double *__restrict__ q,
                                   const double *__restrict__ kvec, double *__restrict__ skc)
{
  __shared__ double sc[kKThreads], ss[kKThreads];
  const int k = blockIdx.x;
  if (k >= nk)
    return;
  const double kx = kvec[3 * k], ky = kvec[3 * k + 1], kz = kvec[3 * k + 2];
  double c = 0, s = 0;
  for (int i = threadIdx.x; i < nsite; i += blockDim.x) {
    double sn, cs;
    sincos(kx * r[3 * i] + ky * r[3 * i + 1] + kz * r[3 * i + 2], &sn, &cs);
    c += q[i] * cs;
    s += q[i] * sn;
  }
  sc[threadIdx.x] = c;
  ss[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sc[threadIdx.x] += sc[threadIdx.x + w];
      ss[threadIdx.x] += ss[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    skc[2 * k] = sc[0];
    skc[2 * k + 1] = ss[0];
  }
}

__global__ void k_kspace_field(int nsite, int nk, const double *__restrict__ r, const double *__restrict__ kvec,
                               const double *__restrict__ ak, const double *__restrict__ skc,
                               double *__restrict__ phi, double *__restrict__ evec)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsite)
    return;
  const double x = r[3 * i], y = r[3 * i + 1], z = r[3 * i + 2];
  double p = 0, gx = 0, gy = 0, gz = 0;
  for (int k = 0; k < nk; k++) {
    const double kx = __ldg(kvec + 3 * k), ky = __ldg(kvec + 3 * k + 1), kz = __ldg(kvec + 3 * k + 2);
    double sn, cs;
    sincos(kx * x + ky * y + kz * z, &sn, &cs);
    const double a2 = 2 * __ldg(ak + k);
    const double cQ = __ldg(skc + 2 * k), sQ = __ldg(skc + 2 * k + 1);
    const double im = a2 * (cQ * sn - sQ * cs);
    gx += im * kx;
    gy += im * ky;
    gz += im * kz;
    p += a2 * (sQ * sn + cQ * cs);
  }
  phi[i] += p;
  evec[3 * i] += gx;
  evec[3 * i + 1] += gy;
  evec[3 * i + 2] += gz;
}

// Adjoint: sum_j q_j g_j . dE_j/dq_i for the reciprocal sum.  With
// E_j = sum_k 2 a_k k (C sin k.r_j - S cos k.r_j) and C, S linear in the
// charges, dE_j/dq_i = sum_k 2 a_k k sin(k.(r_j - r_i)), so the sum is
// sum_k 2 a_k (Ds cos k.r_i - Dc sin k.r_i) with the dipole structure factor
// Dc + i Ds = sum_j q_j (k . g_j) exp(i k.r_j).
__global__ void k_kspace_dipole_structure(int nsite, int nk, const double *__restrict__ r,
                                          const double *__restrict__ q, const double *__restrict__ g,
                                          const double *__restrict__ kvec, double *__restrict__ skd)
{
  __shared__ double sc[kKThreads], ss[kKThreads];
  const int k = blockIdx.x;
  if (k >= nk)
    return;
  const double kx = kvec[3 * k], ky = kvec[3 * k + 1], kz = kvec[3 * k + 2];
  double c = 0, s = 0;
  for (int i = threadIdx.x; i < nsite; i += blockDim.x) {
    double sn, cs;
    sincos(kx * r[3 * i] + ky * r[3 * i + 1] + kz * r[3 * i + 2], &sn, &cs);
    const double w = q[i] * (kx * g[3 * i] + ky * g[3 * i + 1] + kz * g[3 * i + 2]);
    c += w * cs;
    s += w * sn;
  }
  sc[threadIdx.x] = c;
  ss[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sc[threadIdx.x] += sc[threadIdx.x + w];
      ss[threadIdx.x] += ss[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    skd[2 * k] = sc[0];
    skd[2 * k + 1] = ss[0];
  }
}

__global__ void k_kspace_dipole_potential(int nsite, int nk, const double *__restrict__ r,
                                          const double *__restrict__ kvec, const double *__restrict__ ak,
                                          const double *__restrict__ skd, double *__restrict__ psi)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsite)
    return;
  const double x = r[3 * i], y = r[3 * i + 1], z = r[3 * i + 2];
  double p = 0;
  for (int k = 0; k < nk; k++) {
    const double kx = __ldg(kvec + 3 * k), ky = __ldg(kvec + 3 * k + 1), kz = __ldg(kvec + 3 * k + 2);
    double sn, cs;
    sincos(kx * x + ky * y + kz * z, &sn, &cs);
    p += 2 * __ldg(ak + k) * (__ldg(skd + 2 * k + 1) * cs - __ldg(skd + 2 * k) * sn);
  }
  psi[i] += p;
}

cudaError_t launch_kspace_dipole(mmnb_handle *h, const double *d_r, const double *d_g, double *d_skd,
                                 double *d_psi)
{
  if (h->nk == 0)
    return cudaSuccess;
  k_kspace_dipole_structure<<<h->nk, kKThreads, 0, h->stream>>>(h->nsite, h->nk, d_r, h->d_q, d_g, h->d_kvecs,
                                                                 d_skd);
  k_kspace_dipole_potential<<<div_up(h->nsite, 128), 128, 0, h->stream>>>(h->nsite, h->nk, d_r, h->d_kvecs,
                                                                          h->d_ak, d_skd, d_psi);
  h->launches += 2;
  return cudaGetLastError();
}

cudaError_t launch_kspace(mmnb_handle *h, const double *d_r)
{
  if (h->nk == 0)
    return cudaSuccess;
  k_kspace_structure<<<h->nk, kKThreads, 0, h->stream>>>(h->nsite, h->nk, d_r, h->d_q, h->d_kvecs, h->d_skc);
  k_kspace_field<<<div_up(h->nsite, 128), 128, 0, h->stream>>>(h->nsite, h->nk, d_r, h->d_kvecs, h->d_ak,
                                                               h->d_skc, h->d_phi, h->d_evec);
  h->launches += 2;
  return cudaGetLastError();
}

}  // namespace mmnb

// Electrostatic potential at points away from the sites (replaces
// ElecLJ::electrostatic_potential_at_gridpoints, src/eleclj.cpp:1302-1340, its
// periodic branch).  Three terms, each optional as in the reference:
//   * real space (RSpaceEwaldPhiAtGridpoints, src/rspace.c:892-967): every
//     site with a nonzero mask against every point, minimum image with the
//     reference's rounding, cut at rc on the SITE-point distance, switched
//     over [rc - w, rc], erfc(eta r)/r from the Chebyshev table inside its
//     range, the short-range screening of the site's own r_screen;
//   * reciprocal space (kspace_new + kspace_phi, src/kspace.c:35-71, 176-250):
//     the ordinary Ewald k-sum over kspace_cutoff wave vectors, whatever the
//     handle uses for forces (P3M or the k-sum); the points carry no charge, so
//     the structure factor is that of the sites alone;
//   * the neutralising term -pi/(eta^2 V) sum q when the sites are not neutral
//     (src/eleclj.cpp:1330-1338).
// There is no self term: a point is not a charge.
//
// Layout: one thread per point, the sites streamed through shared memory in
// tiles in their own order, so each point's real-space sum is added in the
// reference's site order.  The structure factor is one block per wave vector
// with a fixed-order tree (deterministic); the k-sum at the points is one
// thread per point over all wave vectors.  O(nsite x npoint), like the
// reference: this is an analysis call, not the per-step path.

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "mmnb_internal.cuh"

namespace mmnb {

constexpr int kEspThreads = 128;

struct EspArgs {
  int nsite, npoint;
  Box box;
  double rlo2, rhi2, inv_sw, eta;
  double cheb_min, cheb_max, cheb_inv_dx;
  const double *cheb;
  const double *r, *q, *rscreen;
  const int *mask;
  const double *pts;
  double *phi;
};

// b0 = erfc(eta r)/r: the table inside its range, the closed form outside
__device__ __forceinline__ double esp_b0(const EspArgs &a, double r2)
{
  if (a.cheb_min < r2 && r2 < a.cheb_max) {
    double x = (r2 - a.cheb_min) * a.cheb_inv_dx;
    const unsigned i = (unsigned) x;
    const double2 *c = reinterpret_cast<const double2 *>(a.cheb + 8 * (size_t) i);
    const double2 c01 = __ldg(c), c23 = __ldg(c + 1);
    x -= i;
    return ((c23.y * x + c23.x) * x + c01.y) * x + c01.x;
  }
  const double rm = sqrt(r2);
  return erfc(a.eta * rm) / rm;
}

__global__ void __launch_bounds__(kEspThreads) k_esp_rspace(EspArgs a)
{
  __shared__ double4 srq[kEspThreads];   // x, y, z, q
  __shared__ double srs[kEspThreads];    // r_screen
  __shared__ int smask[kEspThreads];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = j < a.npoint;
  double gx = 0, gy = 0, gz = 0;
  if (live) {
    gx = a.pts[3 * j];
    gy = a.pts[3 * j + 1];
    gz = a.pts[3 * j + 2];
  }
  double p = 0;
  for (int t0 = 0; t0 < a.nsite; t0 += kEspThreads) {
    const int i = t0 + threadIdx.x;
    __syncthreads();
    if (i < a.nsite) {
      srq[threadIdx.x] = make_double4(a.r[3 * i], a.r[3 * i + 1], a.r[3 * i + 2], a.q[i]);
      srs[threadIdx.x] = a.rscreen[i];
      smask[threadIdx.x] = a.mask[i];
    }
    __syncthreads();
    const int n = min(kEspThreads, a.nsite - t0);
    if (!live)
      continue;
    for (int k = 0; k < n; k++) {
      if (!smask[k])
        continue;
      const double4 s = srq[k];
      // site minus point, then the displacement to the central box
      double x = __dsub_rn(s.x, gx), y = __dsub_rn(s.y, gy), z = __dsub_rn(s.z, gz);
      x = __dadd_rn(x, __dmul_rn(-a.box.L[0], floor(__dadd_rn(__dmul_rn(x, a.box.invL[0]), 0.5))));
      y = __dadd_rn(y, __dmul_rn(-a.box.L[1], floor(__dadd_rn(__dmul_rn(y, a.box.invL[1]), 0.5))));
      z = __dadd_rn(z, __dmul_rn(-a.box.L[2], floor(__dadd_rn(__dmul_rn(z, a.box.invL[2]), 0.5))));
      const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
      if (r2 > a.rhi2)
        continue;
      double b0 = esp_b0(a, r2);
      const double rs = srs[k];
      if (r2 < rs * rs) {
        const double invr = 1.0 / sqrt(r2);
        b0 += (-0.5 * r2 * (1.0 / (rs * rs * rs)) + 1.5 / rs) - invr;
      }
      if (r2 > a.rlo2) {
        const double zz = (r2 - a.rlo2) * a.inv_sw;
        b0 *= ((-6 * zz + 15) * zz - 10) * zz * zz * zz + 1;
      }
      p += s.w * b0;
    }
  }
  if (live)
    a.phi[j] = p;
}

// S(k) = sum_i q_i (cos k.r_i, sin k.r_i), one block per wave vector
__global__ void __launch_bounds__(256) k_esp_structure(int nsite, int nk, const double *__restrict__ r,
                                                       const double *__restrict__ q, const double *__restrict__ kvec,
                                                       double *__restrict__ skc)
{
  __shared__ double sc[256], ss[256];
  const int k = blockIdx.x;
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

// phi_j += sum_k 2 a_k (S_c cos k.r_j + S_s sin k.r_j)
__global__ void __launch_bounds__(kEspThreads) k_esp_kspace(int npoint, int nk, const double *__restrict__ pts,
                                                            const double *__restrict__ kvec,
                                                            const double *__restrict__ ak,
                                                            const double *__restrict__ skc, double neutral,
                                                            double *__restrict__ phi)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= npoint)
    return;
  const double x = pts[3 * j], y = pts[3 * j + 1], z = pts[3 * j + 2];
  double p = 0;
  for (int k = 0; k < nk; k++) {
    double sn, cs;
    sincos(__ldg(kvec + 3 * k) * x + __ldg(kvec + 3 * k + 1) * y + __ldg(kvec + 3 * k + 2) * z, &sn, &cs);
    p += 2 * __ldg(ak + k) * (__ldg(skc + 2 * k + 1) * sn + __ldg(skc + 2 * k) * cs);
  }
  phi[j] = (phi[j] + p) + neutral;
}

}  // namespace mmnb

using namespace mmnb;

static int esp_fail(mmnb_handle *h, int code, const std::string &msg)
{
  if (h)
    h->err = msg;
  return code;
}

extern "C" int mmnb_phi_at_points(mmnb_handle *h, const double *r, int npoint, const double *points, double *phi)
{
  if (!h || !r || (npoint > 0 && (!points || !phi)) || npoint < 0)
    return esp_fail(h, MMNB_ERR_ARG, "null handle, positions, points or output, or a negative point count");
  if (npoint > (1 << 30) / 3)
    return esp_fail(h, MMNB_ERR_ARG, "at most 357,913,941 points per call (32-bit point indices)");
  if (!h->params_set)
    return esp_fail(h, MMNB_ERR_STATE, "mmnb_set_params has not been called");
  if (npoint == 0)
    return MMNB_OK;
  const mmnb_config &c = h->cfg;
  // wave vectors of kspace_new(kspace_cutoff, .) (src/kspace.c:35-71): the
  // half space of integer n with |n|^2 <= kc^2, k = 2 pi n / L
  std::vector<double> kv, ak;
  if (c.include_kspace) {
    const double kc = c.kspace_cutoff, n2max = kc * kc + 1e-8;
    const int nmax = (int) floor(kc);
    const double cc = 0.25 / (h->eta * h->eta), f = 4 * M_PI / h->volume;
    for (int nx = 0; nx <= nmax; nx++)
      for (int ny = (nx == 0 ? 0 : -nmax); ny <= nmax; ny++)
        for (int nz = (nx == 0 && ny == 0 ? 1 : -nmax); nz <= nmax; nz++) {
          if (nx * nx + ny * ny + nz * nz > n2max)
            continue;
          const double k[3] = {2 * M_PI * (1.0 / h->box.L[0]) * nx, 2 * M_PI * (1.0 / h->box.L[1]) * ny,
                               2 * M_PI * (1.0 / h->box.L[2]) * nz};
          const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
          kv.insert(kv.end(), k, k + 3);
          ak.push_back(f * exp(-k2 * cc) / k2);
        }
  }
  const int nk = (int) ak.size();
  const size_t n3 = 3 * (size_t) h->nsite, m3 = 3 * (size_t) npoint;
  const size_t total = n3 + m3 + (size_t) npoint + 3 * (size_t) nk + nk + 2 * (size_t) nk;
  double *buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, total * sizeof(double));
  if (e != cudaSuccess)
    return esp_fail(h, MMNB_ERR_CUDA, std::string("potential at points: ") + cudaGetErrorString(e));
  double *d_r = buf, *d_pts = d_r + n3, *d_phi = d_pts + m3, *d_kv = d_phi + npoint, *d_ak = d_kv + 3 * nk,
         *d_skc = d_ak + nk;
  e = cudaMemcpyAsync(d_r, r, n3 * sizeof(double), cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_pts, points, m3 * sizeof(double), cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess && nk > 0) {
    e = cudaMemcpyAsync(d_kv, kv.data(), kv.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_ak, ak.data(), ak.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream);
  }
  if (e == cudaSuccess)
    e = cudaMemsetAsync(d_phi, 0, npoint * sizeof(double), h->stream);
  if (e == cudaSuccess && c.include_rspace) {
    EspArgs a;
    a.nsite = h->nsite;
    a.npoint = npoint;
    a.box = h->box;
    a.rlo2 = h->rlo2;
    a.rhi2 = h->rhi2;
    a.inv_sw = h->inv_sw;
    a.eta = h->eta;
    a.cheb_min = h->cheb_min;
    a.cheb_max = h->cheb_max;
    a.cheb_inv_dx = h->cheb_inv_dx;
    a.cheb = h->d_cheb;
    a.r = d_r;
    a.q = h->d_q;
    a.rscreen = h->d_rscreen;
    a.mask = h->d_mask;
    a.pts = d_pts;
    a.phi = d_phi;
    k_esp_rspace<<<div_up(npoint, kEspThreads), kEspThreads, 0, h->stream>>>(a);
    e = cudaGetLastError();
    h->launches += 1;
  }
  const double neutral = c.include_self ? h->neutral_b : 0.0;
  if (e == cudaSuccess && (nk > 0 || neutral != 0)) {
    if (nk > 0) {
      k_esp_structure<<<nk, 256, 0, h->stream>>>(h->nsite, nk, d_r, h->d_q, d_kv, d_skc);
      e = cudaGetLastError();
      h->launches += 1;
    }
    if (e == cudaSuccess) {
      k_esp_kspace<<<div_up(npoint, kEspThreads), kEspThreads, 0, h->stream>>>(npoint, nk, d_pts, d_kv, d_ak,
                                                                                d_skc, neutral, d_phi);
      e = cudaGetLastError();
      h->launches += 1;
    }
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(phi, d_phi, npoint * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(h->stream);
  cudaFree(buf);
  if (e != cudaSuccess)
    return esp_fail(h, MMNB_ERR_CUDA, std::string("potential at points: ") + cudaGetErrorString(e));
  return MMNB_OK;
}

// P3M reciprocal space on the GPU (replaces p3m_init / p3m_field,
// src/pppm.c:313-393, 498-641).
//
// Steps per evaluation: B-spline charge assignment onto the mesh, cuFFT
// real-to-complex, multiplication by the optimal influence function,
// complex-to-real, interpolation of potential and field back to the sites.
// Differentiation is in real space (gradient of the assignment function,
// the reference default) or, with p3m_ik_differentiate, by -ik on the mesh
// with three extra inverse transforms.
//
// Charge-assignment weights come from the Cox-de Boor recursion for cardinal
// B-splines, which reproduces the reference's per-order polynomials
// (src/pppm.c:69-275) for every order 2..7.  The influence function is the
// Hockney-Eastwood optimum with an alias sum over |p| <= nalias, evaluated
// once per box on the GPU in FP64.

#include "mmnb_internal.cuh"

namespace mmnb {

struct MeshArgs {
  int n[3];
  double A[9];      // mesh-scaled inverse lattice, tensor_t layout: s = A r
  int nsite;
};

// Nearest mesh point and offset of a particle at mesh coordinate s
// (src/pppm.c:533-548): returns the first of the P assigned points and
// w = delta + 1/2 in [0, 1].
template <int P>
__device__ __forceinline__ int bspline_base(double s, double &w)
{
  int j;
  double delta;
  if (P % 2) {
    j = (int) floor(s + 0.5);
    delta = s - j;
  } else {
    j = (int) floor(s);
    delta = s - (j + 0.5);
  }
  w = delta + 0.5;
  return j - ((P + 1) / 2 - 1);
}

// Weights W[p] and negated derivatives ND[p] of the points base + p.
template <int P, typename T>
__device__ __forceinline__ void bspline_eval(T w, T *W, T *ND)
{
  T m[P], prev[P];
  m[0] = T(1);
#pragma unroll
  for (int k = 2; k <= P; k++) {
    const T inv = T(1) / T(k - 1);
#pragma unroll
    for (int i = 0; i < k - 1; i++)
      prev[i] = m[i];
#pragma unroll
    for (int i = 0; i < k; i++) {
      const T a = i < k - 1 ? prev[i] : T(0);
      const T b = i > 0 ? prev[i - 1] : T(0);
      m[i] = ((w + T(i)) * a + (T(k) - w - T(i)) * b) * inv;
    }
  }
#pragma unroll
  for (int p = 0; p < P; p++) {
    const int i = P - 1 - p;
    W[p] = m[i];
    const T a = i < P - 1 ? prev[i] : T(0);
    const T b = i > 0 ? prev[i - 1] : T(0);
    ND[p] = b - a;
  }
}

template <int P>
__device__ __forceinline__ int bspline_weights(double s, double *W, double *ND)
{
  double w;
  const int base = bspline_base<P>(s, w);
  bspline_eval<P, double>(w, W, ND);
  return base;
}

__device__ __forceinline__ int wrap_idx(int i, int n)
{
  i %= n;
  return i < 0 ? i + n : i;
}

// ---- influence function -----------------------------------------------------

constexpr int kGreenThreads = 128;

struct GreenArgs {
  int n[3];
  int nalias, order, ik;
  double rec[9];     // 2 pi inv(latv)^T, tensor_t layout
  double inv_v, inv_4eta2;
  double *green, *kvec, *chi;
};

__device__ __forceinline__ double sincpi_d(double x)
{
  const double y = M_PI * x;
  return fabs(y) < 1e-16 ? 1 - y * y / 6 : sin(y) / y;
}

// G(k) of one half-mesh point g (and its k-vector); returns the point's term of
// the RMS force error sum, sum_p g_p^2 k_p^2 - numerator^2 / denominator
__device__ double green_point(const GreenArgs &a, long g, int nx, int ny, int nz, int nzh)
{
  const int iz = (int) (g % nzh);
  const int iy = (int) ((g / nzh) % ny);
  const int ix = (int) (g / ((long) nzh * ny));
  const double jx = ix > nx / 2 ? ix - nx : ix;
  const double jy = iy > ny / 2 ? iy - ny : iy;
  const double jz = iz;
  const double *R = a.rec;
  double kv[3];
  kv[0] = R[0] * jx + R[3] * jy + R[6] * jz;
  kv[1] = R[1] * jx + R[4] * jy + R[7] * jz;
  kv[2] = R[2] * jx + R[5] * jy + R[8] * jz;
  if (a.kvec) {
    a.kvec[3 * g] = kv[0];
    a.kvec[3 * g + 1] = kv[1];
    a.kvec[3 * g + 2] = kv[2];
  }
  if (ix == 0 && iy == 0 && iz == 0) {
    a.green[g] = 0;
    return 0.0;
  }
  const double k2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
  constexpr int kMaxAlias = 8;
  double ux[2 * kMaxAlias + 1], uy[2 * kMaxAlias + 1], uz[2 * kMaxAlias + 1];
  const int na = a.nalias;
  for (int q = -na; q <= na; q++) {
    ux[q + na] = pow(sincpi_d(jx / nx + q), 2 * a.order);
    uy[q + na] = pow(sincpi_d(jy / ny + q), 2 * a.order);
    uz[q + na] = pow(sincpi_d(jz / nz + q), 2 * a.order);
  }
  double num = 0, d1 = 0, d2 = 0, chi = 0;
  for (int px = -na; px <= na; px++) {
    const double mx = jx + px * nx;
    for (int py = -na; py <= na; py++) {
      const double my = jy + py * ny;
      for (int pz = -na; pz <= na; pz++) {
        const double mz = jz + pz * nz;
        if (fabs(mx) < 1e-16 && fabs(my) < 1e-16 && fabs(mz) < 1e-16)
          continue;
        const double kpx = R[0] * mx + R[3] * my + R[6] * mz;
        const double kpy = R[1] * mx + R[4] * my + R[7] * mz;
        const double kpz = R[2] * mx + R[5] * my + R[8] * mz;
        const double kp2 = kpx * kpx + kpy * kpy + kpz * kpz;
        const double u2 = ux[px + na] * uy[py + na] * uz[pz + na];
        const double gg = 4 * M_PI / kp2 * exp(-kp2 * a.inv_4eta2);
        if (a.ik) {
          num += gg * u2 * (kv[0] * kpx + kv[1] * kpy + kv[2] * kpz);
          d1 += u2;
        } else {
          num += gg * kp2 * u2;
          d1 += u2;
          d2 += u2 * kp2;
        }
        chi += gg * gg * kp2;
      }
    }
  }
  const double den = a.ik ? d1 * d1 * k2 : d1 * d2;
  a.green[g] = a.inv_v * num / den;
  chi -= num * num / den;
  return chi;
}

__global__ void k_green(GreenArgs a)
{
  const int nx = a.n[0], ny = a.n[1], nz = a.n[2], nzh = nz / 2 + 1;
  const long g = (long) blockIdx.x * blockDim.x + threadIdx.x;
  const double chi = g < (long) nx * ny * nzh ? green_point(a, g, nx, ny, nz, nzh) : 0.0;
  if (!a.chi)
    return;
  // chi of this block's points, summed in a fixed order (one partial per block)
  __shared__ double part[kGreenThreads / 32];
  double v = chi;
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0)
    part[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < kGreenThreads / 32; w++)
      t += part[w];
    a.chi[blockIdx.x] = t;
  }
}

// G(k) and the k-vectors of the handle's mesh at screening eta (p3m_init,
// src/pppm.c:313-393); with chi non-null also the reference's dimensionless RMS
// force error estimate V^(-1/3) sqrt(2 |sum|), its per-block partials added in
// block order on the host so that the value does not depend on scheduling
cudaError_t launch_p3m_green(mmnb_handle *h, double eta, double *chi)
{
  GreenArgs a;
  for (int d = 0; d < 3; d++)
    a.n[d] = h->mesh[d];
  a.nalias = h->cfg.p3m_alias_sum_limit;
  a.order = h->cfg.p3m_assignment_order;
  a.ik = h->cfg.p3m_ik_differentiate;
  // 2 pi inv(latv)^T for the (diagonal) lattice
  for (int i = 0; i < 9; i++)
    a.rec[i] = 0;
  for (int d = 0; d < 3; d++)
    a.rec[4 * d] = 2 * M_PI * (1.0 / h->box.L[d]);
  a.inv_v = 1.0 / h->volume;
  a.inv_4eta2 = 1 / ((2 * eta) * (2 * eta));
  a.green = h->d_green;
  a.kvec = h->d_kvec;
  a.chi = chi ? h->d_chi_part : nullptr;
  const long nk = (long) h->mesh[0] * h->mesh[1] * (h->mesh[2] / 2 + 1);
  const int nblock = (int) div_up(nk, kGreenThreads);
  k_green<<<nblock, kGreenThreads, 0, h->stream>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !chi)
    return e;
  std::vector<double> part(nblock);
  e = cudaMemcpyAsync(part.data(), h->d_chi_part, sizeof(double) * nblock, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess)
    return e;
  double sum = 0;
  for (int b = 0; b < nblock; b++)
    sum += part[b];
  *chi = pow(a.inv_v, 1.0 / 3.0) * sqrt(2 * fabs(sum));
  return cudaSuccess;
}

// ---- FP64 spread / gather -----------------------------------------------------

template <int P>
__global__ void k_spread_fp64(MeshArgs m, const double *__restrict__ r, const double *__restrict__ q,
                              const int *__restrict__ mask, double *__restrict__ mesh)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nsite)
    return;
  const double qi = q[i];
  if (!(mask[i] & MMNB_SITE_HAS_Q) || qi == 0)
    return;
  const double x = r[3 * i], y = r[3 * i + 1], z = r[3 * i + 2];
  double W[3][P], ND[3][P];
  int base[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double s = m.A[d] * x + m.A[3 + d] * y + m.A[6 + d] * z;
    base[d] = bspline_weights<P>(s, W[d], ND[d]);
  }
  int iy_[P], iz_[P];
#pragma unroll
  for (int p = 0; p < P; p++) {
    iy_[p] = wrap_idx(base[1] + p, m.n[1]);
    iz_[p] = wrap_idx(base[2] + p, m.n[2]);
  }
  for (int a = 0; a < P; a++) {
    const int ix = wrap_idx(base[0] + a, m.n[0]);
#pragma unroll
    for (int b = 0; b < P; b++) {
      const double qw = W[0][a] * W[1][b] * qi;
      double *row = mesh + ((size_t) ix * m.n[1] + iy_[b]) * m.n[2];
#pragma unroll
      for (int c = 0; c < P; c++)
        atomicAdd(row + iz_[c], qw * W[2][c]);
    }
  }
}

__global__ void k_green_mul(long nk, const double *__restrict__ green, cufftDoubleComplex *__restrict__ meshk,
                            const double *__restrict__ kvec, cufftDoubleComplex *__restrict__ egk)
{
  const long g = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nk)
    return;
  const double a = green[g];
  cufftDoubleComplex v = meshk[g];
  v.x *= a;
  v.y *= a;
  meshk[g] = v;
  if (egk) {
    // -ik times the potential: (k im, -k re) per component (src/pppm.c:583-594)
    for (int d = 0; d < 3; d++) {
      const double k = kvec[3 * g + d];
      egk[d * nk + g] = make_cuDoubleComplex(k * v.y, -k * v.x);
    }
  }
}

template <int P>
__global__ void k_gather_fp64(MeshArgs m, const double *__restrict__ r, const double *__restrict__ mesh,
                              const double *__restrict__ egrid, size_t nr, double *__restrict__ phi,
                              double *__restrict__ evec)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nsite)
    return;
  const double x = r[3 * i], y = r[3 * i + 1], z = r[3 * i + 2];
  double W[3][P], ND[3][P];
  int base[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double s = m.A[d] * x + m.A[3 + d] * y + m.A[6 + d] * z;
    base[d] = bspline_weights<P>(s, W[d], ND[d]);
  }
  int iy_[P], iz_[P];
#pragma unroll
  for (int p = 0; p < P; p++) {
    iy_[p] = wrap_idx(base[1] + p, m.n[1]);
    iz_[p] = wrap_idx(base[2] + p, m.n[2]);
  }
  double ph = 0, gx = 0, gy = 0, gz = 0;
  for (int a = 0; a < P; a++) {
    const int ix = wrap_idx(base[0] + a, m.n[0]);
#pragma unroll
    for (int b = 0; b < P; b++) {
      const size_t rowoff = ((size_t) ix * m.n[1] + iy_[b]) * m.n[2];
      const double wxy = W[0][a] * W[1][b];
#pragma unroll
      for (int c = 0; c < P; c++) {
        const size_t k = rowoff + iz_[c];
        const double pv = __ldg(mesh + k);
        ph += wxy * W[2][c] * pv;
        if (egrid) {
          const double ww = wxy * W[2][c];
          gx += ww * __ldg(egrid + k);
          gy += ww * __ldg(egrid + nr + k);
          gz += ww * __ldg(egrid + 2 * nr + k);
        } else {
          gx += ND[0][a] * W[1][b] * W[2][c] * pv;
          gy += W[0][a] * ND[1][b] * W[2][c] * pv;
          gz += wxy * ND[2][c] * pv;
        }
      }
    }
  }
  phi[i] += ph;
  if (egrid) {
    evec[3 * i] += gx;
    evec[3 * i + 1] += gy;
    evec[3 * i + 2] += gz;
  } else {
    // E = A^T (-grad_s phi)  (left_operate, include/cart.h:28-36)
    evec[3 * i] += gx * m.A[0] + gy * m.A[1] + gz * m.A[2];
    evec[3 * i + 1] += gx * m.A[3] + gy * m.A[4] + gz * m.A[5];
    evec[3 * i + 2] += gx * m.A[6] + gy * m.A[7] + gz * m.A[8];
  }
}

static MeshArgs mesh_args(mmnb_handle *h)
{
  MeshArgs m;
  for (int d = 0; d < 3; d++)
    m.n[d] = h->mesh[d];
  for (int i = 0; i < 9; i++)
    m.A[i] = 0;
  // inverse of the diagonal lattice as the reference's inverse() computes it,
  // rows scaled by the mesh size (src/pppm.c:428, 523-525)
  const double xx = h->box.L[0], yy = h->box.L[1], zz = h->box.L[2];
  const double det = xx * yy * zz;
  const double id = 1.0 / det;
  m.A[0] = id * (yy * zz) * h->mesh[0];
  m.A[4] = id * (xx * zz) * h->mesh[1];
  m.A[8] = id * (xx * yy) * h->mesh[2];
  m.nsite = h->nsite;
  return m;
}

// stage bit 1: charge assignment and the FFT round trip; bit 2: interpolation
template <int P>
static cudaError_t p3m_fp64_p(mmnb_handle *h, const double *d_r, int stage)
{
  const MeshArgs m = mesh_args(h);
  const size_t nr = (size_t) h->mesh[0] * h->mesh[1] * h->mesh[2];
  const long nk = (long) h->mesh[0] * h->mesh[1] * (h->mesh[2] / 2 + 1);
  const bool ik = h->cfg.p3m_ik_differentiate != 0;
  if (stage & 1) {
    cudaError_t e = cudaMemsetAsync(h->d_mesh, 0, sizeof(double) * nr, h->stream);
    if (e != cudaSuccess)
      return e;
    k_spread_fp64<P><<<div_up(h->nsite, 128), 128, 0, h->stream>>>(m, d_r, h->d_q, h->d_mask, h->d_mesh);
    timing_mark(h, "p3m_spread");
    if (cufftSetStream(h->plan_r2c, h->stream) != CUFFT_SUCCESS ||
        cufftSetStream(h->plan_c2r, h->stream) != CUFFT_SUCCESS ||
        cufftExecD2Z(h->plan_r2c, h->d_mesh, h->d_meshk) != CUFFT_SUCCESS)
      return cudaErrorUnknown;
    k_green_mul<<<div_up(nk, 256), 256, 0, h->stream>>>(nk, h->d_green, h->d_meshk, h->d_kvec,
                                                        ik ? h->d_egridk : nullptr);
    if (ik)
      for (int d = 0; d < 3; d++)
        if (cufftExecZ2D(h->plan_c2r, h->d_egridk + d * nk, h->d_egrid + d * nr) != CUFFT_SUCCESS)
          return cudaErrorUnknown;
    if (cufftExecZ2D(h->plan_c2r, h->d_meshk, h->d_mesh) != CUFFT_SUCCESS)
      return cudaErrorUnknown;
    timing_mark(h, "p3m_fft");
    h->launches += 2;
  }
  if (stage & 2) {
    k_gather_fp64<P><<<div_up(h->nsite, 128), 128, 0, h->stream>>>(m, d_r, h->d_mesh, ik ? h->d_egrid : nullptr,
                                                                   nr, h->d_phi, h->d_evec);
    timing_mark(h, "p3m_gather");
    h->launches += 1;
  }
  return cudaGetLastError();
}

cudaError_t launch_p3m_fp64(mmnb_handle *h, const double *d_r, int stage)
{
  switch (h->cfg.p3m_assignment_order) {
  case 2: return p3m_fp64_p<2>(h, d_r, stage);
  case 3: return p3m_fp64_p<3>(h, d_r, stage);
  case 4: return p3m_fp64_p<4>(h, d_r, stage);
  case 5: return p3m_fp64_p<5>(h, d_r, stage);
  case 6: return p3m_fp64_p<6>(h, d_r, stage);
  case 7: return p3m_fp64_p<7>(h, d_r, stage);
  default: return cudaErrorInvalidValue;
  }
}

// ---- adjoint: the mesh potential of a dipole density ------------------------
//
// For a loss L of the forces, dL/dq_i holds, besides g_i . E_i (g = dL/dF),
// sum_j q_j g_j . dE_j/dq_i: the potential at r_i of point dipoles
// p_j = q_j g_j, as the mesh sees them.  The map "charges -> mesh field at the
// sites" is spread, solve, gather; its transpose runs the three steps
// backwards with each one transposed:
//   * real-space differentiation: E_j gathers the mesh potential with the
//     vector weights A^T (-grad_s W)(r_j), and the solve (real, even influence
//     function) is symmetric, so the dipoles are spread with those vector
//     weights, solved with the same influence function and gathered with the
//     plain weights W;
//   * ik differentiation: E_j,d gathers C2R(-i k_d G rho^) with W; that
//     operator is real and odd, its transpose C2R(+i k_d G .), so the three
//     dipole components are spread with W and the solve sums
//     i k_d G D^_d over d into one mesh.

template <int P>
__global__ void k_spread_dipole_fp64(MeshArgs m, const double *__restrict__ r, const double *__restrict__ q,
                                     const int *__restrict__ mask, const double *__restrict__ g, int ik, size_t nr,
                                     double *__restrict__ mesh)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nsite)
    return;
  const double qi = q[i];
  if (!(mask[i] & MMNB_SITE_HAS_Q) || qi == 0)
    return;
  const double px = qi * g[3 * i], py = qi * g[3 * i + 1], pz = qi * g[3 * i + 2];
  const double x = r[3 * i], y = r[3 * i + 1], z = r[3 * i + 2];
  double W[3][P], ND[3][P];
  int base[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double s = m.A[d] * x + m.A[3 + d] * y + m.A[6 + d] * z;
    base[d] = bspline_weights<P>(s, W[d], ND[d]);
  }
  int iy_[P], iz_[P];
#pragma unroll
  for (int p = 0; p < P; p++) {
    iy_[p] = wrap_idx(base[1] + p, m.n[1]);
    iz_[p] = wrap_idx(base[2] + p, m.n[2]);
  }
  // p . A^T v = (A p) . v for the vector weight v of the gather
  const double c0 = m.A[0] * px + m.A[3] * py + m.A[6] * pz;
  const double c1 = m.A[1] * px + m.A[4] * py + m.A[7] * pz;
  const double c2 = m.A[2] * px + m.A[5] * py + m.A[8] * pz;
  for (int a = 0; a < P; a++) {
    const int ix = wrap_idx(base[0] + a, m.n[0]);
#pragma unroll
    for (int b = 0; b < P; b++) {
      const size_t rowoff = ((size_t) ix * m.n[1] + iy_[b]) * m.n[2];
#pragma unroll
      for (int c = 0; c < P; c++) {
        const size_t k = rowoff + iz_[c];
        if (ik) {
          const double w = W[0][a] * W[1][b] * W[2][c];
          atomicAdd(mesh + k, px * w);
          atomicAdd(mesh + nr + k, py * w);
          atomicAdd(mesh + 2 * nr + k, pz * w);
        } else {
          atomicAdd(mesh + k, c0 * ND[0][a] * W[1][b] * W[2][c] + c1 * W[0][a] * ND[1][b] * W[2][c] +
                                  c2 * W[0][a] * W[1][b] * ND[2][c]);
        }
      }
    }
  }
}

// ik: out = G sum_d i k_d D^_d
__global__ void k_dipole_green_ik(long nk, const double *__restrict__ green, const double *__restrict__ kvec,
                                  const cufftDoubleComplex *__restrict__ dk, cufftDoubleComplex *__restrict__ out)
{
  const long g = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nk)
    return;
  double re = 0, im = 0;
  for (int d = 0; d < 3; d++) {
    const double k = kvec[3 * g + d];
    const cufftDoubleComplex v = dk[d * nk + g];
    re -= k * v.y;
    im += k * v.x;
  }
  const double a = green[g];
  out[g] = make_cuDoubleComplex(a * re, a * im);
}

template <int P>
__global__ void k_gather_potential_fp64(MeshArgs m, const double *__restrict__ r, const double *__restrict__ mesh,
                                        double *__restrict__ out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.nsite)
    return;
  const double x = r[3 * i], y = r[3 * i + 1], z = r[3 * i + 2];
  double W[3][P], ND[3][P];
  int base[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double s = m.A[d] * x + m.A[3 + d] * y + m.A[6 + d] * z;
    base[d] = bspline_weights<P>(s, W[d], ND[d]);
  }
  int iy_[P], iz_[P];
#pragma unroll
  for (int p = 0; p < P; p++) {
    iy_[p] = wrap_idx(base[1] + p, m.n[1]);
    iz_[p] = wrap_idx(base[2] + p, m.n[2]);
  }
  double ph = 0;
  for (int a = 0; a < P; a++) {
    const int ix = wrap_idx(base[0] + a, m.n[0]);
#pragma unroll
    for (int b = 0; b < P; b++) {
      const size_t rowoff = ((size_t) ix * m.n[1] + iy_[b]) * m.n[2];
      const double wxy = W[0][a] * W[1][b];
#pragma unroll
      for (int c = 0; c < P; c++)
        ph += wxy * W[2][c] * __ldg(mesh + rowoff + iz_[c]);
    }
  }
  out[i] += ph;
}

template <int P>
static cudaError_t p3m_dipole_p(mmnb_handle *h, const double *d_r, const double *d_g, const P3mScratch &s,
                                double *d_psi)
{
  const MeshArgs m = mesh_args(h);
  const size_t nr = (size_t) h->mesh[0] * h->mesh[1] * h->mesh[2];
  const long nk = (long) h->mesh[0] * h->mesh[1] * (h->mesh[2] / 2 + 1);
  const int ik = h->cfg.p3m_ik_differentiate ? 1 : 0;
  const int nmesh = ik ? 3 : 1;
  cudaError_t e = cudaMemsetAsync(s.spread, 0, sizeof(double) * nr * nmesh, h->stream);
  if (e != cudaSuccess)
    return e;
  k_spread_dipole_fp64<P><<<div_up(h->nsite, 128), 128, 0, h->stream>>>(m, d_r, h->d_q, h->d_mask, d_g, ik, nr,
                                                                         s.spread);
  if (cufftSetStream(s.r2c, h->stream) != CUFFT_SUCCESS || cufftSetStream(s.c2r, h->stream) != CUFFT_SUCCESS)
    return cudaErrorUnknown;
  for (int d = 0; d < nmesh; d++)
    if (cufftExecD2Z(s.r2c, s.spread + d * nr, s.spreadk + d * nk) != CUFFT_SUCCESS)
      return cudaErrorUnknown;
  if (ik)
    k_dipole_green_ik<<<div_up(nk, 256), 256, 0, h->stream>>>(nk, h->d_green, h->d_kvec, s.spreadk, s.solvek);
  else
    k_green_mul<<<div_up(nk, 256), 256, 0, h->stream>>>(nk, h->d_green, s.spreadk, h->d_kvec, nullptr);
  if (cufftExecZ2D(s.c2r, ik ? s.solvek : s.spreadk, s.solve) != CUFFT_SUCCESS)
    return cudaErrorUnknown;
  k_gather_potential_fp64<P><<<div_up(h->nsite, 128), 128, 0, h->stream>>>(m, d_r, s.solve, d_psi);
  h->launches += 3;
  return cudaGetLastError();
}

cudaError_t launch_p3m_dipole_fp64(mmnb_handle *h, const double *d_r, const double *d_g, const P3mScratch &s,
                                   double *d_psi)
{
  switch (h->cfg.p3m_assignment_order) {
  case 2: return p3m_dipole_p<2>(h, d_r, d_g, s, d_psi);
  case 3: return p3m_dipole_p<3>(h, d_r, d_g, s, d_psi);
  case 4: return p3m_dipole_p<4>(h, d_r, d_g, s, d_psi);
  case 5: return p3m_dipole_p<5>(h, d_r, d_g, s, d_psi);
  case 6: return p3m_dipole_p<6>(h, d_r, d_g, s, d_psi);
  case 7: return p3m_dipole_p<7>(h, d_r, d_g, s, d_psi);
  default: return cudaErrorInvalidValue;
  }
}

// ---- mixed form: FP32 weights, 64-bit fixed-point mesh, FP32 FFT -------------
//
// Charge assignment accumulates q w_x w_y w_z in 64-bit fixed point
// (2^32 units per unit charge), so the mesh, and everything computed from it,
// is bitwise independent of the order in which sites are spread.

// One thread per site in the caller's order: the position, charge and mask
// loads are independent and coalesced (no sorted-order indirection in front
// of them); the fixed-point adds do not depend on the order anyway.
template <int P>
__global__ void k_spread_mixed(MeshArgs m, const double *__restrict__ r, const double *__restrict__ q,
                               const int *__restrict__ mask, int nsite, unsigned long long *__restrict__ mesh)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsite || !(mask[i] & MMNB_SITE_HAS_Q))
    return;
  const float qi = (float) q[i];
  const double x = r[3 * i], y = r[3 * i + 1], z = r[3 * i + 2];
  float W[3][P], ND[3][P];
  int base[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double w;
    base[d] = bspline_base<P>(m.A[d] * x + m.A[3 + d] * y + m.A[6 + d] * z, w);
    bspline_eval<P, float>((float) w, W[d], ND[d]);
  }
  int iy_[P], iz_[P];
#pragma unroll
  for (int p = 0; p < P; p++) {
    iy_[p] = wrap_idx(base[1] + p, m.n[1]);
    iz_[p] = wrap_idx(base[2] + p, m.n[2]);
  }
  for (int a = 0; a < P; a++) {
    const int ix = wrap_idx(base[0] + a, m.n[0]);
#pragma unroll
    for (int b = 0; b < P; b++) {
      const float qw = W[0][a] * W[1][b] * qi;
      unsigned long long *row = mesh + ((size_t) ix * m.n[1] + iy_[b]) * m.n[2];
#pragma unroll
      for (int c = 0; c < P; c++)
        atomicAdd(row + iz_[c], (unsigned long long) __float2ll_rn(qw * W[2][c] * 4294967296.0f));
    }
  }
}

// The same charge assignment with P threads per site, thread a adding the
// site's plane x = base + a (P^2 adds): P times the parallelism for small
// systems whose one-thread-per-site grid leaves SMs idle.  Same fixed-point
// values, so the same mesh.
template <int P>
__global__ void k_spread_mixed_planes(MeshArgs m, const double *__restrict__ r, const double *__restrict__ q,
                                      const int *__restrict__ mask, int nsite, unsigned long long *__restrict__ mesh)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t / P, a = t % P;
  if (i >= nsite || !(mask[i] & MMNB_SITE_HAS_Q))
    return;
  const float qi = (float) q[i];
  const double x = r[3 * i], y = r[3 * i + 1], z = r[3 * i + 2];
  float W[3][P], ND[3][P];
  int base[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double w;
    base[d] = bspline_base<P>(m.A[d] * x + m.A[3 + d] * y + m.A[6 + d] * z, w);
    bspline_eval<P, float>((float) w, W[d], ND[d]);
  }
  float wa = 0.f;
#pragma unroll
  for (int p = 0; p < P; p++)
    if (p == a)
      wa = W[0][p];
  int iz_[P];
#pragma unroll
  for (int p = 0; p < P; p++)
    iz_[p] = wrap_idx(base[2] + p, m.n[2]);
  const int ix = wrap_idx(base[0] + a, m.n[0]);
#pragma unroll
  for (int b = 0; b < P; b++) {
    const float qw = wa * W[1][b] * qi;
    unsigned long long *row = mesh + ((size_t) ix * m.n[1] + wrap_idx(base[1] + b, m.n[1])) * m.n[2];
#pragma unroll
    for (int c = 0; c < P; c++)
      atomicAdd(row + iz_[c], (unsigned long long) __float2ll_rn(qw * W[2][c] * 4294967296.0f));
  }
}

// The same charge assignment with P lanes per site along z: lane c of a site
// adds the points z = base + c of its P^2 rows, so one instruction's
// reductions from a site go to P consecutive mesh words (two 32-byte
// sectors), where a thread per site sends each of its lanes' reductions to a
// different sector.  The L2 handles a warp's reductions per sector: about
// 2.5x fewer sector operations.  32 / P sites per warp; the last 32 mod P
// lanes idle.  Same fixed-point values, so the same mesh.
template <int P>
__global__ void k_spread_mixed_zlanes(MeshArgs m, const double *__restrict__ r, const double *__restrict__ q,
                                      const int *__restrict__ mask, int nsite, unsigned long long *__restrict__ mesh)
{
  constexpr int S = 32 / P;  // sites per warp
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int i = warp * S + lane / P, c = lane % P;
  if (lane >= S * P || i >= nsite || !(mask[i] & MMNB_SITE_HAS_Q))
    return;
  const float qi = (float) q[i];
  const double x = r[3 * i], y = r[3 * i + 1], z = r[3 * i + 2];
  float W[3][P], ND[3][P];
  int base[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double w;
    base[d] = bspline_base<P>(m.A[d] * x + m.A[3 + d] * y + m.A[6 + d] * z, w);
    bspline_eval<P, float>((float) w, W[d], ND[d]);
  }
  float wc = 0.f;
#pragma unroll
  for (int p = 0; p < P; p++)
    if (p == c)
      wc = W[2][p];
  const int iz = wrap_idx(base[2] + c, m.n[2]);
  for (int a = 0; a < P; a++) {
    const int ix = wrap_idx(base[0] + a, m.n[0]);
#pragma unroll
    for (int b = 0; b < P; b++) {
      const float qw = W[0][a] * W[1][b] * qi;
      unsigned long long *row = mesh + ((size_t) ix * m.n[1] + wrap_idx(base[1] + b, m.n[1])) * m.n[2];
      atomicAdd(row + iz, (unsigned long long) __float2ll_rn(qw * wc * 4294967296.0f));
    }
  }
}

// fixed-point mesh -> FP32 FFT input; clears the fixed-point mesh for the next step
__global__ void k_mesh_fx_to_f32(size_t n, unsigned long long *__restrict__ fx, float *__restrict__ out)
{
  const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  out[i] = (float) ((double) (long long) fx[i] * kFxInv);
  fx[i] = 0ull;
}

__global__ void k_green_mul32(long nk, const float *__restrict__ green, cufftComplex *__restrict__ meshk)
{
  const long g = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nk)
    return;
  const float a = green[g];
  cufftComplex v = meshk[g];
  v.x *= a;
  v.y *= a;
  meshk[g] = v;
}

// ik differentiation: the potential spectrum G rho^ in place and the three
// field spectra -i k_d G rho^ (the FP64 form's k_green_mul, in FP32)
__global__ void k_green_mul32_ik(long nk, const float *__restrict__ green, const double *__restrict__ kvec,
                                 cufftComplex *__restrict__ meshk, cufftComplex *__restrict__ egk)
{
  const long g = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nk)
    return;
  const float a = green[g];
  cufftComplex v = meshk[g];
  v.x *= a;
  v.y *= a;
  meshk[g] = v;
  for (int d = 0; d < 3; d++) {
    const float k = (float) kvec[3 * g + d];
    egk[d * nk + g] = make_cuComplex(k * v.y, -k * v.x);
  }
}

__global__ void k_green_to_f32(long nk, const double *__restrict__ green, float *__restrict__ out)
{
  const long g = (long) blockIdx.x * blockDim.x + threadIdx.x;
  if (g < nk)
    out[g] = (float) green[g];
}

// Interpolation writes its own fixed-point words (phi, Ex, Ey, Ez per site),
// which k_finalize adds to the pair kernels' sums: it touches nothing the
// pair kernels write, so it runs on the side stream beside them.
template <int P>
__global__ void k_gather_mixed(MeshArgs m, const double *__restrict__ r, int nsite, const float *__restrict__ mesh,
                               long long *__restrict__ acck)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsite)
    return;
  const double x = r[3 * i], y = r[3 * i + 1], z = r[3 * i + 2];
  float W[3][P], ND[3][P];
  int base[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double w;
    base[d] = bspline_base<P>(m.A[d] * x + m.A[3 + d] * y + m.A[6 + d] * z, w);
    bspline_eval<P, float>((float) w, W[d], ND[d]);
  }
  int iy_[P], iz_[P];
#pragma unroll
  for (int p = 0; p < P; p++) {
    iy_[p] = wrap_idx(base[1] + p, m.n[1]);
    iz_[p] = wrap_idx(base[2] + p, m.n[2]);
  }
  float ph = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
  for (int a = 0; a < P; a++) {
    const int ix = wrap_idx(base[0] + a, m.n[0]);
#pragma unroll
    for (int b = 0; b < P; b++) {
      const float *row = mesh + ((size_t) ix * m.n[1] + iy_[b]) * m.n[2];
      const float wxy = W[0][a] * W[1][b];
      const float dxy = ND[0][a] * W[1][b];
      const float xdy = W[0][a] * ND[1][b];
      float s0 = 0.f, s1 = 0.f;
#pragma unroll
      for (int c = 0; c < P; c++) {
        const float pv = __ldg(row + iz_[c]);
        s0 = fmaf(W[2][c], pv, s0);
        s1 = fmaf(ND[2][c], pv, s1);
      }
      ph = fmaf(wxy, s0, ph);
      gx = fmaf(dxy, s0, gx);
      gy = fmaf(xdy, s0, gy);
      gz = fmaf(wxy, s1, gz);
    }
  }
  const float A0 = (float) m.A[0], A4 = (float) m.A[4], A8 = (float) m.A[8];
  longlong4 o;
  o.x = __float2ll_rn(ph * 4294967296.0f);
  o.y = __float2ll_rn(gx * A0 * 4294967296.0f);
  o.z = __float2ll_rn(gy * A4 * 4294967296.0f);
  o.w = __float2ll_rn(gz * A8 * 4294967296.0f);
  reinterpret_cast<longlong4 *>(acck)[i] = o;
}

// ik differentiation: the potential and the three field components
// interpolated with the assignment weights (the field meshes are already the
// Cartesian field), into the same fixed-point words as k_gather_mixed
template <int P>
__global__ void k_gather_mixed_ik(MeshArgs m, const double *__restrict__ r, int nsite, const float *__restrict__ mesh,
                                  const float *__restrict__ egrid, size_t nr, long long *__restrict__ acck)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsite)
    return;
  const double x = r[3 * i], y = r[3 * i + 1], z = r[3 * i + 2];
  float W[3][P], ND[3][P];
  int base[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double w;
    base[d] = bspline_base<P>(m.A[d] * x + m.A[3 + d] * y + m.A[6 + d] * z, w);
    bspline_eval<P, float>((float) w, W[d], ND[d]);
  }
  int iy_[P], iz_[P];
#pragma unroll
  for (int p = 0; p < P; p++) {
    iy_[p] = wrap_idx(base[1] + p, m.n[1]);
    iz_[p] = wrap_idx(base[2] + p, m.n[2]);
  }
  float ph = 0.f, ex = 0.f, ey = 0.f, ez = 0.f;
  for (int a = 0; a < P; a++) {
    const int ix = wrap_idx(base[0] + a, m.n[0]);
#pragma unroll
    for (int b = 0; b < P; b++) {
      const size_t rowoff = ((size_t) ix * m.n[1] + iy_[b]) * m.n[2];
      const float wxy = W[0][a] * W[1][b];
#pragma unroll
      for (int c = 0; c < P; c++) {
        const size_t k = rowoff + iz_[c];
        const float ww = wxy * W[2][c];
        ph = fmaf(ww, __ldg(mesh + k), ph);
        ex = fmaf(ww, __ldg(egrid + k), ex);
        ey = fmaf(ww, __ldg(egrid + nr + k), ey);
        ez = fmaf(ww, __ldg(egrid + 2 * nr + k), ez);
      }
    }
  }
  longlong4 o;
  o.x = __float2ll_rn(ph * 4294967296.0f);
  o.y = __float2ll_rn(ex * 4294967296.0f);
  o.z = __float2ll_rn(ey * 4294967296.0f);
  o.w = __float2ll_rn(ez * 4294967296.0f);
  reinterpret_cast<longlong4 *>(acck)[i] = o;
}

cudaError_t launch_green32(mmnb_handle *h)
{
  const long nk = (long) h->mesh[0] * h->mesh[1] * (h->mesh[2] / 2 + 1);
  k_green_to_f32<<<div_up(nk, 256), 256, 0, h->stream>>>(nk, h->d_green, h->d_green32);
  return cudaGetLastError();
}

// charge assignment of sites [lo, hi) into the fixed-point mesh, in the
// layout the handle's tuning picks
template <int P>
static void spread_mixed_p(mmnb_handle *h, const MeshArgs &m, const double *d_r, int lo, int hi)
{
  const int n = hi - lo;
  if (n <= 0)
    return;
  const double *r = d_r + 3 * (size_t) lo;
  const double *q = h->d_q + lo;
  const int *mask = h->d_mask + lo;
  if (h->tune.spread_planes == 2)
    k_spread_mixed_zlanes<P><<<div_up(div_up(n, 32 / P) * 32, 128), 128, 0, h->stream>>>(m, r, q, mask, n,
                                                                                       h->d_mesh_fx);
  else if (h->tune.spread_planes)
    k_spread_mixed_planes<P><<<div_up(n * P, 128), 128, 0, h->stream>>>(m, r, q, mask, n, h->d_mesh_fx);
  else
    k_spread_mixed<P><<<div_up(n, 128), 128, 0, h->stream>>>(m, r, q, mask, n, h->d_mesh_fx);
  h->launches += 1;
}

// stage bits: 1 charge assignment and transforms, 2 interpolation, 4 (with 1)
// the transforms without the assignment (done piecewise by
// launch_spread_mixed_range)
template <int P>
static cudaError_t p3m_mixed_p(mmnb_handle *h, const double *d_r, int stage)
{
  const MeshArgs m = mesh_args(h);
  const size_t nr = (size_t) h->mesh[0] * h->mesh[1] * h->mesh[2];
  const long nk = (long) h->mesh[0] * h->mesh[1] * (h->mesh[2] / 2 + 1);
  if (stage & 1) {
    if (!(stage & 4))
      spread_mixed_p<P>(h, m, d_r, 0, h->nsite);
    k_mesh_fx_to_f32<<<div_up((long) nr, 256), 256, 0, h->stream>>>(nr, h->d_mesh_fx, h->d_mesh32);
    timing_mark(h, "p3m_spread");
    if (cufftSetStream(h->plan_r2c32, h->stream) != CUFFT_SUCCESS ||
        cufftSetStream(h->plan_c2r32, h->stream) != CUFFT_SUCCESS ||
        cufftExecR2C(h->plan_r2c32, h->d_mesh32, h->d_meshk32) != CUFFT_SUCCESS)
      return cudaErrorUnknown;
    if (h->d_egrid32) {
      k_green_mul32_ik<<<div_up(nk, 256), 256, 0, h->stream>>>(nk, h->d_green32, h->d_kvec, h->d_meshk32,
                                                               h->d_egridk32);
      for (int d = 0; d < 3; d++)
        if (cufftExecC2R(h->plan_c2r32, h->d_egridk32 + d * nk, h->d_egrid32 + d * nr) != CUFFT_SUCCESS)
          return cudaErrorUnknown;
    } else {
      k_green_mul32<<<div_up(nk, 256), 256, 0, h->stream>>>(nk, h->d_green32, h->d_meshk32);
    }
    if (cufftExecC2R(h->plan_c2r32, h->d_meshk32, h->d_mesh32) != CUFFT_SUCCESS)
      return cudaErrorUnknown;
    timing_mark(h, "p3m_fft");
    h->launches += 2;
  }
  if (stage & 2) {
    if (h->d_egrid32)
      k_gather_mixed_ik<P><<<div_up(h->nsite, 128), 128, 0, h->stream>>>(m, d_r, h->nsite, h->d_mesh32,
                                                                          h->d_egrid32, nr, h->mx.acck);
    else
      k_gather_mixed<P><<<div_up(h->nsite, 128), 128, 0, h->stream>>>(m, d_r, h->nsite, h->d_mesh32, h->mx.acck);
    timing_mark(h, "p3m_gather");
    h->launches += 1;
  }
  return cudaGetLastError();
}

template <int P>
static cudaError_t spread_range_p(mmnb_handle *h, const double *d_r, int lo, int hi)
{
  spread_mixed_p<P>(h, mesh_args(h), d_r, lo, hi);
  return cudaGetLastError();
}

cudaError_t launch_spread_mixed_range(mmnb_handle *h, const double *d_r, int lo, int hi)
{
  switch (h->cfg.p3m_assignment_order) {
  case 2: return spread_range_p<2>(h, d_r, lo, hi);
  case 3: return spread_range_p<3>(h, d_r, lo, hi);
  case 4: return spread_range_p<4>(h, d_r, lo, hi);
  case 5: return spread_range_p<5>(h, d_r, lo, hi);
  case 6: return spread_range_p<6>(h, d_r, lo, hi);
  case 7: return spread_range_p<7>(h, d_r, lo, hi);
  default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_p3m_mixed(mmnb_handle *h, const double *d_r, int stage)
{
  switch (h->cfg.p3m_assignment_order) {
  case 2: return p3m_mixed_p<2>(h, d_r, stage);
  case 3: return p3m_mixed_p<3>(h, d_r, stage);
  case 4: return p3m_mixed_p<4>(h, d_r, stage);
  case 5: return p3m_mixed_p<5>(h, d_r, stage);
  case 6: return p3m_mixed_p<6>(h, d_r, stage);
  case 7: return p3m_mixed_p<7>(h, d_r, stage);
  default: return cudaErrorInvalidValue;
  }
}

}  // namespace mmnb

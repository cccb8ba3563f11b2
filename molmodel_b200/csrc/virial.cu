// Virial of the nonbonded energy for volume moves: dU/ds at s = 1 along the
// path the reference's volume moves take (MSys::scale, src/msys.cpp:416-421,
// with ElecLJ::scale, src/eleclj.cpp:1268-1280): the box edges times s, every
// molecule translated rigidly so its centre of mass is times s, eta / s, the
// P3M influence function / s with the mesh counts kept, the real-space cutoff
// and switch kept.  The reference has no virial; its own check of this path is
// MSimProgram::test_scale (src/msimprog.cpp:379-400), the energy before and
// after one such scaling.
//
// With eta proportional to 1/L every electrostatic term (real-space erfc,
// exclusion corrections, reciprocal space, self and neutralising terms) is
// homogeneous of degree -1 in the lengths, so along the path its derivative is
// -U_elec plus the work of the forces against the sites' fixed offsets from
// their molecules' centres; the terms that are not homogeneous are the LJ
// pairs, the switch (its width and rc stay fixed) and the LJ tail (2 pi / V):
//
//   dU/ds = sum_i F_i . (r_i - R_mol(i)) - U_elec - X - 3 U_tail
//
// F_i the total force on site i, R_mol(i) its molecule's centre of mass, and X
// the sum over group pairs inside the cutoff of (LJ force scalar) r^2 over the
// LJ site pairs plus (switch derivative x unswitched pair energy) R^2 of the
// anchors -- the pair kernels accumulate X beside the forces when this entry
// point asks them to, in FP64 (FP64 form) or in 64-bit fixed point (mixed
// form), and the sums below run in FP64 in a fixed order.  Screened charges
// (r_screen > 0) bring a fixed length into the Coulomb terms and are refused.

#include "mmnb_internal.cuh"

#include <string>
#include <vector>

namespace mmnb {

constexpr int kVirThreads = 256;

// per molecule: its centre of mass, then sum over its sites of F . (r - R)
__global__ void k_virial_mol(int nmol, const int *__restrict__ mol, const double *__restrict__ mass,
                             const double *__restrict__ r, const double *__restrict__ f, double *__restrict__ out)
{
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nmol)
    return;
  const int a = mol[2 * m], b = mol[2 * m + 1];
  double mt = 0, cx = 0, cy = 0, cz = 0;
  for (int i = a; i < b; i++) {
    mt += mass[i];
    cx += mass[i] * r[3 * i];
    cy += mass[i] * r[3 * i + 1];
    cz += mass[i] * r[3 * i + 2];
  }
  cx /= mt;
  cy /= mt;
  cz /= mt;
  double w = 0;
  for (int i = a; i < b; i++)
    w += f[3 * i] * (r[3 * i] - cx) + f[3 * i + 1] * (r[3 * i + 1] - cy) + f[3 * i + 2] * (r[3 * i + 2] - cz);
  out[m] = w;
}

__device__ __forceinline__ double block_sum_vir(double v, double *sh)
{
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  const double t = sh[0];
  __syncthreads();
  return t;
}

// one block: res[0] = sum of the molecules' F . (r - R), res[1] = X
__global__ void __launch_bounds__(kVirThreads) k_virial_sum(int nmol, const double *__restrict__ mol_w,
                                                            const double *__restrict__ part, int npart,
                                                            const unsigned long long *__restrict__ fixed,
                                                            double *__restrict__ res)
{
  __shared__ double sh[kVirThreads];
  double w = 0, x = 0;
  for (int k = threadIdx.x; k < nmol; k += blockDim.x)
    w += mol_w[k];
  for (int k = threadIdx.x; k < npart; k += blockDim.x)
    x += part[k];
  w = block_sum_vir(w, sh);
  x = block_sum_vir(x, sh);
  if (threadIdx.x == 0) {
    if (fixed)
      x += (double) (long long) *fixed * kFxInv;
    res[0] = w;
    res[1] = x;
  }
}

}  // namespace mmnb

using namespace mmnb;

static int vir_fail(mmnb_handle *h, int code, const std::string &msg)
{
  if (h)
    h->err = "mmnb_virial: " + msg;
  return code;
}

extern "C" int mmnb_virial(mmnb_handle *h, const double *r, int nmol, const int *mol, const double *site_mass,
                           double *f, double *u, mmnb_energy *e, double *w)
{
  if (!h || !r || !mol || !site_mass || !w)
    return vir_fail(h, MMNB_ERR_ARG, "null handle, positions, molecules, masses or output");
  if (!h->params_set)
    return vir_fail(h, MMNB_ERR_STATE, "mmnb_set_params has not been called");
  if (h->has_rscreen)
    return vir_fail(h, MMNB_ERR_UNSUPPORTED, "screened charges (r_screen > 0) are not homogeneous in the lengths");
  if (nmol < 1)
    return vir_fail(h, MMNB_ERR_ARG, "nmol must be >= 1");
  std::vector<char> seen(h->nsite, 0);
  for (int m = 0; m < nmol; m++) {
    const int a = mol[2 * m], b = mol[2 * m + 1];
    if (a < 0 || b > h->nsite || b <= a)
      return vir_fail(h, MMNB_ERR_ARG, "molecule " + std::to_string(m) + " has an invalid site range");
    double mt = 0;
    for (int i = a; i < b; i++) {
      if (seen[i])
        return vir_fail(h, MMNB_ERR_ARG, "site " + std::to_string(i) + " belongs to two molecules");
      seen[i] = 1;
      if (!(site_mass[i] >= 0))
        return vir_fail(h, MMNB_ERR_ARG, "site masses must be >= 0");
      mt += site_mass[i];
    }
    if (!(mt > 0))
      return vir_fail(h, MMNB_ERR_ARG, "molecule " + std::to_string(m) + " has no mass");
  }
  for (int i = 0; i < h->nsite; i++)
    if (!seen[i])
      return vir_fail(h, MMNB_ERR_ARG, "site " + std::to_string(i) + " belongs to no molecule");
  // scratch: molecule ranges, masses, per-molecule sums, two results
  cudaError_t ce = cudaSuccess;
  if (h->vir_mol_cap < nmol) {
    if (h->d_vir_mol)
      cudaFree(h->d_vir_mol);
    if (h->d_vir_molw)
      cudaFree(h->d_vir_molw);
    h->d_vir_mol = nullptr;
    h->d_vir_molw = nullptr;
    h->vir_mol_cap = 0;
    if ((ce = cudaMalloc(&h->d_vir_mol, sizeof(int) * 2 * (size_t) nmol)) != cudaSuccess ||
        (ce = cudaMalloc(&h->d_vir_molw, sizeof(double) * ((size_t) nmol + 2))) != cudaSuccess)
      return vir_fail(h, MMNB_ERR_CUDA, std::string("scratch: ") + cudaGetErrorString(ce));
    h->vir_mol_cap = nmol;
  }
  if (!h->d_vir_mass && (ce = cudaMalloc(&h->d_vir_mass, sizeof(double) * (size_t) h->nsite)) != cudaSuccess)
    return vir_fail(h, MMNB_ERR_CUDA, std::string("scratch: ") + cudaGetErrorString(ce));
  if ((ce = cudaMemcpyAsync(h->d_vir_mol, mol, sizeof(int) * 2 * (size_t) nmol, cudaMemcpyHostToDevice,
                            h->stream)) != cudaSuccess ||
      (ce = cudaMemcpyAsync(h->d_vir_mass, site_mass, sizeof(double) * (size_t) h->nsite, cudaMemcpyHostToDevice,
                            h->stream)) != cudaSuccess)
    return vir_fail(h, MMNB_ERR_CUDA, cudaGetErrorString(ce));
  // the evaluation, with the pair kernels accumulating X
  mmnb_energy en;
  h->want_virial = true;
  const int s = mmnb_compute(h, r, f, u, &en, nullptr, nullptr);
  h->want_virial = false;
  if (s)
    return s;
  if (e)
    *e = en;
  // X's partial sums: per row (FP64 water kernel), per block (other kernels,
  // then the exclusion kernel's 1-4 LJ blocks), or one fixed-point word
  // (mixed water kernel)
  const double *part = h->d_vir_part;
  int npart = 0;
  const unsigned long long *fixed = nullptr;
  if (h->cfg.include_rspace) {
    if (h->used_water64) {
      part = h->d_vir_row;
      npart = h->ngroup;
    } else if (h->used_water) {
      fixed = h->d_wsum + 4;
    } else {
      npart = h->lj_pair_blocks;
    }
  }
  double *res = h->d_vir_molw + nmol;
  k_virial_mol<<<div_up(nmol, kVirThreads), kVirThreads, 0, h->stream>>>(nmol, h->d_vir_mol, h->d_vir_mass,
                                                                         h->d_r, h->d_f, h->d_vir_molw);
  k_virial_sum<<<1, kVirThreads, 0, h->stream>>>(nmol, h->d_vir_molw, part, npart, fixed, res);
  h->launches += 2;
  double out[3] = {0, 0, 0};
  if ((ce = cudaGetLastError()) != cudaSuccess ||
      (ce = cudaMemcpyAsync(out, res, sizeof(double) * 2, cudaMemcpyDeviceToHost, h->stream)) != cudaSuccess)
    return vir_fail(h, MMNB_ERR_CUDA, cudaGetErrorString(ce));
  if (h->cfg.include_rspace && h->use_14) {
    // the 1-4 LJ terms of the exclusion kernel (intramolecular: they add to X)
    std::vector<double> p14(h->lj_excl_blocks);
    if ((ce = cudaMemcpyAsync(p14.data(), h->d_vir_part + h->lj_pair_blocks, sizeof(double) * p14.size(),
                              cudaMemcpyDeviceToHost, h->stream)) != cudaSuccess)
      return vir_fail(h, MMNB_ERR_CUDA, cudaGetErrorString(ce));
    if ((ce = cudaStreamSynchronize(h->stream)) != cudaSuccess)
      return vir_fail(h, MMNB_ERR_CUDA, cudaGetErrorString(ce));
    for (double v : p14)
      out[2] += v;
  }
  if ((ce = cudaStreamSynchronize(h->stream)) != cudaSuccess)
    return vir_fail(h, MMNB_ERR_CUDA, cudaGetErrorString(ce));
  *w = out[0] - en.elec - (out[1] + out[2]) - 3 * en.lj_correction;
  return MMNB_OK;
}

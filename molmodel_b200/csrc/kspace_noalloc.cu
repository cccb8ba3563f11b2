// Ordinary Ewald reciprocal sum for callers that cannot allocate device memory.
//
// mmnb_create allocates every buffer the k-sum needs (wave vectors, a_k and
// the structure factors) with cudaMalloc.  Some callers cannot do that: a host
// program that has reserved all device memory for its own pool (cudaMalloc
// then fails), or a driver loop that must not let an allocation or free
// synchronise the device in the middle of a step.  mmnb_kspace_field_noalloc
// gives them the same computation with no allocation at all: its only scratch
// memory is the fixed array below, which exists once per device for the life
// of the process, and the caller passes positions, charges and the output
// arrays as device pointers.
//
// Limits and sharing: the array holds at most kNoallocMaxK wave vectors (about
// a cutoff of 12 in units of the reciprocal lattice); larger cutoffs are
// rejected.  Every call on a device uses the same array and overwrites it —
// calls whose kernels overlap on the GPU (different streams, or host threads)
// race and give wrong results.  Nothing in it needs to start at zero: each call
// writes the wave-vector table and the structure factors before reading them.

#include "mmnb_internal.cuh"

#include <mutex>

namespace mmnb {

constexpr int kNoallocMaxK = 4096;
constexpr int kNoallocMaxDevices = 64;

// [0, 3K) wave vectors, [3K, 4K) a_k, [4K, 6K) structure factor (cos, sin), [6K] count
__device__ __align__(256) static double g_noalloc_kspace[6 * kNoallocMaxK + 8];

// Wave vectors in the order the k-sum walks them (src/kspace.c:35-58): the
// half space of integer n with |n|^2 <= kc^2 + 1e-8, sorted by |n|^2, largest
// first, ties in enumeration order (the reference's qsort does not promise a
// tie order; ties only change the order of the floating-point sum).
//
// One warp ranks every point of the enumeration box (nx in [0, nmax], ny and
// nz in [-nmax, nmax], lexicographic, i.e. the enumeration order) in two
// passes over chunks of 32 consecutive points: the first counts the points of
// each shell |n|^2 = s, lane 0 turns the counts into the first slot of each
// shell (largest s first), and the second gives each point its slot = first
// slot of its shell + points of the shell in earlier chunks + points of the
// shell in earlier lanes of this chunk (__match_any_sync).  The box has at
// most 14 x 27 x 27 = 10,206 points (kc <= 13.5), so each pass takes at most
// 319 steps of the warp.
constexpr int kNoallocMaxShell = 192;  // |n|^2 <= kc^2 + 1e-8 < 192 for kc <= kNoallocMaxCut
constexpr double kNoallocMaxCut = 13.5;

__global__ void __launch_bounds__(32) k_noalloc_table(double kc, double rx, double ry, double rz, double volume,
                                                       double eta, double *scratch)
{
  __shared__ int first[kNoallocMaxShell + 1], seen[kNoallocMaxShell + 1];
  const int lane = threadIdx.x;
  double *kvec = scratch, *ak = scratch + 3 * kNoallocMaxK;
  const double n2max = kc * kc + 1e-8;
  const int nmax = (int) floor(kc);
  const int side = 2 * nmax + 1;
  const int nbox = (nmax + 1) * side * side;
  for (int s = lane; s <= kNoallocMaxShell; s += 32) {
    first[s] = 0;
    seen[s] = 0;
  }
  __syncwarp();
  // shell of enumeration point i, or -1 outside the half space or the cutoff
  auto shell = [&](int i, int &nx, int &ny, int &nz) -> int {
    if (i >= nbox)
      return -1;
    nx = i / (side * side);
    ny = (i / side) % side - nmax;
    nz = i % side - nmax;
    if (nx == 0 && (ny < 0 || (ny == 0 && nz < 1)))
      return -1;
    const int n2 = nx * nx + ny * ny + nz * nz;
    return n2 <= n2max ? n2 : -1;
  };
  for (int c = 0; c < nbox; c += 32) {
    int nx, ny, nz;
    const int s = shell(c + lane, nx, ny, nz);
    if (s > 0)
      atomicAdd(&first[s], 1);
  }
  __syncwarp();
  if (lane == 0) {
    int run = 0;
    for (int s = kNoallocMaxShell; s >= 1; s--) {
      const int n = first[s];
      first[s] = run;
      run += n;
    }
    scratch[6 * kNoallocMaxK] = run;
  }
  __syncwarp();
  const double c2 = 0.25 / (eta * eta), f = 4 * M_PI / volume;
  const unsigned lower = (1u << lane) - 1;
  for (int c = 0; c < nbox; c += 32) {
    int nx = 0, ny = 0, nz = 0;
    const int s = shell(c + lane, nx, ny, nz);
    const unsigned same = __match_any_sync(0xffffffffu, s);
    if (s > 0) {
      const int slot = first[s] + seen[s] + __popc(same & lower);
      if (slot < kNoallocMaxK) {
        const double kx = rx * nx, ky = ry * ny, kz = rz * nz;
        const double k2 = kx * kx + ky * ky + kz * kz;
        kvec[3 * slot] = kx;
        kvec[3 * slot + 1] = ky;
        kvec[3 * slot + 2] = kz;
        ak[slot] = f * exp(-k2 * c2) / k2;
      }
    }
    __syncwarp();
    // the lowest lane of each shell present in this chunk advances its count
    if (s > 0 && (same & lower) == 0)
      seen[s] += __popc(same);
    __syncwarp();
  }
}

constexpr int kNoallocThreads = 256;

__global__ void k_noalloc_structure(int nsite, const double *__restrict__ r, const double *__restrict__ q,
                                    double *scratch)
{
  __shared__ double sc[kNoallocThreads], ss[kNoallocThreads];
  const int k = blockIdx.x;
  const double *kvec = scratch;
  double *skc = scratch + 4 * kNoallocMaxK;
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

__global__ void k_noalloc_field(int nsite, int nk, const double *__restrict__ r, const double *scratch,
                                double *__restrict__ phi, double *__restrict__ evec)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsite)
    return;
  const double *kvec = scratch, *ak = scratch + 3 * kNoallocMaxK, *skc = scratch + 4 * kNoallocMaxK;
  const double x = r[3 * i], y = r[3 * i + 1], z = r[3 * i + 2];
  double p = 0, gx = 0, gy = 0, gz = 0;
  for (int k = 0; k < nk; k++) {
    const double kx = kvec[3 * k], ky = kvec[3 * k + 1], kz = kvec[3 * k + 2];
    double sn, cs;
    sincos(kx * x + ky * y + kz * z, &sn, &cs);
    const double a2 = 2 * ak[k];
    const double cQ = skc[2 * k], sQ = skc[2 * k + 1];
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

// Device address of the scratch array, looked up once per device with that
// device current (the array's name is only a host-side stand-in).
static double *noalloc_scratch(int dev, int &status)
{
  static std::mutex mu;
  static double *addr[kNoallocMaxDevices] = {nullptr};
  status = MMNB_OK;
  if (dev < 0 || dev >= kNoallocMaxDevices) {
    status = set_global_error(MMNB_ERR_ARG, "mmnb_kspace_field_noalloc: device ordinal out of range");
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_kspace);
    if (e != cudaSuccess) {
      status = set_global_error(MMNB_ERR_CUDA, std::string("mmnb_kspace_field_noalloc: cudaGetSymbolAddress: ") +
                                                   cudaGetErrorString(e));
      return nullptr;
    }
    addr[dev] = (double *) p;
  }
  return addr[dev];
}

}  // namespace mmnb

using namespace mmnb;

extern "C" int mmnb_kspace_field_noalloc(int nsite, const double *d_r, const double *d_q, int bctype,
                                         const double box[3], double eta, double kspace_cutoff, double *d_phi,
                                         double *d_evec, void *stream)
{
  if (nsite <= 0 || !d_r || !d_q || !d_phi || !d_evec || !box)
    return set_global_error(MMNB_ERR_ARG, "mmnb_kspace_field_noalloc: null array or nsite <= 0");
  if (bctype != MMNB_CUBIC && bctype != MMNB_ORTHORHOMBIC)
    return set_global_error(MMNB_ERR_UNSUPPORTED, "mmnb_kspace_field_noalloc: cubic or orthorhombic boxes only");
  double L[3];
  for (int d = 0; d < 3; d++) {
    L[d] = bctype == MMNB_CUBIC ? box[0] : box[d];
    if (!(L[d] > 0))
      return set_global_error(MMNB_ERR_ARG, "mmnb_kspace_field_noalloc: box lengths must be > 0");
  }
  if (!(eta > 0) || !(kspace_cutoff > 0))
    return set_global_error(MMNB_ERR_ARG, "mmnb_kspace_field_noalloc: eta and kspace_cutoff must be > 0");
  // Past a cutoff of 13.5 the half space holds more than the array's wave
  // vectors whatever the box (a ball of radius 13.5 - sqrt(3)/2 alone gives
  // 4219 half-space points), so such cutoffs, infinities and NaN are refused
  // before any counting; below it the exact count is a loop of at most
  // 14 x 27 x 27 steps.
  if (!(kspace_cutoff <= kNoallocMaxCut))
    return set_global_error(MMNB_ERR_ARG, "mmnb_kspace_field_noalloc: kspace_cutoff " +
                                              std::to_string(kspace_cutoff) +
                                              " needs more wave vectors than this entry point holds (at most " +
                                              std::to_string(kNoallocMaxK) + ")");
  const double n2max = kspace_cutoff * kspace_cutoff + 1e-8;
  const int nmax = (int) floor(kspace_cutoff);
  long nk = 0;
  for (int nx = 0; nx <= nmax; nx++)
    for (int ny = (nx == 0 ? 0 : -nmax); ny <= nmax; ny++)
      for (int nz = (nx == 0 && ny == 0 ? 1 : -nmax); nz <= nmax; nz++)
        if (nx * nx + ny * ny + nz * nz <= n2max)
          nk++;
  if (nk > kNoallocMaxK)
    return set_global_error(MMNB_ERR_ARG, "mmnb_kspace_field_noalloc: kspace_cutoff " +
                                              std::to_string(kspace_cutoff) + " needs " + std::to_string(nk) +
                                              " wave vectors; this entry point holds at most " +
                                              std::to_string(kNoallocMaxK));
  if (nk == 0)
    return MMNB_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return set_global_error(MMNB_ERR_CUDA, std::string("mmnb_kspace_field_noalloc: ") + cudaGetErrorString(e));
  int status;
  double *scratch = noalloc_scratch(dev, status);
  if (!scratch)
    return status;
  cudaStream_t s = (cudaStream_t) stream;
  k_noalloc_table<<<1, 32, 0, s>>>(kspace_cutoff, 2 * M_PI * (1.0 / L[0]), 2 * M_PI * (1.0 / L[1]),
                                  2 * M_PI * (1.0 / L[2]), L[0] * L[1] * L[2], eta, scratch);
  k_noalloc_structure<<<(int) nk, kNoallocThreads, 0, s>>>(nsite, d_r, d_q, scratch);
  k_noalloc_field<<<div_up(nsite, 128), 128, 0, s>>>(nsite, (int) nk, d_r, scratch, d_phi, d_evec);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_global_error(MMNB_ERR_CUDA, std::string("mmnb_kspace_field_noalloc: ") + cudaGetErrorString(e));
  return MMNB_OK;
}

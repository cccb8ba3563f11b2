// Molecular dynamics on the device: velocity Verlet with rigid 3-site water.
//
// One step, as MDyn::run performs it (src/mdyn.cpp:142-160):
//   v += f dt / 2m;  x += v dt;  constrain positions (v += dx / dt);
//   f = F(x) (the nonbonded evaluation of this library);
//   v += f dt / 2m;  constrain velocities.
// The reference constrains with ConstraintGroup (src/constraint.cpp:295-358):
// Newton iterations of the linearised constraints with the displacement
// directions taken from the previous positions (SHAKE), then one linear
// solve for the velocities (RATTLE).  For a rigid triangle both have closed
// forms: the positions follow from SETTLE (Miyamoto & Kollman, J. Comput.
// Chem. 13, 952 (1992)), the velocities from a 3 x 3 solve, both in FP64.
// Their results are the constraint solutions the reference's iterations
// converge to.
//
// The step (force zeroing, the two half kicks with their constraints, the
// evaluation and the energy record) is captured once into a CUDA graph and
// replayed; kinetic energy is reduced per block and summed in index order by
// the last block, and each step's (kinetic, potential, conserved) energies are
// appended to a device log that is read back once per run.

#include <algorithm>
#include <string>
#include <vector>

#include "mmnb_internal.cuh"

struct mmnb_md {
  mmnb_handle *h = nullptr;
  double dt = 0;
  int rigid = 0;
  int nsite = 0, nmol = 0;
  // rigid water: masses and the canonical triangle (centre of mass at the
  // origin, O on +y): O at (0, ra), H at (-/+ rc, -rb)
  double m_o = 0, m_h = 0, ra = 0, rb = 0, rc = 0, d_oh = 0, d_hh = 0;
  double *d_r = nullptr, *d_v = nullptr, *d_f = nullptr, *d_minv = nullptr, *d_m = nullptr;
  double *d_energy = nullptr;   // the evaluation's energies (elec, lj, tail, total)
  double *d_ke_part = nullptr;  // per block
  double *d_log = nullptr;      // 3 per step
  unsigned long long *d_ctl = nullptr;  // [0] finished-block counter, [1] log position
  int log_cap = 0;
  int ke_blocks = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long gen = -1;                // the handle's buffer generation at the capture
  std::string err;
};

// Several replicas stepped by one graph launch: an independent branch per
// replica, each on its replica's stream.
struct mmnb_md_batch {
  std::vector<mmnb_md *> md;
  cudaStream_t master = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> done;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<long> gen;        // each replica handle's buffer generation at the capture
  std::string err;
};

namespace mmnb {

constexpr int kMdThreads = 256;

__global__ void k_md_scale(double *__restrict__ v, int n, double s)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    v[i] *= s;
}

struct MdArgs {
  int nsite, nmol, rigid;
  double dt;
  double m_o, m_h, ra, rb, rc;
  double *r, *v;
  const double *f, *minv, *m;
  // energy record
  const double *energy;
  double *ke_part, *log;
  unsigned long long *ctl;
  int log_cap;
};

struct V3 {
  double x, y, z;
};

__device__ __forceinline__ V3 ld3(const double *p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ void st3(double *p, V3 a)
{
  p[0] = a.x;
  p[1] = a.y;
  p[2] = a.z;
}
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b)
{
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ V3 unit(V3 a) { return rsqrt(dot(a, a)) * a; }

// SETTLE for one molecule.  a0, b0, c0: positions before the drift (a valid
// triangle); a1, b1, c1: after the drift.  Returns the constrained positions.
//
// The constraint displacements are built from the old bond vectors, which
// lie in the old triangle's plane, so in a frame whose Z axis is that plane's
// normal the new positions keep the drifted z coordinates (origin at the
// drifted centre of mass, which the constraints do not move).  A canonical
// triangle tilted by phi about X and psi about Y reproduces those three z
// values; the remaining rotation theta about Z is fixed by the displacements
// having no net torque about the old positions (pairwise central forces):
// alpha sin(theta) + beta cos(theta) = gamma.
__device__ void settle_positions(const MdArgs &a, V3 a0, V3 b0, V3 c0, V3 &a1, V3 &b1, V3 &c1)
{
  const double M = a.m_o + 2 * a.m_h;
  const V3 com = (1.0 / M) * (a.m_o * a1 + a.m_h * (b1 + c1));
  const V3 a1d = a1 - com, b1d = b1 - com, c1d = c1 - com;
  const V3 ez = unit(cross(b0 - a0, c0 - a0));
  const V3 ex = unit(cross(a1d, ez));
  const V3 ey = cross(ez, ex);
  // old bond vectors from O and drifted positions in the frame
  const V3 ob = b0 - a0, oc = c0 - a0;
  const double xb0 = dot(ob, ex), yb0 = dot(ob, ey), xc0 = dot(oc, ex), yc0 = dot(oc, ey);
  const double za1 = dot(a1d, ez);
  const double xb1 = dot(b1d, ex), yb1 = dot(b1d, ey), zb1 = dot(b1d, ez);
  const double xc1 = dot(c1d, ex), yc1 = dot(c1d, ey), zc1 = dot(c1d, ez);
  // tilts
  const double sphi = za1 / a.ra;
  const double cphi = sqrt(fmax(0.0, 1 - sphi * sphi));
  const double spsi = (zb1 - zc1) / (2 * a.rc * cphi);
  const double cpsi = sqrt(fmax(0.0, 1 - spsi * spsi));
  const double ya2 = a.ra * cphi;
  const double xb2 = -a.rc * cpsi;
  const double yb2 = -a.rb * cphi - a.rc * spsi * sphi;
  const double yc2 = -a.rb * cphi + a.rc * spsi * sphi;
  // in-plane rotation
  const double alpha = xb2 * (xb0 - xc0) + yb0 * yb2 + yc0 * yc2;
  const double beta = xb2 * (yc0 - yb0) + xb0 * yb2 + xc0 * yc2;
  const double gamma = xb0 * yb1 - xb1 * yb0 + xc0 * yc1 - xc1 * yc0;
  const double ab2 = alpha * alpha + beta * beta;
  const double sth = (alpha * gamma - beta * sqrt(fmax(0.0, ab2 - gamma * gamma))) / ab2;
  const double cth = sqrt(fmax(0.0, 1 - sth * sth));
  // rotated canonical triangle, back to the lab frame
  const double xa3 = -ya2 * sth, ya3 = ya2 * cth;
  const double xb3 = xb2 * cth - yb2 * sth, yb3 = xb2 * sth + yb2 * cth;
  const double xc3 = -xb2 * cth - yc2 * sth, yc3 = -xb2 * sth + yc2 * cth;
  a1 = com + xa3 * ex + ya3 * ey + za1 * ez;
  b1 = com + xb3 * ex + yb3 * ey + zb1 * ez;
  c1 = com + xc3 * ex + yc3 * ey + zc1 * ez;
}

// velocity constraint: v += M^-1 sum_k mu_k u_k with u the current bond
// vectors, mu from (v_i - v_j) . u_ij = 0 for the three bonds (Cramer's rule)
__device__ void settle_velocities(const MdArgs &a, V3 ra_, V3 rb_, V3 rc_, V3 &va, V3 &vb, V3 &vc)
{
  const double io = 1.0 / a.m_o, ih = 1.0 / a.m_h;
  const V3 uab = ra_ - rb_, uac = ra_ - rc_, ubc = rb_ - rc_;
  // constraint k: g_k . v = 0; the correction of mu_l changes g_k . v by S_kl mu_l
  const double s11 = (io + ih) * dot(uab, uab), s22 = (io + ih) * dot(uac, uac), s33 = 2 * ih * dot(ubc, ubc);
  const double s12 = io * dot(uab, uac), s13 = -ih * dot(uab, ubc), s23 = ih * dot(uac, ubc);
  const double r1 = -dot(va - vb, uab), r2 = -dot(va - vc, uac), r3 = -dot(vb - vc, ubc);
  const double det = s11 * (s22 * s33 - s23 * s23) - s12 * (s12 * s33 - s23 * s13) + s13 * (s12 * s23 - s22 * s13);
  const double m1 = (r1 * (s22 * s33 - s23 * s23) - s12 * (r2 * s33 - s23 * r3) + s13 * (r2 * s23 - s22 * r3)) / det;
  const double m2 = (s11 * (r2 * s33 - s23 * r3) - r1 * (s12 * s33 - s23 * s13) + s13 * (s12 * r3 - r2 * s13)) / det;
  const double m3 = (s11 * (s22 * r3 - r2 * s23) - s12 * (s12 * r3 - r2 * s13) + r1 * (s12 * s23 - s22 * s13)) / det;
  va = va + io * (m1 * uab + m2 * uac);
  vb = vb + ih * (-1.0 * m1 * uab + m3 * ubc);
  vc = vc + ih * (-1.0 * m2 * uac - m3 * ubc);
}

// first half kick, drift, position constraint (one thread per molecule, or
// per site without constraints)
__global__ void k_md_drift(MdArgs a)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const double hdt = 0.5 * a.dt;
  if (!a.rigid) {
    if (t >= a.nsite)
      return;
    V3 v = ld3(a.v + 3 * t) + (hdt * a.minv[t]) * ld3(a.f + 3 * t);
    st3(a.v + 3 * t, v);
    st3(a.r + 3 * t, ld3(a.r + 3 * t) + a.dt * v);
    return;
  }
  if (t >= a.nmol)
    return;
  const int s = 3 * t;
  V3 x0[3], x1[3], v[3];
  for (int k = 0; k < 3; k++) {
    x0[k] = ld3(a.r + 3 * (s + k));
    v[k] = ld3(a.v + 3 * (s + k)) + (hdt * a.minv[s + k]) * ld3(a.f + 3 * (s + k));
    x1[k] = x0[k] + a.dt * v[k];
  }
  V3 y[3] = {x1[0], x1[1], x1[2]};
  settle_positions(a, x0[0], x0[1], x0[2], y[0], y[1], y[2]);
  const double idt = 1.0 / a.dt;
  for (int k = 0; k < 3; k++) {
    st3(a.r + 3 * (s + k), y[k]);
    st3(a.v + 3 * (s + k), v[k] + idt * (y[k] - x1[k]));
  }
}

__device__ __forceinline__ double md_block_sum(double x, double *sh)
{
  sh[threadIdx.x] = x;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  return sh[0];
}

// second half kick, velocity constraint, kinetic energy and the step's record
__global__ void __launch_bounds__(kMdThreads) k_md_kick(MdArgs a, int kick)
{
  __shared__ double sh[kMdThreads];
  __shared__ bool last;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const double hdt = kick ? 0.5 * a.dt : 0.0;
  double ke = 0;
  if (!a.rigid) {
    if (t < a.nsite) {
      V3 v = ld3(a.v + 3 * t) + (hdt * a.minv[t]) * ld3(a.f + 3 * t);
      st3(a.v + 3 * t, v);
      ke = 0.5 * a.m[t] * dot(v, v);
    }
  } else if (t < a.nmol) {
    const int s = 3 * t;
    V3 x[3], v[3];
    for (int k = 0; k < 3; k++) {
      x[k] = ld3(a.r + 3 * (s + k));
      v[k] = ld3(a.v + 3 * (s + k)) + (hdt * a.minv[s + k]) * ld3(a.f + 3 * (s + k));
    }
    settle_velocities(a, x[0], x[1], x[2], v[0], v[1], v[2]);
    for (int k = 0; k < 3; k++) {
      st3(a.v + 3 * (s + k), v[k]);
      ke += 0.5 * a.m[s + k] * dot(v[k], v[k]);
    }
  }
  const double bs = md_block_sum(ke, sh);
  if (threadIdx.x == 0) {
    a.ke_part[blockIdx.x] = bs;
    __threadfence();
    last = atomicAdd(a.ctl, 1ull) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last)
    return;
  __threadfence();
  double k = 0;
  for (int b = threadIdx.x; b < (int) gridDim.x; b += blockDim.x)
    k += a.ke_part[b];
  __syncthreads();
  k = md_block_sum(k, sh);
  if (threadIdx.x == 0) {
    const unsigned long long n = a.ctl[1];
    if (a.log && n < (unsigned long long) a.log_cap) {
      a.log[3 * n] = k;
      a.log[3 * n + 1] = a.energy[3];
      a.log[3 * n + 2] = k + a.energy[3];
    }
    a.ctl[1] = n + 1;
    a.ctl[0] = 0ull;
  }
}

}  // namespace mmnb

using namespace mmnb;

static int md_fail(mmnb_md *md, int code, const std::string &msg)
{
  if (md)
    md->err = msg;
  return code;
}

#define MDCK(x)                                                                              \
  do {                                                                                       \
    cudaError_t e_ = (x);                                                                    \
    if (e_ != cudaSuccess)                                                                   \
      return md_fail(md, MMNB_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

static MdArgs md_args(mmnb_md *md, double *log)
{
  MdArgs a;
  a.nsite = md->nsite;
  a.nmol = md->nmol;
  a.rigid = md->rigid;
  a.dt = md->dt;
  a.m_o = md->m_o;
  a.m_h = md->m_h;
  a.ra = md->ra;
  a.rb = md->rb;
  a.rc = md->rc;
  a.r = md->d_r;
  a.v = md->d_v;
  a.f = md->d_f;
  a.minv = md->d_minv;
  a.m = md->d_m;
  a.energy = md->d_energy;
  a.ke_part = md->d_ke_part;
  a.log = log;
  a.ctl = md->d_ctl;
  a.log_cap = md->log_cap;
  return a;
}

extern "C" {

int mmnb_md_create(mmnb_handle *h, const double *site_mass, double dt, int rigid_water, double r_oh,
                   double hoh_angle_deg, mmnb_md **out)
{
  if (!out)
    return MMNB_ERR_ARG;
  *out = nullptr;
  if (!h || !h->params_set || !site_mass || !(dt > 0))
    return MMNB_ERR_ARG;
  mmnb_md *md = new mmnb_md;
  md->h = h;
  md->dt = dt;
  md->rigid = rigid_water ? 1 : 0;
  md->nsite = h->nsite;
  std::vector<double> m(site_mass, site_mass + h->nsite), minv(h->nsite);
  for (int i = 0; i < h->nsite; i++) {
    if (!(m[i] > 0)) {
      delete md;
      return MMNB_ERR_ARG;
    }
    minv[i] = 1.0 / m[i];
  }
  if (md->rigid) {
    // every group [O, H, H] with equal H masses, the same masses in every molecule
    bool ok = h->nsite == 3 * h->ngroup && r_oh > 0 && hoh_angle_deg > 0 && hoh_angle_deg < 180;
    for (int g = 0; ok && g < h->ngroup; g++)
      ok = h->group[2 * g] == 3 * g && h->group[2 * g + 1] == 3 * g + 3 && m[3 * g] == m[0] &&
           m[3 * g + 1] == m[1] && m[3 * g + 2] == m[1];
    if (!ok) {
      delete md;
      return MMNB_ERR_ARG;
    }
    md->nmol = h->ngroup;
    md->m_o = m[0];
    md->m_h = m[1];
    md->d_oh = r_oh;
    md->d_hh = 2 * r_oh * sin(0.5 * hoh_angle_deg * M_PI / 180.0);
    const double height = sqrt(r_oh * r_oh - 0.25 * md->d_hh * md->d_hh);
    const double M = md->m_o + 2 * md->m_h;
    md->ra = 2 * md->m_h * height / M;
    md->rb = height - md->ra;
    md->rc = 0.5 * md->d_hh;
  }
  const size_t n3 = 3 * (size_t) h->nsite;
  md->ke_blocks = div_up(md->rigid ? md->nmol : md->nsite, kMdThreads);
  if (cudaMalloc(&md->d_r, n3 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&md->d_v, n3 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&md->d_f, n3 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&md->d_m, h->nsite * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&md->d_minv, h->nsite * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&md->d_energy, 8 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&md->d_ke_part, md->ke_blocks * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&md->d_ctl, 2 * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMemcpy(md->d_m, m.data(), h->nsite * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(md->d_minv, minv.data(), h->nsite * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(md->d_ctl, 0, 2 * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMemset(md->d_v, 0, n3 * sizeof(double)) != cudaSuccess) {
    mmnb_md_destroy(md);
    return MMNB_ERR_CUDA;
  }
  *out = md;
  return MMNB_OK;
}

int mmnb_md_set_state(mmnb_md *md, const double *r, const double *v)
{
  if (!md || !r)
    return MMNB_ERR_ARG;
  mmnb_handle *h = md->h;
  const size_t n3 = 3 * (size_t) md->nsite;
  MDCK(cudaMemcpyAsync(md->d_r, r, n3 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  if (v)
    MDCK(cudaMemcpyAsync(md->d_v, v, n3 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  else
    MDCK(cudaMemsetAsync(md->d_v, 0, n3 * sizeof(double), h->stream));
  // velocities obey the constraints before the first step (the positions
  // are taken as given: a rigid triangle)
  MDCK(cudaMemsetAsync(md->d_ctl, 0, 2 * sizeof(unsigned long long), h->stream));
  const MdArgs a = md_args(md, nullptr);
  k_md_kick<<<md->ke_blocks, kMdThreads, 0, h->stream>>>(a, 0);
  MDCK(cudaGetLastError());
  // forces at the initial positions (the first half kick uses them) through
  // the host call, which also sizes the neighbour rows
  std::vector<double> f(n3, 0.0);
  mmnb_energy en;
  int s = mmnb_compute(h, r, f.data(), nullptr, &en, nullptr, nullptr);
  if (s)
    return md_fail(md, s, mmnb_last_error(h));
  MDCK(cudaMemcpyAsync(md->d_f, f.data(), n3 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  MDCK(cudaMemsetAsync(md->d_ctl, 0, 2 * sizeof(unsigned long long), h->stream));
  MDCK(cudaStreamSynchronize(h->stream));
  return MMNB_OK;
}

// Record one step on the handle's stream (which must be capturing).
static int md_record(mmnb_md *md, double *log)
{
  mmnb_handle *h = md->h;
  const MdArgs a = md_args(md, log);
  const int n = md->rigid ? md->nmol : md->nsite;
  k_md_drift<<<div_up(n, 128), 128, 0, h->stream>>>(a);
  cudaError_t e = cudaMemsetAsync(md->d_f, 0, 3 * (size_t) md->nsite * sizeof(double), h->stream);
  if (e != cudaSuccess)
    return md_fail(md, MMNB_ERR_CUDA, cudaGetErrorString(e));
  const int s = mmnb_compute_device(h, md->d_r, md->d_f, md->d_energy);
  if (s)
    return md_fail(md, s, mmnb_last_error(h));
  k_md_kick<<<md->ke_blocks, kMdThreads, 0, h->stream>>>(a, 1);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return md_fail(md, MMNB_ERR_CUDA, cudaGetErrorString(e));
  return MMNB_OK;
}

static void md_drop_graph(mmnb_md *md)
{
  if (md->exec) {
    cudaGraphExecDestroy(md->exec);
    md->exec = nullptr;
  }
  if (md->graph) {
    cudaGraphDestroy(md->graph);
    md->graph = nullptr;
  }
}

static int md_capture(mmnb_md *md, double *log)
{
  mmnb_handle *h = md->h;
  md_drop_graph(md);
  MDCK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  h->capturing = true;
  const int s = md_record(md, log);
  cudaGraph_t g = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(h->stream, &g);
  h->capturing = false;
  if (s) {
    if (g)
      cudaGraphDestroy(g);
    return s;
  }
  MDCK(ec);
  md->graph = g;
  MDCK(cudaGraphInstantiate(&md->exec, g, cudaGraphInstantiateFlagUseNodePriority));
  md->gen = h->buf_gen;
  return MMNB_OK;
}

// the log holds at least nsteps steps (a reallocation invalidates the graph)
static int md_reserve_log(mmnb_md *md, int nsteps)
{
  if (md->log_cap >= nsteps)
    return MMNB_OK;
  if (md->d_log)
    cudaFree(md->d_log);
  md->d_log = nullptr;
  md->log_cap = 0;
  MDCK(cudaMalloc(&md->d_log, 3 * (size_t) nsteps * sizeof(double)));
  md->log_cap = nsteps;
  md_drop_graph(md);
  return MMNB_OK;
}

int mmnb_md_run(mmnb_md *md, int nsteps, double *energies)
{
  if (!md || nsteps < 0)
    return MMNB_ERR_ARG;
  mmnb_handle *h = md->h;
  if (nsteps == 0)
    return MMNB_OK;
  if (const int s = md_reserve_log(md, nsteps))
    return s;
  // captured again when the handle's buffers were reallocated since (rows
  // regrown, mmnb_scale, mmnb_set_params): the graph holds their addresses
  if (!md->exec || md->gen != h->buf_gen) {
    const int s = md_capture(md, md->d_log);
    if (s)
      return s;
  }
  MDCK(cudaMemsetAsync(md->d_ctl + 1, 0, sizeof(unsigned long long), h->stream));
  MDCK(cudaMemsetAsync(h->d_flags + kFlagOverflow, 0, sizeof(int), h->stream));
  for (int i = 0; i < nsteps; i++)
    MDCK(cudaGraphLaunch(md->exec, h->stream));
  int flags[kFlagCount];
  MDCK(cudaMemcpyAsync(flags, h->d_flags, sizeof(flags), cudaMemcpyDeviceToHost, h->stream));
  if (energies)
    MDCK(cudaMemcpyAsync(energies, md->d_log, 3 * (size_t) nsteps * sizeof(double), cudaMemcpyDeviceToHost,
                         h->stream));
  MDCK(cudaStreamSynchronize(h->stream));
  h->evals += nsteps;
  h->first = false;
  (void) flags;
  // rows cut at their capacity or a non-finite coordinate during the run: the
  // status says which; after an overflow the rows are regrown, so running again
  // from a saved state evaluates complete rows
  long trunc = 0;
  if (const int st = mmnb_check(h, &trunc, nullptr))
    return md_fail(md, st, std::string("during the run: ") + h->err);
  return MMNB_OK;
}

int mmnb_md_get_state(mmnb_md *md, double *r, double *v)
{
  if (!md)
    return MMNB_ERR_ARG;
  mmnb_handle *h = md->h;
  const size_t n3 = 3 * (size_t) md->nsite;
  if (r)
    MDCK(cudaMemcpyAsync(r, md->d_r, n3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (v)
    MDCK(cudaMemcpyAsync(v, md->d_v, n3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  MDCK(cudaStreamSynchronize(h->stream));
  return MMNB_OK;
}

const char *mmnb_md_last_error(const mmnb_md *md) { return md ? md->err.c_str() : "null md handle"; }

int mmnb_md_destroy(mmnb_md *md)
{
  if (!md)
    return MMNB_OK;
  if (md->h && md->h->stream)
    cudaStreamSynchronize(md->h->stream);
  if (md->exec)
    cudaGraphExecDestroy(md->exec);
  if (md->graph)
    cudaGraphDestroy(md->graph);
  void *p[] = {md->d_r, md->d_v, md->d_f, md->d_m, md->d_minv, md->d_energy, md->d_ke_part, md->d_ctl, md->d_log};
  for (void *q : p)
    if (q)
      cudaFree(q);
  delete md;
  return MMNB_OK;
}

int mmnb_md_scale_velocities(mmnb_md *md, double factor)
{
  if (!md)
    return MMNB_ERR_ARG;
  mmnb_handle *h = md->h;
  const int n3 = 3 * md->nsite;
  k_md_scale<<<div_up(n3, 256), 256, 0, h->stream>>>(md->d_v, n3, factor);
  MDCK(cudaGetLastError());
  MDCK(cudaStreamSynchronize(h->stream));
  return MMNB_OK;
}

// ---- replica batch --------------------------------------------------------------

int mmnb_md_batch_create(mmnb_md *const *mds, int n, mmnb_md_batch **out)
{
  if (!out || !mds || n <= 0)
    return MMNB_ERR_ARG;
  *out = nullptr;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < i; j++)
      if (!mds[i] || mds[i] == mds[j] || mds[i]->h == mds[j]->h || mds[i]->h->stream == mds[j]->h->stream)
        return MMNB_ERR_ARG;  // every replica needs its own handle and stream
  mmnb_md_batch *b = new mmnb_md_batch;
  b->md.assign(mds, mds + n);
  if (cudaSetDevice(mds[0]->h->dev) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) {
    mmnb_md_batch_destroy(b);
    return MMNB_ERR_CUDA;
  }
  b->done.resize(n, nullptr);
  for (int i = 0; i < n; i++)
    if (cudaEventCreateWithFlags(&b->done[i], cudaEventDisableTiming) != cudaSuccess) {
      mmnb_md_batch_destroy(b);
      return MMNB_ERR_CUDA;
    }
  *out = b;
  return MMNB_OK;
}

static int batch_fail(mmnb_md_batch *b, int code, const std::string &msg)
{
  b->err = msg;
  return code;
}

// one graph: a fork from the master stream into every replica's stream, each
// replica's step recorded on its own stream, a join back
static int batch_capture(mmnb_md_batch *b)
{
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  cudaError_t e = cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess)
    return batch_fail(b, MMNB_ERR_CUDA, cudaGetErrorString(e));
  int s = MMNB_OK;
  e = cudaEventRecord(b->fork, b->master);
  for (size_t i = 0; i < b->md.size() && e == cudaSuccess && !s; i++) {
    mmnb_md *md = b->md[i];
    mmnb_handle *h = md->h;
    e = cudaStreamWaitEvent(h->stream, b->fork, 0);
    if (e != cudaSuccess)
      break;
    h->capturing = true;
    s = md_record(md, md->d_log);
    h->capturing = false;
    if (s)
      break;
    if ((e = cudaEventRecord(b->done[i], h->stream)) == cudaSuccess)
      e = cudaStreamWaitEvent(b->master, b->done[i], 0);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(b->master, &g);
  if (s || e != cudaSuccess || ec != cudaSuccess) {
    if (g)
      cudaGraphDestroy(g);
    if (s)
      return batch_fail(b, s, "replica step: " + b->md[0]->err);
    return batch_fail(b, MMNB_ERR_CUDA, cudaGetErrorString(e != cudaSuccess ? e : ec));
  }
  b->graph = g;
  e = cudaGraphInstantiate(&b->exec, g, cudaGraphInstantiateFlagUseNodePriority);
  if (e != cudaSuccess)
    return batch_fail(b, MMNB_ERR_CUDA, cudaGetErrorString(e));
  b->gen.clear();
  for (mmnb_md *md : b->md)
    b->gen.push_back(md->h->buf_gen);
  return MMNB_OK;
}

int mmnb_md_batch_run(mmnb_md_batch *b, int nsteps, double *const *energies)
{
  if (!b || nsteps < 0)
    return MMNB_ERR_ARG;
  if (nsteps == 0)
    return MMNB_OK;
  for (mmnb_md *md : b->md) {
    const int cap = md->log_cap;
    if (const int s = md_reserve_log(md, nsteps))
      return batch_fail(b, s, md->err);
    if (md->log_cap != cap && b->exec) {
      cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
    }
  }
  // captured again when a replica handle's buffers were reallocated since
  bool stale = !b->exec || b->gen.size() != b->md.size();
  for (size_t i = 0; !stale && i < b->md.size(); i++)
    stale = b->gen[i] != b->md[i]->h->buf_gen;
  if (stale) {
    if (b->exec) {
      cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
    }
    if (const int s = batch_capture(b))
      return s;
  }
  cudaError_t e = cudaSuccess;
  for (mmnb_md *md : b->md) {
    if (e == cudaSuccess)
      e = cudaMemsetAsync(md->d_ctl + 1, 0, sizeof(unsigned long long), md->h->stream);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(md->h->d_flags + kFlagOverflow, 0, sizeof(int), md->h->stream);
    if (e == cudaSuccess)
      e = cudaEventRecord(md->h->ev_fork, md->h->stream);
    if (e == cudaSuccess)
      e = cudaStreamWaitEvent(b->master, md->h->ev_fork, 0);
  }
  for (int i = 0; i < nsteps && e == cudaSuccess; i++)
    e = cudaGraphLaunch(b->exec, b->master);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(b->master);
  if (e != cudaSuccess)
    return batch_fail(b, MMNB_ERR_CUDA, cudaGetErrorString(e));
  int overflow = 0;
  for (size_t i = 0; i < b->md.size(); i++) {
    mmnb_md *md = b->md[i];
    int flags[kFlagCount];
    e = cudaMemcpy(flags, md->h->d_flags, sizeof(flags), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && energies && energies[i])
      e = cudaMemcpy(energies[i], md->d_log, 3 * (size_t) nsteps * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
      return batch_fail(b, MMNB_ERR_CUDA, cudaGetErrorString(e));
    md->h->evals += nsteps;
    overflow = std::max(overflow, flags[kFlagOverflow]);
  }
  (void) overflow;
  // every replica's status (rows cut at capacity are regrown for the next run)
  int status = MMNB_OK;
  std::string msg;
  for (size_t i = 0; i < b->md.size(); i++) {
    long trunc = 0;
    if (const int st = mmnb_check(b->md[i]->h, &trunc, nullptr)) {
      if (!status) {
        status = st;
        msg = "replica " + std::to_string(i) + " during the run: " + b->md[i]->h->err;
      }
    }
  }
  if (status)
    return batch_fail(b, status, msg);
  return MMNB_OK;
}

const char *mmnb_md_batch_last_error(const mmnb_md_batch *b) { return b ? b->err.c_str() : "null batch"; }

int mmnb_md_batch_destroy(mmnb_md_batch *b)
{
  if (!b)
    return MMNB_OK;
  if (b->master)
    cudaStreamSynchronize(b->master);
  if (b->exec)
    cudaGraphExecDestroy(b->exec);
  if (b->graph)
    cudaGraphDestroy(b->graph);
  for (cudaEvent_t ev : b->done)
    if (ev)
      cudaEventDestroy(ev);
  if (b->fork)
    cudaEventDestroy(b->fork);
  if (b->master)
    cudaStreamDestroy(b->master);
  delete b;
  return MMNB_OK;
}

}  // extern "C"

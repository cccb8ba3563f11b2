// Internal declarations of libmmnb (sm_100a).  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mmnb.h"

namespace mmnb {

constexpr int kCheb = 512;          // Chebyshev segments (include/cheby.h:10)
constexpr int kChebWMax = 2048;     // segments of the rigid-water FP64 kernel's continued table
constexpr int kMaxGroup = 8;        // sites per group handled by the pair kernels
constexpr int kMaxOrder = 7;        // P3M assignment order (src/pppm.c:61)
constexpr int kWarp = 32;

// flag words shared by the list-build kernels (device memory)
enum FlagIndex {
  kFlagRebuild = 0,    // 1 when this evaluation rebuilds the list
  kFlagOverflow = 1,   // largest row length seen when a row overflowed
  kFlagError = 2,      // MMNB_ERR_DEVICE when a device-side check failed
  kFlagMaxRow = 3,     // largest row length of the last build
  // 4: evaluations, 5: rebuilds, 6: the list check's block counter
  kFlagPruneFull = 7,  // 1: the water kernel reads the full rows and writes the pruned ones
  kFlagPruneValid = 8, // 1 while the pruned rows belong to the current build
  kFlagListTrunc = 9,  // 1 while the current list has rows cut at their capacity
  kFlagTruncEvals = 10,// evaluations finished on such a list since the last mmnb_check
  kFlagForceRebuild = 11, // 1: the next list check rebuilds (set by the host, cleared by the check)
  kFlagCount = 12
};

// Box in the form the kernels use (cubic and orthorhombic).
struct Box {
  double L[3];      // edge lengths
  double invL[3];   // 1 / L, as the reference computes it (src/rspace.c:399-404)
};

// Cell-list geometry (src/nbrlist.cpp:9-17, 84-123).
struct CellGeom {
  int n;            // cells per dimension
  double lc[3];     // cell edge = L * (1.0 / n)
  double c2;        // (cutoff + width)^2
};

// Fixed-point scale of the mixed form's accumulators: 2^32 units per unit of
// potential, field or force (range +-2^31, resolution 2.3e-10).
constexpr double kFxScale = 4294967296.0;
constexpr double kFxInv = 1.0 / 4294967296.0;
constexpr int kAccStride = 8;  // phi, Ex, Ey, Ez, Lx, Ly, Lz, (pad) per site

// Launch choices that do not change any result (mmnb_autotune times them).
struct Tuning {
  int water_minb = 5;      // rigid-water pair kernel: 4 or 5 resident warps per SM / 4 (128 or 96 registers)
  int spread_planes = 2;   // mixed P3M spread: 0 one thread per site, 1 P threads per site (x planes),
                           // 2 P lanes per site along z (coalesced reductions)
  int p3m_side = 1;        // P3M mesh work on the side stream (1) or in line (0)
  int water64_warps = 12;  // FP64 rigid-water kernel: warps per block (12, 10 or 8; fewer when the
                           // rings and the table do not fit in shared memory)
};

// Device buffers of the mixed-precision form.
struct MixedBufs {
  float4 *site = nullptr;        // sorted, padded slots: offset from the anchor (xyz), charge (w); or,
                                 // for the rigid-water kernel, three packed slots per group
  float4 *par = nullptr;         // sorted, padded slots: sigma, sqrt(epsilon), rscreen, mask bits
  double4 *anchor = nullptr;     // sorted groups: anchor position (FP64)
  float4 *anc32 = nullptr;       // rigid-water kernel, sorted groups: the anchor's offset from the corner
                                 // of its list cell (FP32) and the cell's coordinates (10 bits each, in w)
  long long *acc = nullptr;      // per site (original order), kAccStride fixed-point values
  long long *acck = nullptr;     // per site (original order): P3M interpolation phi, Ex, Ey, Ez
};

// Stage timing with CUDA events recorded on the handle's stream.  Each
// evaluation starts with a "start" mark; a stage's time is the interval from
// the previous mark to its own.
struct Timing {
  bool on = false;
  std::vector<cudaEvent_t> pool;   // reused between resets
  std::vector<std::string> names;  // one per recorded mark
  size_t used = 0;
};

}  // namespace mmnb

struct mmnb_handle {
  mmnb_config cfg{};
  int nsite = 0, ngroup = 0, maxgs = 1, G = 1;   // G: padded sites per group slot
  int dev = 0;
  cudaStream_t stream = nullptr;       // stream every launch goes to
  cudaStream_t own_stream = nullptr;   // created by mmnb_create, destroyed by mmnb_destroy
  // P3M charge assignment and FFTs run on `side`, forked from and joined back
  // into `stream`, concurrently with the list and pair kernels
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  std::string err;

  // derived settings
  double rc = 0, nlw = 0, eta = 0, rlo2 = 0, rhi2 = 0, inv_sw = 0;  // inv_sw = 1/(rhi2 - rlo2)
  mmnb::Box box{};
  double volume = 0, min_diameter = 0;
  bool params_set = false, any_q = false, any_lj = false, has_rscreen = false;
  bool any_gexcl = false, use_14 = false;
  bool lj_on_anchors_only = false;   // every LJ site is its group's first site (rigid water)
  bool water = false;                // every group is [O(q, LJ), H(q), H(q)] with no screening or group exclusions
  // ... and every O has the same charge, sigma and epsilon and every H the
  // same charge (the rigid-water kernel then copies only the H offsets)
  bool water_uni = false;
  float uni_qO = 0, uni_qH = 0, uni_sig = 0, uni_seps = 0;
  bool want_fields = false;          // this evaluation must produce per-site potential and field
  bool want_virial = false;          // this evaluation's pair kernels also sum the virial's pair term
  bool used_water = false;           // the last evaluation ran the water kernel
  bool used_water64 = false;         // the last evaluation ran the FP64 water kernel
  double totA = 0, totB = 0, lj_correction = 0, neutral_b = 0;

  // host topology
  std::vector<int> group;            // 2*ngroup
  std::vector<int> group_of_site;
  std::vector<int> excl_ptr, excl_idx;   // per-site excluded partners, both directions, sorted
  std::vector<int> p14_ptr, p14_idx;     // per-site 1-4 partners, both directions, sorted
  std::vector<int> gexcl_ptr, gexcl_idx; // per-group group-excluded partners, sorted

  // device topology and parameters (original site order)
  int *d_group = nullptr;
  int *d_excl_ptr = nullptr, *d_excl_idx = nullptr;
  int *d_p14_ptr = nullptr, *d_p14_idx = nullptr;
  int *d_gexcl_ptr = nullptr, *d_gexcl_idx = nullptr;
  int *d_mask = nullptr;
  double *d_q = nullptr, *d_sig = nullptr, *d_eps = nullptr, *d_rscreen = nullptr;
  double *d_cheb = nullptr;          // 512 x 8 doubles (7 used) + nothing else
  double cheb_min = 0, cheb_max = 0, cheb_inv_dx = 0;
  // the rigid-water FP64 kernel's table: cheb_w_nseg x (c0, c1), then x (c2, c3)
  double *d_cheb_w = nullptr;
  int cheb_w_nseg = 0;
  // 512 x 4: the cubics of -eta d/d(eta) of the table (mmnb_virial)
  double *d_cheb_d = nullptr;
  int water64_grid = 0;              // persistent blocks of that kernel (0: not sized yet)
  int water64_warps = 0;             // warps per block of that kernel
  size_t water64_smem = 0;

  // neighbour list
  mmnb::CellGeom cg{};
  int ncell3 = 0;
  int nstencil = 0;                  // offsets incl. (0,0,0) first
  int *d_stencil = nullptr;          // 3 ints per offset
  int *d_cell_rank = nullptr;        // reference cell index -> Morton rank
  int *d_cell_of_rank = nullptr;     // Morton rank -> reference cell index
  int *d_cell_of_group = nullptr;    // per group, reference numbering
  int *d_cell_count = nullptr;       // per rank
  int *d_cell_start = nullptr;       // per rank, ncell3+1
  int *d_slot = nullptr;             // per group, slot inside its cell
  int *d_sorted = nullptr;           // sorted position -> group
  int *d_rank = nullptr;             // group -> sorted position
  double *d_anchor = nullptr;        // 3*ngroup current anchors (original order)
  double *d_last = nullptr;          // 3*ngroup anchors at the last rebuild
  double *d_anchor_sorted = nullptr; // 3*ngroup anchors at the last rebuild, sorted order
  float4 *d_anchor32 = nullptr;      // the same, wrapped into the box, FP32 (list pre-test)
  double *d_top2 = nullptr;          // per-block top-2 displacements
  int top2_blocks = 0;
  int rebuild_grid = 0;              // blocks of the cooperative rebuild launch (0: not sized yet)
  int *d_block_sum = nullptr;        // per rebuild block: its segment's cell count
  int block_sum_cap = 0;
  int rowcap = 0;
  int *d_nbr = nullptr;              // ngroup * rowcap, sorted positions
  int *d_nbr_count = nullptr;        // ngroup
  // rows pruned to rc + prune_margin for the rigid-water kernel (same rowcap),
  // and the sorted anchors at the last prune
  int *d_pnbr = nullptr, *d_pcount = nullptr;
  double *d_plast = nullptr;
  double prune_margin = 0;           // 0: no pruning
  int *d_flags = nullptr;            // mmnb::kFlagCount ints
  // bumped by every (re)allocation of a device buffer: a captured graph holds
  // the addresses of its launch, so it is replayed only while this is unchanged
  long buf_gen = 0;
  long graph_gen = -1;               // buf_gen when mmnb_graph_capture ran
  int *h_flags = nullptr;            // pinned mirror
  long rebuilds = 0, evals = 0;
  long launches = 0;                 // kernels of this library launched so far
  long launch_per_eval = 0;          // kernels in the captured evaluation
  bool first = true;
  int force_rebuild_next = 0;

  // sorted, padded site data (FP64 form)
  double4 *d_sr = nullptr;           // ngroup*G sites: x, y, z, q
  double4 *d_sp = nullptr;           // sig, eps, rscreen, (mask as double)
  int *d_site_of_slot = nullptr;     // ngroup*G -> original site (or -1)

  // outputs (original order)
  double *d_phi = nullptr, *d_evec = nullptr, *d_ljf = nullptr;
  double *d_lj_part = nullptr;       // LJ energy partials: pair-kernel blocks, then exclusion blocks
  double *d_lj_row = nullptr;        // FP64 water kernel: LJ energy of each row (sorted order)
  double *d_lj_row_part = nullptr;   // finalize: per block, its slice of d_lj_row
  // mmnb_virial: the pair kernels' virial term (per block: pair-kernel blocks,
  // then exclusion blocks; per row: FP64 water kernel), molecule ranges,
  // masses and per-molecule sums (allocated on first use)
  double *d_vir_part = nullptr, *d_vir_row = nullptr;
  int *d_vir_mol = nullptr;
  double *d_vir_molw = nullptr, *d_vir_mass = nullptr;
  int vir_mol_cap = 0;
  // [0], [1]: fixed-point Coulomb and LJ pair energies of the water kernel;
  // [2]: block counter of the finalize kernel's last-block reduction;
  // [3]: row counter of the FP64 water kernel; [4]: the mixed water kernel's
  // fixed-point virial term
  unsigned long long *d_wsum = nullptr;
  // parameter gradients (allocated on first use): six per-site outputs, dL/dF,
  // the dipole structure factor of the reciprocal sum
  double *d_bwd = nullptr;
  size_t bwd_cap = 0;
  double *h_bwd = nullptr;  // pinned: the gradient slots come back in one copy
  bool grad_ready = false;           // the last evaluation was mmnb_forward's and nothing changed since
  // FP64 dipole solve for a mixed-form handle, which has no FP64 meshes or plans
  double *d_gmesh = nullptr;
  cufftDoubleComplex *d_gmeshk = nullptr;
  cufftHandle gplan_r2c = 0, gplan_c2r = 0;
  // host copies of the site parameters, and the LJ classes of the tail:
  // distinct (sigma, epsilon) as printed with %12.6g, their site counts, and
  // each site's class (-1 without LJ)
  std::vector<double> hq, hsig, heps;
  std::vector<double> cls_sig, cls_eps;
  std::vector<long> cls_n;
  std::vector<int> site_cls;
  int lj_pair_blocks = 0, lj_excl_blocks = 0;
  double *d_elec_part = nullptr;     // per block
  int elec_blocks = 0;
  double *d_energy = nullptr;        // 4 doubles
  // host path staging
  double *d_r = nullptr, *d_f = nullptr;
  double *h_r = nullptr, *h_f = nullptr, *h_out = nullptr;  // pinned

  // P3M
  bool p3m = false;
  int mesh[3] = {0, 0, 0};
  cufftHandle plan_r2c = 0, plan_c2r = 0;
  double *d_mesh = nullptr;
  cufftDoubleComplex *d_meshk = nullptr;
  double *d_green = nullptr;         // nx*ny*(nz/2+1)
  double *d_kvec = nullptr;          // 3 per k-point (ik differentiation)
  double *d_egrid = nullptr;         // 3 real meshes (ik)
  cufftDoubleComplex *d_egridk = nullptr;
  double *d_chi_part = nullptr;      // per-block partials of the mesh error sum
  double p3m_chi = 0;                // the mesh's dimensionless RMS force error estimate
  bool eta_optimised = false;        // eta chosen by p3m_optimize's criterion
  // mixed-precision P3M
  cufftHandle plan_r2c32 = 0, plan_c2r32 = 0;
  float *d_mesh32 = nullptr;
  cufftComplex *d_meshk32 = nullptr;
  float *d_green32 = nullptr;
  float *d_egrid32 = nullptr;        // ik differentiation: three FP32 field meshes
  cufftComplex *d_egridk32 = nullptr;
  unsigned long long *d_mesh_fx = nullptr;

  // ordinary Ewald
  bool kspace = false;
  int nk = 0, kmax = 0;
  int *d_kint = nullptr;             // 3 per k
  double *d_kvecs = nullptr;         // 3 per k
  double *d_ak = nullptr;
  double *d_skc = nullptr;           // 2 per k: sum q cos, sum q sin

  // mixed form
  mmnb::MixedBufs mx;

  mmnb::Timing timing;
  mmnb::Tuning tune;

  // one captured evaluation (mmnb_graph_capture / mmnb_graph_launch)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  // the host call's own graph (d_r -> d_f, d_energy), captured on first use
  // and dropped whenever rows, parameters, box or stream change
  cudaGraph_t hgraph = nullptr;
  cudaGraphExec_t hgraph_exec = nullptr;
  long host_launch_per_eval = 0;
  // the host call copies the forces back in chunks and adds each as it lands
  static constexpr int kChunks = 2;
  cudaEvent_t ev_chunk[kChunks] = {};
  cudaEvent_t ev_eval = nullptr;  // the host call's evaluation has ended (or failed)
  // ... and, replaying its graph, copies the positions in kInChunks pieces on
  // a stream of its own: the graph's mesh branch assigns the charges of each
  // piece as it lands (mixed form), everything else waits for the last piece
  static constexpr int kInChunks = 2;
  cudaStream_t copy_in = nullptr;
  cudaEvent_t ev_in[kInChunks] = {};
  cudaEvent_t ev_free = nullptr;  // the handle's stream has let go of d_r
  bool in_chunks = false;         // set while that graph is captured
  // the host call's status block in mapped pinned memory: k_finalize writes
  // the energies [0, 4), the flags (ints, from double 4 on) and then, after a
  // system-wide fence, the ready word; the host spins on that word instead of
  // copying the block back after the evaluation
  static constexpr int kStatusDoubles = 16;
  static constexpr int kStatusReady = 15;  // double slot of the ready word
  double *h_status = nullptr;
  double *d_status = nullptr;  // its device alias
  bool want_status = false;    // set while the host call records its evaluation: no
                               // other evaluation writes the block
  bool capturing = false;
};

namespace mmnb {

// ---- launchers (defined in the .cu files) ----------------------------------
// drop the host call's graph (called when what it captured changes)
void drop_host_graph(mmnb_handle *h);
// LJ tail correction (src/eleclj.cpp:1247-1266) for totals A and B; linear in both
double lj_tail_ab(const mmnb_handle *h, double A, double B);
// anchors, rebuild decision; then the rebuild (a no-op launch when not due)
cudaError_t launch_list_check(mmnb_handle *h, const double *d_r, int force);
cudaError_t launch_list_rebuild(mmnb_handle *h);
cudaError_t launch_sort_sites(mmnb_handle *h, const double *d_r);
cudaError_t launch_rspace_fp64(mmnb_handle *h);
cudaError_t launch_prep_mixed(mmnb_handle *h, const double *d_r);
cudaError_t launch_rspace_mixed(mmnb_handle *h);
cudaError_t launch_rspace_water(mmnb_handle *h);
cudaError_t launch_sort_water64(mmnb_handle *h, const double *d_r);
cudaError_t launch_rspace_water64(mmnb_handle *h);
cudaError_t launch_exclusions(mmnb_handle *h, const double *d_r);
cudaError_t launch_p3m_green(mmnb_handle *h, double eta, double *chi);
// stage bit 1: spread + FFT round trip, bit 2: gather
cudaError_t launch_p3m_fp64(mmnb_handle *h, const double *d_r, int stage);
// FP64 meshes and plans of the adjoint's dipole solve: spread/spreadk hold one
// mesh (three with ik differentiation); solvek/solve the summed ik spectrum
// and its transform (ik only; otherwise the solve happens in place)
struct P3mScratch {
  double *spread = nullptr, *solve = nullptr;
  cufftDoubleComplex *spreadk = nullptr, *solvek = nullptr;
  cufftHandle r2c = 0, c2r = 0;
};
// d_psi += mesh potential of the dipoles q_j g_j (g: 3 per site), FP64
cudaError_t launch_p3m_dipole_fp64(mmnb_handle *h, const double *d_r, const double *d_g, const P3mScratch &s,
                                   double *d_psi);
// d_psi += reciprocal-sum potential of the dipoles q_j g_j; d_skd: 2 per k
cudaError_t launch_kspace_dipole(mmnb_handle *h, const double *d_r, const double *d_g, double *d_skd,
                                 double *d_psi);
cudaError_t launch_p3m_mixed(mmnb_handle *h, const double *d_r, int stage);
// write back and drop [p, p + bytes) from the host cores' caches (hostmem.cpp)
void evict_host_lines(const void *p, size_t bytes);

// the mixed charge assignment of sites [lo, hi) alone; stage bit 4 of
// launch_p3m_mixed then skips it (the mesh words are integer sums, so the
// pieces give the mesh of one launch over all sites, bit for bit)
cudaError_t launch_spread_mixed_range(mmnb_handle *h, const double *d_r, int lo, int hi);
cudaError_t launch_green32(mmnb_handle *h);
cudaError_t launch_kspace(mmnb_handle *h, const double *d_r);
cudaError_t launch_finalize(mmnb_handle *h, double *d_f, double *d_energy);
cudaError_t launch_energy(mmnb_handle *h, double *d_energy);

// helpers shared by the .cu files
void timing_mark(mmnb_handle *h, const char *name);
int set_global_error(int code, const std::string &msg);  // read back by mmnb_last_error(NULL)
int pair_blocks(const mmnb_handle *h);
int excl_blocks(const mmnb_handle *h);

#ifdef __CUDACC__
// binary search of key in CSR row `row` (sorted)
__device__ __forceinline__ bool csr_has(const int *ptr, const int *idx, int row, int key)
{
  int lo = ptr[row], hi = ptr[row + 1] - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int v = idx[mid];
    if (key < v)
      hi = mid - 1;
    else if (key > v)
      lo = mid + 1;
    else
      return true;
  }
  return false;
}

// b0 = erfc(eta r)/r, b1 = (b0 + 2 eta/sqrt(pi) exp(-eta^2 r^2)) / r^2 from the
// reference's 512-segment Chebyshev table (8 doubles per segment) inside
// (cmin, cmax), from erfc/exp outside it; seg and f: the table segment and the
// position in it (seg = -1 outside the table)
__device__ __forceinline__ void ewald_table_b(const double *cheb, double cmin, double cmax, double inv_dx,
                                              double eta, double r2, double &b0, double &b1, int &seg, double &f)
{
  if (cmin < r2 && r2 < cmax) {
    double x = (r2 - cmin) * inv_dx;
    const unsigned i = (unsigned) x;
    const double2 *c = reinterpret_cast<const double2 *>(cheb + 8 * (size_t) i);
    const double2 c01 = __ldg(c), c23 = __ldg(c + 1), c45 = __ldg(c + 2), c67 = __ldg(c + 3);
    x -= i;
    b0 = ((c23.y * x + c23.x) * x + c01.y) * x + c01.x;
    b1 = (c67.x * x + c45.y) * x + c45.x;
    seg = (int) i;
    f = x;
  } else {
    const double r = sqrt(r2);
    const double er = eta * r;
    const double e = exp(-(er * er));
    b0 = erfc(er) / r;
    b1 = (b0 + eta * M_2_SQRTPI * e) / r2;
    seg = -1;
    f = 0;
  }
}

// The same from the cubic alone: t0[i] = (c0, c1), t1[i] = (c2, c3) of segment i
// (the rigid-water kernels' copy of the table, whose first 512 segments are the
// reference's), b1 from the cubic's derivative -- the reference stores b1's
// quadratic as exactly -2 k c_k / dx (k = 1..3), so the two differ only in
// rounding.  Same range, segment and position as ewald_table_b; half the reads.
__device__ __forceinline__ void ewald_table_half(const double2 *t0, const double2 *t1, double cmin, double cmax,
                                                 double inv_dx, double eta, double r2, double &b0, double &b1,
                                                 int &seg, double &f)
{
  if (cmin < r2 && r2 < cmax) {
    double x = (r2 - cmin) * inv_dx;
    const unsigned i = (unsigned) x;
    const double2 c01 = __ldg(t0 + i), c23 = __ldg(t1 + i);
    x -= i;
    b0 = ((c23.y * x + c23.x) * x + c01.y) * x + c01.x;
    b1 = -2 * inv_dx * ((3 * c23.y * x + 2 * c23.x) * x + c01.y);
    seg = (int) i;
    f = x;
  } else {
    const double r = sqrt(r2);
    const double er = eta * r;
    const double e = exp(-(er * er));
    b0 = erfc(er) / r;
    b1 = (b0 + eta * M_2_SQRTPI * e) / r2;
    seg = -1;
    f = 0;
  }
}

// minimum image of one site displacement, rounded as the reference rounds it
__device__ __forceinline__ void min_image_ref(const Box &b, double &x, double &y, double &z)
{
  x = __dadd_rn(x, __dmul_rn(-b.L[0], floor(__dadd_rn(__dmul_rn(x, b.invL[0]), 0.5))));
  y = __dadd_rn(y, __dmul_rn(-b.L[1], floor(__dadd_rn(__dmul_rn(y, b.invL[1]), 0.5))));
  z = __dadd_rn(z, __dmul_rn(-b.L[2], floor(__dadd_rn(__dmul_rn(z, b.invL[2]), 0.5))));
}

// anchor displacement with the reference's minimum-image rounding
__device__ __forceinline__ double anchor_disp(const Box &b, double4 ri, double4 rj, double &x, double &y, double &z,
                                              double &sx, double &sy, double &sz)
{
  x = __dsub_rn(ri.x, rj.x);
  y = __dsub_rn(ri.y, rj.y);
  z = __dsub_rn(ri.z, rj.z);
  sx = __dmul_rn(-b.L[0], floor(__dadd_rn(__dmul_rn(x, b.invL[0]), 0.5)));
  sy = __dmul_rn(-b.L[1], floor(__dadd_rn(__dmul_rn(y, b.invL[1]), 0.5)));
  sz = __dmul_rn(-b.L[2], floor(__dadd_rn(__dmul_rn(z, b.invL[2]), 0.5)));
  x = __dadd_rn(x, sx);
  y = __dadd_rn(y, sy);
  z = __dadd_rn(z, sz);
  return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

#endif

inline int div_up(long a, long b) { return (int) ((a + b - 1) / b); }

}  // namespace mmnb

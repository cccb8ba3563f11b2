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
constexpr int kMaxGroup = 8;        // sites per group handled by the pair kernels
constexpr int kMaxOrder = 7;        // P3M assignment order (src/pppm.c:61)
constexpr int kWarp = 32;

// flag words shared by the list-build kernels (device memory)
enum FlagIndex {
  kFlagRebuild = 0,    // 1 when this evaluation rebuilds the list
  kFlagOverflow = 1,   // largest row length seen when a row overflowed
  kFlagError = 2,      // MMNB_ERR_DEVICE when a device-side check failed
  kFlagMaxRow = 3,     // largest row length of the last build
  kFlagCount = 8
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

// Device buffers of the mixed-precision form.
struct MixedBufs {
  float4 *site_xyzq = nullptr;   // sorted, padded: offset from anchor (xyz) + charge (w)
  float2 *site_lj = nullptr;     // sorted, padded: sigma, sqrt(epsilon)
  int *site_mask = nullptr;      // sorted, padded
  double *anchor = nullptr;      // sorted anchors (3 per group), wrapped into the box
  long long *acc = nullptr;      // fixed-point accumulators: per sorted site 7 values
  float *cheb32 = nullptr;       // unused placeholder for an FP32 table
  int *mesh_fx = nullptr;        // unused
};

struct Timing {
  bool on = false;
  std::vector<cudaEvent_t> ev;
  std::vector<std::string> names;
  std::vector<double> ms;
};

}  // namespace mmnb

struct mmnb_handle {
  mmnb_config cfg{};
  int nsite = 0, ngroup = 0, maxgs = 1, G = 1;   // G: padded sites per group slot
  int dev = 0;
  cudaStream_t stream = nullptr;
  std::string err;

  // derived settings
  double rc = 0, nlw = 0, eta = 0, rlo2 = 0, rhi2 = 0;
  mmnb::Box box{};
  double volume = 0, min_diameter = 0;
  bool params_set = false, any_q = false, any_lj = false, has_rscreen = false;
  bool any_gexcl = false, use_14 = false;
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
  double *d_top2 = nullptr;          // per-block top-2 displacements
  int top2_blocks = 0;
  int rowcap = 0;
  int *d_nbr = nullptr;              // ngroup * rowcap, sorted positions
  int *d_nbr_count = nullptr;        // ngroup
  int *d_flags = nullptr;            // mmnb::kFlagCount ints
  int *h_flags = nullptr;            // pinned mirror
  long rebuilds = 0, evals = 0;
  bool first = true;
  int force_rebuild_next = 0;

  // sorted, padded site data (FP64 form)
  double4 *d_sr = nullptr;           // ngroup*G sites: x, y, z, q
  double4 *d_sp = nullptr;           // sig, eps, rscreen, (mask as double)
  int *d_site_of_slot = nullptr;     // ngroup*G -> original site (or -1)

  // outputs (original order)
  double *d_phi = nullptr, *d_evec = nullptr, *d_ljf = nullptr;
  double *d_lj_part = nullptr;       // per sorted group LJ energy
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
  double p3m_chi = 0;
  // mixed-precision P3M
  cufftHandle plan_r2c32 = 0, plan_c2r32 = 0;
  float *d_mesh32 = nullptr;
  cufftComplex *d_meshk32 = nullptr;
  float *d_green32 = nullptr;
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
};

namespace mmnb {

// ---- launchers (defined in the .cu files) ----------------------------------
cudaError_t launch_gather_anchors(mmnb_handle *h, const double *d_r);
cudaError_t launch_rebuild_decide(mmnb_handle *h, int force);
cudaError_t launch_build_list(mmnb_handle *h);
cudaError_t launch_sort_sites(mmnb_handle *h, const double *d_r);
cudaError_t launch_rspace_fp64(mmnb_handle *h);
cudaError_t launch_rspace_mixed(mmnb_handle *h, const double *d_r);
cudaError_t launch_exclusions(mmnb_handle *h, const double *d_r);
cudaError_t launch_p3m_green(mmnb_handle *h);
cudaError_t launch_p3m_fp64(mmnb_handle *h, const double *d_r);
cudaError_t launch_p3m_mixed(mmnb_handle *h, const double *d_r);
cudaError_t launch_kspace(mmnb_handle *h, const double *d_r);
cudaError_t launch_finalize(mmnb_handle *h, double *d_f, double *d_energy);

// helpers shared by the .cu files
void timing_mark(mmnb_handle *h, const char *name);

inline int div_up(long a, long b) { return (int) ((a + b - 1) / b); }

}  // namespace mmnb

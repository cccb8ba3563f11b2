// Cell neighbour list on the GPU: rebuild trigger, cell assignment, Morton
// counting sort and warp-ballot list build.
//
// Semantics follow the reference's NeighborList exactly (src/nbrlist.cpp):
//   * a rebuild happens on the first evaluation and whenever the two largest
//     anchor moves since the last build add up to more than the skin
//     (coordinates_changed, :51-77);
//   * a group's cell is round(x / l_cell) mod n per axis with
//     l_cell = L * (1.0 / n) (rebuild_periodic :228-234, Cubic/Orthorhombic
//     nearest_lattice_point src/bcond.cpp:31-34, include/pbc.h:25-31, 52-59);
//   * groups in the same cell are paired unconditionally (:243-244);
//   * groups in cells joined by the reference's cell stencil are paired when
//     their minimum-image distance squared is below (cutoff + width)^2
//     (:245-248, include/bcond.hpp:56-60).
// The arithmetic that decides membership (cell index, squared distance,
// displacement test) uses explicitly rounded FP64 operations so it cannot be
// contracted into FMAs: it is the same IEEE sequence the reference executes,
// and the pair set is identical, not merely close.
//
// The list is stored FULL (each unordered pair in both rows) so the pair
// kernels accumulate on their own rows only, without atomics.  Rows are
// indexed by sorted position (groups ordered by the Morton rank of their cell).

#include <cooperative_groups.h>

#include "mmnb_internal.cuh"

namespace mmnb {

__device__ __forceinline__ double exact_wrap(double x, double L, double invL)
{
  // x - L * floor(x * (1/L) + 0.5)   (include/pbc.h:8-14)
  return __dsub_rn(x, __dmul_rn(L, floor(__dadd_rn(__dmul_rn(x, invL), 0.5))));
}

__device__ __forceinline__ double exact_sq3(double x, double y, double z)
{
  return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

// merge two (largest, second largest) pairs of a multiset
__device__ __forceinline__ void top2_merge(double &a, double &b, double a2, double b2)
{
  const double hi = fmax(a, a2), lo = fmin(a, a2);
  b = fmax(lo, fmax(b, b2));
  a = hi;
}

constexpr int kCheckThreads = 256;

__device__ __forceinline__ void block_top2(double &a, double &b, double *sa, double *sb)
{
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      double x = sa[threadIdx.x], y = sb[threadIdx.x];
      top2_merge(x, y, sa[threadIdx.x + s], sb[threadIdx.x + s]);
      sa[threadIdx.x] = x;
      sb[threadIdx.x] = y;
    }
    __syncthreads();
  }
  a = sa[0];
  b = sb[0];
}

// Anchors of this evaluation, the two largest anchor moves since the last
// build, and the rebuild decision (first || forced || largest + second >
// width || fixed interval), all in one launch: each block reduces its share,
// the last block to finish merges the block results.  On a rebuild the last
// block also clears the cell counts for the rebuild kernel.
// flags[4] counts evaluations, flags[5] rebuilds, flags[6] is the block counter.
__global__ void __launch_bounds__(kCheckThreads) k_list_check(const double *__restrict__ r,
                                                              const int *__restrict__ group, int ngroup,
                                                              const double *__restrict__ last, double width,
                                                              int first, int force, int interval,
                                                              double *__restrict__ anchor,
                                                              double *__restrict__ partial, int *__restrict__ flags,
                                                              int *__restrict__ cell_count, int ncell3)
{
  __shared__ double sa[kCheckThreads], sb[kCheckThreads];
  __shared__ bool last_block;
  double a = 0, b = 0;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngroup; g += gridDim.x * blockDim.x) {
    const int s0 = group[2 * g];
    const double x = r[3 * s0], y = r[3 * s0 + 1], z = r[3 * s0 + 2];
    anchor[3 * g] = x;
    anchor[3 * g + 1] = y;
    anchor[3 * g + 2] = z;
    const double dx = __dsub_rn(x, last[3 * g]);
    const double dy = __dsub_rn(y, last[3 * g + 1]);
    const double dz = __dsub_rn(z, last[3 * g + 2]);
    const double d = __dsqrt_rn(exact_sq3(dx, dy, dz));
    if (d > a) {
      b = a;
      a = d;
    } else if (d > b) {
      b = d;
    }
  }
  block_top2(a, b, sa, sb);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = a;
    partial[2 * blockIdx.x + 1] = b;
    __threadfence();
    last_block = atomicAdd(flags + 6, 1) == (int) gridDim.x - 1;
  }
  __syncthreads();
  if (!last_block)
    return;
  __threadfence();
  a = b = 0;
  for (int i = threadIdx.x; i < (int) gridDim.x; i += blockDim.x)
    top2_merge(a, b, partial[2 * i], partial[2 * i + 1]);
  block_top2(a, b, sa, sb);
  __shared__ int rebuild_s;
  if (threadIdx.x == 0) {
    const int count = flags[4];
    int rebuild = first || force || (__dadd_rn(b, a) > width);
    if (interval > 0 && count % interval == 0)
      rebuild = 1;
    flags[kFlagRebuild] = rebuild;
    flags[4] = count + 1;
    if (rebuild)
      flags[5] += 1;  // rebuild counter
    flags[6] = 0;
    rebuild_s = rebuild;
  }
  __syncthreads();
  if (rebuild_s)
    for (int c = threadIdx.x; c < ncell3; c += blockDim.x)
      cell_count[c] = 0;
}

struct RebuildArgs {
  int ngroup, ncell3, nstencil, rowcap;
  CellGeom cg;
  Box box;
  const double *anchor;      // this evaluation's anchors (original order)
  const int *cell_rank;      // reference cell index -> Morton rank
  const int *stencil;        // 3 per offset, components in [0, n)
  int *flags;
  int *cell_of_group, *cell_count, *slot, *start, *sorted, *rank;
  double *last, *anchor_sorted;
  int *nbr, *nbr_count;
};

constexpr int kRebuildThreads = 256;
constexpr int kBuildWarps = kRebuildThreads / 32;

// cell = round(x / l_cell) mod n per axis; the anchors become the new "last"
__device__ __forceinline__ void cell_assign(const RebuildArgs &a, int g)
{
  const int n = a.cg.n;
  int ijk[3];
  for (int d = 0; d < 3; d++) {
    const double x = a.anchor[3 * g + d];
    ijk[d] = (int) floor(__dadd_rn(__ddiv_rn(x, a.cg.lc[d]), 0.5));
    ijk[d] %= n;
    if (ijk[d] < 0)
      ijk[d] += n;
    a.last[3 * g + d] = x;
  }
  const int c = (ijk[0] * n + ijk[1]) * n + ijk[2];
  a.cell_of_group[g] = c;
  a.slot[g] = atomicAdd(&a.cell_count[a.cell_rank[c]], 1);
}

// exclusive scan of the per-rank counts by one block
__device__ void scan_cells(const RebuildArgs &a, int *part)
{
  const int nt = blockDim.x;
  const int per = (a.ncell3 + nt - 1) / nt;
  const int beg = threadIdx.x * per;
  const int end = min(beg + per, a.ncell3);
  int s = 0;
  for (int i = beg; i < end; i++)
    s += a.cell_count[i];
  part[threadIdx.x] = s;
  __syncthreads();
  // Hillis-Steele inclusive scan of the partial sums
  for (int off = 1; off < nt; off <<= 1) {
    const int v = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = threadIdx.x > 0 ? part[threadIdx.x - 1] : 0;
  for (int i = beg; i < end; i++) {
    a.start[i] = run;
    run += a.cell_count[i];
  }
  if (threadIdx.x == nt - 1)
    a.start[a.ncell3] = part[nt - 1];
}

// order a cell's members by group index (deterministic lists), then record
// sorted positions and the anchors the list is built from
__device__ __forceinline__ void cell_finish(const RebuildArgs &a, int c)
{
  const int b = a.start[c], e = a.start[c + 1];
  for (int i = b + 1; i < e; i++) {
    const int v = a.sorted[i];
    int j = i - 1;
    while (j >= b && a.sorted[j] > v) {
      a.sorted[j + 1] = a.sorted[j];
      j--;
    }
    a.sorted[j + 1] = v;
  }
  for (int i = b; i < e; i++) {
    const int g = a.sorted[i];
    a.rank[g] = i;
    a.anchor_sorted[3 * i] = a.last[3 * g];
    a.anchor_sorted[3 * i + 1] = a.last[3 * g + 1];
    a.anchor_sorted[3 * i + 2] = a.last[3 * g + 2];
  }
}

// one warp per sorted group; lanes walk stencil cells, members are compacted
// into the row with a ballot
__device__ __forceinline__ void build_row(const RebuildArgs &a, int p, int lane)
{
  const int n = a.cg.n;
  const int gi = a.sorted[p];
  const int ci = a.cell_of_group[gi];
  const int ix = ci / (n * n), iy = (ci / n) % n, iz = ci % n;
  const double xi = a.anchor_sorted[3 * p], yi = a.anchor_sorted[3 * p + 1], zi = a.anchor_sorted[3 * p + 2];
  int *row = a.nbr + (size_t) p * a.rowcap;
  const unsigned below = (1u << lane) - 1;
  int count = 0;
  for (int s0 = 0; s0 < a.nstencil; s0 += 32) {
    const int s = s0 + lane;
    int beg = 0, end = 0;
    if (s < a.nstencil) {
      const int jx = (ix + a.stencil[3 * s]) % n;
      const int jy = (iy + a.stencil[3 * s + 1]) % n;
      const int jz = (iz + a.stencil[3 * s + 2]) % n;
      const int rj = a.cell_rank[(jx * n + jy) * n + jz];
      beg = a.start[rj];
      end = a.start[rj + 1];
    }
    const bool same = (s == 0);
    for (int m = 0;; m++) {
      const int q = beg + m;
      const bool has = q < end;
      if (!__any_sync(0xffffffffu, has))
        break;
      bool take = false;
      if (has && q != p) {
        if (same) {
          take = true;
        } else {
          const double dx = exact_wrap(__dsub_rn(xi, a.anchor_sorted[3 * q]), a.box.L[0], a.box.invL[0]);
          const double dy = exact_wrap(__dsub_rn(yi, a.anchor_sorted[3 * q + 1]), a.box.L[1], a.box.invL[1]);
          const double dz = exact_wrap(__dsub_rn(zi, a.anchor_sorted[3 * q + 2]), a.box.L[2], a.box.invL[2]);
          take = exact_sq3(dx, dy, dz) < a.cg.c2;
        }
      }
      const unsigned bal = __ballot_sync(0xffffffffu, take);
      if (take) {
        const int idx = count + __popc(bal & below);
        if (idx < a.rowcap)
          row[idx] = q;
      }
      count += __popc(bal);
    }
  }
  if (lane == 0) {
    a.nbr_count[p] = min(count, a.rowcap);
    if (count > a.rowcap)
      atomicMax(&a.flags[kFlagOverflow], count);
    atomicMax(&a.flags[kFlagMaxRow], count);
  }
}

// The whole rebuild in one cooperative launch: cell assignment, counting-sort
// scan, scatter, per-cell ordering, list rows, separated by grid-wide
// barriers.  Without a rebuild due every block returns at once (the decision
// is read from device memory, so the launch sits in a CUDA graph unchanged).
__global__ void __launch_bounds__(kRebuildThreads) k_list_rebuild(RebuildArgs a)
{
  if (!a.flags[kFlagRebuild])
    return;
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  __shared__ int part[kRebuildThreads];
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (int g = tid; g < a.ngroup; g += nth)
    cell_assign(a, g);
  grid.sync();
  if (blockIdx.x == 0)
    scan_cells(a, part);
  grid.sync();
  for (int g = tid; g < a.ngroup; g += nth)
    a.sorted[a.start[a.cell_rank[a.cell_of_group[g]]] + a.slot[g]] = g;
  grid.sync();
  for (int c = tid; c < a.ncell3; c += nth)
    cell_finish(a, c);
  grid.sync();
  const int lane = threadIdx.x & 31;
  for (int p = tid >> 5; p < a.ngroup; p += nth >> 5)
    build_row(a, p, lane);
}

cudaError_t launch_list_check(mmnb_handle *h, const double *d_r, int force)
{
  k_list_check<<<h->top2_blocks, kCheckThreads, 0, h->stream>>>(
      d_r, h->d_group, h->ngroup, h->d_last, h->nlw, h->first ? 1 : 0, force, h->cfg.rebuild_interval, h->d_anchor,
      h->d_top2, h->d_flags, h->d_cell_count, h->ncell3);
  h->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_list_rebuild(mmnb_handle *h)
{
  if (h->rebuild_grid == 0) {
    int per_sm = 0, nsm = 0;
    cudaError_t e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_list_rebuild, kRebuildThreads, 0)) !=
            cudaSuccess ||
        (e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->dev)) != cudaSuccess)
      return e;
    if (per_sm < 1)
      return cudaErrorLaunchOutOfResources;
    h->rebuild_grid = std::min(per_sm * nsm, div_up(h->ngroup, kBuildWarps));
  }
  RebuildArgs a;
  a.ngroup = h->ngroup;
  a.ncell3 = h->ncell3;
  a.nstencil = h->nstencil;
  a.rowcap = h->rowcap;
  a.cg = h->cg;
  a.box = h->box;
  a.anchor = h->d_anchor;
  a.cell_rank = h->d_cell_rank;
  a.stencil = h->d_stencil;
  a.flags = h->d_flags;
  a.cell_of_group = h->d_cell_of_group;
  a.cell_count = h->d_cell_count;
  a.slot = h->d_slot;
  a.start = h->d_cell_start;
  a.sorted = h->d_sorted;
  a.rank = h->d_rank;
  a.last = h->d_last;
  a.anchor_sorted = h->d_anchor_sorted;
  a.nbr = h->d_nbr;
  a.nbr_count = h->d_nbr_count;
  void *args[] = {&a};
  h->launches += 1;
  return cudaLaunchCooperativeKernel((const void *) k_list_rebuild, dim3(h->rebuild_grid), dim3(kRebuildThreads),
                                     args, 0, h->stream);
}

}  // namespace mmnb

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

__global__ void k_gather_anchors(const double *__restrict__ r, const int *__restrict__ group, int ngroup,
                                 double *__restrict__ anchor)
{
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroup)
    return;
  const int a = group[2 * g];
  anchor[3 * g] = r[3 * a];
  anchor[3 * g + 1] = r[3 * a + 1];
  anchor[3 * g + 2] = r[3 * a + 2];
}

// merge two (largest, second largest) pairs of a multiset
__device__ __forceinline__ void top2_merge(double &a, double &b, double a2, double b2)
{
  const double hi = fmax(a, a2), lo = fmin(a, a2);
  b = fmax(lo, fmax(b, b2));
  a = hi;
}

constexpr int kTop2Threads = 256;

__global__ void k_top2(const double *__restrict__ anchor, const double *__restrict__ last, int n,
                       double *__restrict__ partial)
{
  __shared__ double sa[kTop2Threads], sb[kTop2Threads];
  double a = 0, b = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double dx = __dsub_rn(anchor[3 * i], last[3 * i]);
    const double dy = __dsub_rn(anchor[3 * i + 1], last[3 * i + 1]);
    const double dz = __dsub_rn(anchor[3 * i + 2], last[3 * i + 2]);
    const double d = __dsqrt_rn(exact_sq3(dx, dy, dz));
    if (d > a) {
      b = a;
      a = d;
    } else if (d > b) {
      b = d;
    }
  }
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
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = sa[0];
    partial[2 * blockIdx.x + 1] = sb[0];
  }
}

// flags[kFlagRebuild] = first || forced || largest + second > width.
// flags[4] counts evaluations for the fixed-interval mode.
__global__ void k_decide(const double *__restrict__ partial, int nblocks, double width, int first,
                         int force, int interval, int *__restrict__ flags)
{
  __shared__ double sa[kTop2Threads], sb[kTop2Threads];
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x)
    top2_merge(a, b, partial[2 * i], partial[2 * i + 1]);
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
  if (threadIdx.x == 0) {
    const int count = flags[4];
    int rebuild = first || force || (__dadd_rn(sb[0], sa[0]) > width);
    if (interval > 0 && count % interval == 0)
      rebuild = 1;
    flags[kFlagRebuild] = rebuild;
    flags[4] = count + 1;
    if (rebuild)
      flags[5] += 1;  // rebuild counter
  }
}

__global__ void k_cell_assign(const double *__restrict__ anchor, int ngroup, CellGeom cg,
                              const int *__restrict__ cell_rank, const int *__restrict__ flags,
                              int *__restrict__ cell_of_group, int *__restrict__ cell_count,
                              int *__restrict__ slot, double *__restrict__ last)
{
  if (!flags[kFlagRebuild])
    return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroup)
    return;
  const int n = cg.n;
  int ijk[3];
  for (int d = 0; d < 3; d++) {
    const double x = anchor[3 * g + d];
    ijk[d] = (int) floor(__dadd_rn(__ddiv_rn(x, cg.lc[d]), 0.5));
    ijk[d] %= n;
    if (ijk[d] < 0)
      ijk[d] += n;
    last[3 * g + d] = x;
  }
  const int c = (ijk[0] * n + ijk[1]) * n + ijk[2];
  cell_of_group[g] = c;
  slot[g] = atomicAdd(&cell_count[cell_rank[c]], 1);
}

// exclusive scan of per-rank counts, one block
constexpr int kScanThreads = 1024;

__global__ void k_scan_cells(const int *__restrict__ count, int ncell3, const int *__restrict__ flags,
                             int *__restrict__ start)
{
  if (!flags[kFlagRebuild])
    return;
  __shared__ int part[kScanThreads];
  const int per = (ncell3 + kScanThreads - 1) / kScanThreads;
  const int beg = threadIdx.x * per;
  const int end = min(beg + per, ncell3);
  int s = 0;
  for (int i = beg; i < end; i++)
    s += count[i];
  part[threadIdx.x] = s;
  __syncthreads();
  // Hillis-Steele inclusive scan of the partial sums
  for (int off = 1; off < kScanThreads; off <<= 1) {
    const int v = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = threadIdx.x > 0 ? part[threadIdx.x - 1] : 0;
  for (int i = beg; i < end; i++) {
    start[i] = run;
    run += count[i];
  }
  if (threadIdx.x == kScanThreads - 1)
    start[ncell3] = part[kScanThreads - 1];
}

__global__ void k_cell_scatter(int ngroup, const int *__restrict__ cell_of_group,
                               const int *__restrict__ cell_rank, const int *__restrict__ start,
                               const int *__restrict__ slot, const int *__restrict__ flags,
                               int *__restrict__ sorted)
{
  if (!flags[kFlagRebuild])
    return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroup)
    return;
  sorted[start[cell_rank[cell_of_group[g]]] + slot[g]] = g;
}

// order each cell's members by group index (deterministic lists), then record
// sorted positions and the anchors the list is built from
__global__ void k_cell_finish(int ncell3, const int *__restrict__ start, const double *__restrict__ last,
                              const int *__restrict__ flags, int *__restrict__ sorted,
                              int *__restrict__ rank, double *__restrict__ anchor_sorted)
{
  if (!flags[kFlagRebuild])
    return;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell3)
    return;
  const int b = start[c], e = start[c + 1];
  for (int i = b + 1; i < e; i++) {
    const int v = sorted[i];
    int j = i - 1;
    while (j >= b && sorted[j] > v) {
      sorted[j + 1] = sorted[j];
      j--;
    }
    sorted[j + 1] = v;
  }
  for (int i = b; i < e; i++) {
    const int g = sorted[i];
    rank[g] = i;
    anchor_sorted[3 * i] = last[3 * g];
    anchor_sorted[3 * i + 1] = last[3 * g + 1];
    anchor_sorted[3 * i + 2] = last[3 * g + 2];
  }
}

struct BuildArgs {
  int ngroup, nstencil, rowcap;
  CellGeom cg;
  Box box;
  const int *stencil;        // 3 per offset, components in [0, n)
  const int *sorted;
  const int *cell_of_group;
  const int *cell_rank;
  const int *start;
  const double *anchor_sorted;
  const int *flags;
  int *nbr;
  int *nbr_count;
  int *flags_w;
};

constexpr int kBuildWarps = 8;

// one warp per sorted group; lanes walk stencil cells, members are compacted
// into the row with a ballot
__global__ void __launch_bounds__(kBuildWarps * 32) k_build_list(BuildArgs a)
{
  if (!a.flags[kFlagRebuild])
    return;
  const int lane = threadIdx.x & 31;
  const int p = blockIdx.x * kBuildWarps + (threadIdx.x >> 5);
  if (p >= a.ngroup)
    return;
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
      atomicMax(&a.flags_w[kFlagOverflow], count);
    atomicMax(&a.flags_w[kFlagMaxRow], count);
  }
}

cudaError_t launch_gather_anchors(mmnb_handle *h, const double *d_r)
{
  k_gather_anchors<<<div_up(h->ngroup, 256), 256, 0, h->stream>>>(d_r, h->d_group, h->ngroup, h->d_anchor);
  h->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_rebuild_decide(mmnb_handle *h, int force)
{
  k_top2<<<h->top2_blocks, kTop2Threads, 0, h->stream>>>(h->d_anchor, h->d_last, h->ngroup, h->d_top2);
  k_decide<<<1, kTop2Threads, 0, h->stream>>>(h->d_top2, h->top2_blocks, h->nlw, h->first ? 1 : 0, force,
                                               h->cfg.rebuild_interval, h->d_flags);
  h->launches += 2;
  return cudaGetLastError();
}

cudaError_t launch_build_list(mmnb_handle *h)
{
  cudaError_t e;
  if ((e = cudaMemsetAsync(h->d_cell_count, 0, sizeof(int) * h->ncell3, h->stream)) != cudaSuccess)
    return e;
  k_cell_assign<<<div_up(h->ngroup, 256), 256, 0, h->stream>>>(h->d_anchor, h->ngroup, h->cg, h->d_cell_rank,
                                                                h->d_flags, h->d_cell_of_group, h->d_cell_count,
                                                                h->d_slot, h->d_last);
  k_scan_cells<<<1, kScanThreads, 0, h->stream>>>(h->d_cell_count, h->ncell3, h->d_flags, h->d_cell_start);
  k_cell_scatter<<<div_up(h->ngroup, 256), 256, 0, h->stream>>>(h->ngroup, h->d_cell_of_group, h->d_cell_rank,
                                                                 h->d_cell_start, h->d_slot, h->d_flags,
                                                                 h->d_sorted);
  k_cell_finish<<<div_up(h->ncell3, 128), 128, 0, h->stream>>>(h->ncell3, h->d_cell_start, h->d_last, h->d_flags,
                                                                h->d_sorted, h->d_rank, h->d_anchor_sorted);
  BuildArgs a;
  a.ngroup = h->ngroup;
  a.nstencil = h->nstencil;
  a.rowcap = h->rowcap;
  a.cg = h->cg;
  a.box = h->box;
  a.stencil = h->d_stencil;
  a.sorted = h->d_sorted;
  a.cell_of_group = h->d_cell_of_group;
  a.cell_rank = h->d_cell_rank;
  a.start = h->d_cell_start;
  a.anchor_sorted = h->d_anchor_sorted;
  a.flags = h->d_flags;
  a.nbr = h->d_nbr;
  a.nbr_count = h->d_nbr_count;
  a.flags_w = h->d_flags;
  k_build_list<<<div_up(h->ngroup, kBuildWarps), kBuildWarps * 32, 0, h->stream>>>(a);
  h->launches += 5;
  return cudaGetLastError();
}

}  // namespace mmnb

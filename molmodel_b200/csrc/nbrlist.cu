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
// and the pair set is identical, not merely close.  The list build first
// tests each candidate in FP32 against a band around (cutoff + width)^2 wide
// enough to hold every FP32 rounding error; only candidates inside the band
// take the FP64 test, so the decision is the FP64 one.
//
// The list is stored FULL (each unordered pair in both rows) so the pair
// kernels accumulate on their own rows only, without atomics.  Rows are
// indexed by sorted position (groups ordered by the Morton rank of their cell).

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>

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
  __syncthreads();  // sa, sb may be reused at once
}

// Anchors of this evaluation, the two largest anchor moves since the last
// build, and the rebuild decision (first || forced || largest + second >
// width || fixed interval), all in one launch: each block reduces its share,
// the last block to finish merges the block results.  On a rebuild the last
// block also clears the cell counts for the rebuild kernel.
// flags[4] counts evaluations, flags[5] rebuilds, flags[6] is the block counter.
// With pruned rows (prune > 0; the rigid-water kernel) the same pass takes
// the two largest moves since the last prune (plast, sorted order of the
// build) and sets flags[kFlagPruneFull] when the pruned rows must be made
// again: after a rebuild, while they are not valid, or when those moves add
// up to more than the prune margin.
__global__ void __launch_bounds__(kCheckThreads) k_list_check(const double *__restrict__ r,
                                                              const int *__restrict__ group, int ngroup,
                                                              const double *__restrict__ last, double width,
                                                              int first, int force, int interval,
                                                              double *__restrict__ anchor,
                                                              double *__restrict__ partial, int *__restrict__ flags,
                                                              int *__restrict__ cell_count, int ncell3,
                                                              double prune, const int *__restrict__ rank,
                                                              const double *__restrict__ plast)
{
  __shared__ double sa[kCheckThreads], sb[kCheckThreads];
  __shared__ bool last_block;
  double a = 0, b = 0, pa = 0, pb = 0;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngroup; g += gridDim.x * blockDim.x) {
    const int s0 = group[2 * g];
    const double x = r[3 * s0], y = r[3 * s0 + 1], z = r[3 * s0 + 2];
    anchor[3 * g] = x;
    anchor[3 * g + 1] = y;
    anchor[3 * g + 2] = z;
    const double dx = __dsub_rn(x, last[3 * g]);
    const double dy = __dsub_rn(y, last[3 * g + 1]);
    const double dz = __dsub_rn(z, last[3 * g + 2]);
    // squared moves: the square root (monotonic, correctly rounded) is
    // taken of the two largest only, in the last block
    const double d = exact_sq3(dx, dy, dz);
    if (d > a) {
      b = a;
      a = d;
    } else if (d > b) {
      b = d;
    }
    if (prune > 0) {
      const int p = rank[g];
      const double ex = x - plast[3 * p], ey = y - plast[3 * p + 1], ez = z - plast[3 * p + 2];
      const double e = ex * ex + ey * ey + ez * ez;
      if (e > pa) {
        pb = pa;
        pa = e;
      } else if (e > pb) {
        pb = e;
      }
    }
  }
  block_top2(a, b, sa, sb);
  if (prune > 0)
    block_top2(pa, pb, sa, sb);
  if (threadIdx.x == 0) {
    partial[4 * blockIdx.x] = a;
    partial[4 * blockIdx.x + 1] = b;
    partial[4 * blockIdx.x + 2] = pa;
    partial[4 * blockIdx.x + 3] = pb;
    __threadfence();
    last_block = atomicAdd(flags + 6, 1) == (int) gridDim.x - 1;
  }
  __syncthreads();
  if (!last_block)
    return;
  __threadfence();
  a = b = pa = pb = 0;
  for (int i = threadIdx.x; i < (int) gridDim.x; i += blockDim.x) {
    top2_merge(a, b, partial[4 * i], partial[4 * i + 1]);
    top2_merge(pa, pb, partial[4 * i + 2], partial[4 * i + 3]);
  }
  block_top2(a, b, sa, sb);
  block_top2(pa, pb, sa, sb);
  a = __dsqrt_rn(a);
  b = __dsqrt_rn(b);
  pa = sqrt(pa);
  pb = sqrt(pb);
  __shared__ int rebuild_s;
  if (threadIdx.x == 0) {
    const int count = flags[4];
    int rebuild = first || force || flags[kFlagForceRebuild] || (__dadd_rn(b, a) > width);
    flags[kFlagForceRebuild] = 0;
    if (interval > 0 && count % interval == 0)
      rebuild = 1;
    flags[kFlagRebuild] = rebuild;
    flags[4] = count + 1;
    if (rebuild)
      flags[5] += 1;  // rebuild counter
    flags[6] = 0;
    rebuild_s = rebuild;
    if (rebuild) {
      flags[kFlagPruneValid] = 0;
      flags[kFlagListTrunc] = 0;
    }
    flags[kFlagPruneFull] = prune > 0 ? (rebuild || !flags[kFlagPruneValid] || pa + pb > prune) : 1;
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
  // FP32 pre-test of the list build: sorted anchors wrapped into the box, and
  // squared distances that are certainly inside (< c2lo) or outside (> c2hi)
  // of (cutoff + width)^2 whatever the FP32 rounding; only the rest take the
  // exact FP64 test, so the pair set is the same
  float4 *anchor32;
  float Lf[3], invLf[3];
  float c2lo, c2hi;
  // per-row cull of stencil cells: a cell whose every point is farther than
  // sqrt(c2cull) > cutoff + width from the row's anchor holds no partner
  float lcf[3], c2cull;
  int *block_sum;            // per block of the launch: its segment's cell count
  int *scatter;              // groups by cell before the in-cell ordering (ngroup)
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
    // a non-finite anchor converts to cell 0 (float-to-int conversion gives 0
    // for NaN and saturates): flagged, the host reports it
    if (!isfinite(x))
      a.flags[kFlagError] = MMNB_ERR_DEVICE;
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

// Exclusive scan of the 256 values of a block (one per thread); returns the
// thread's exclusive prefix and the block total in *total.
__device__ __forceinline__ int block_exclusive_scan(int v, int *warp_tot, int *total)
{
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o)
      incl += u;
  }
  if (lane == 31)
    warp_tot[w] = incl;
  __syncthreads();
  int before = 0, all = 0;
  for (int k = 0; k < kRebuildThreads / 32; k++) {
    const int t = warp_tot[k];
    before += k < w ? t : 0;
    all += t;
  }
  __syncthreads();
  *total = all;
  return before + incl - v;
}

// Counting-sort offsets over the whole grid: each block sums a contiguous
// segment of the per-rank cell counts (phase 1); after a grid barrier each
// block adds the sums of the blocks before it and scans its segment (phase 2).
__device__ __forceinline__ void scan_segment(const RebuildArgs &a, int &lo, int &hi)
{
  const int seg = (a.ncell3 + gridDim.x - 1) / gridDim.x;
  lo = min(a.ncell3, (int) blockIdx.x * seg);
  hi = min(a.ncell3, lo + seg);
}

__device__ void scan_cells_sum(const RebuildArgs &a, int *warp_tot)
{
  int lo, hi;
  scan_segment(a, lo, hi);
  int v = 0;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x)
    v += a.cell_count[i];
  int total;
  block_exclusive_scan(v, warp_tot, &total);
  if (threadIdx.x == 0)
    a.block_sum[blockIdx.x] = total;
}

__device__ void scan_cells_write(const RebuildArgs &a, int *warp_tot)
{
  int lo, hi;
  scan_segment(a, lo, hi);
  int v = 0;
  for (int k = threadIdx.x; k < (int) blockIdx.x; k += blockDim.x)
    v += a.block_sum[k];
  int run;
  block_exclusive_scan(v, warp_tot, &run);
  for (int i0 = lo; i0 < hi; i0 += blockDim.x) {
    const int i = i0 + threadIdx.x;
    const int c = i < hi ? a.cell_count[i] : 0;
    int tile;
    const int ex = block_exclusive_scan(c, warp_tot, &tile);
    if (i < hi)
      a.start[i] = run + ex;
    run += tile;
  }
  // the last block's running offset ends at the total
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
    a.start[a.ncell3] = run;
}

// Final sorted position of the group scattered to position i (members of a
// cell ordered by group index: deterministic lists), its rank, and the
// anchors the list is built from.
__device__ __forceinline__ void place_group(const RebuildArgs &a, int i)
{
  const int g = a.scatter[i];
  const int rj = a.cell_rank[a.cell_of_group[g]];
  const int b = a.start[rj], e = a.start[rj + 1];
  int r = 0;
  for (int j = b; j < e; j++)
    r += a.scatter[j] < g;
  const int pos = b + r;
  a.sorted[pos] = g;
  a.rank[g] = pos;
  float w[3];
  for (int d = 0; d < 3; d++) {
    const double x = a.last[3 * g + d];
    a.anchor_sorted[3 * pos + d] = x;
    w[d] = (float) (x - a.box.L[d] * floor(x * a.box.invL[d]));
  }
  a.anchor32[pos] = make_float4(w[0], w[1], w[2], 0.f);
}

// one warp per sorted group.  Per batch of 32 stencil cells the members are
// laid out in one candidate sequence (cell order, then member order; a warp
// scan of the cells' counts gives each cell's offset), the lanes test
// consecutive candidates, and the accepted ones are compacted into the row
// with a ballot.  Rows are in a fixed order (deterministic lists).
constexpr int kCand = 128;  // candidates staged per warp at a time
constexpr int kSeg = 256;   // stencil cells whose member ranges a warp fetches at a time

__device__ __forceinline__ void build_row(const RebuildArgs &a, int p, int lane, int *cand, int2 *ranges)
{
  const int n = a.cg.n;
  const int gi = a.sorted[p];
  const int ci = a.cell_of_group[gi];
  const int ix = ci / (n * n), iy = (ci / n) % n, iz = ci % n;
  const double xi = a.anchor_sorted[3 * p], yi = a.anchor_sorted[3 * p + 1], zi = a.anchor_sorted[3 * p + 2];
  const float4 wi = a.anchor32[p];
  int *row = a.nbr + (size_t) p * a.rowcap;
  const unsigned below = (1u << lane) - 1;
  int count = 0;
  for (int g0 = 0; g0 < a.nstencil; g0 += kSeg) {
    // the member ranges of a segment of stencil cells, fetched with independent
    // loads (one dependent chain per cell instead of one per batch of 32);
    // the cells that can hold a partner and are not empty are compacted in
    // stencil order, so the batches below see only them (the own cell, stencil
    // entry 0, always has the row's group and comes first)
    const int segn = min(kSeg, a.nstencil - g0);
    int kept = 0;
#pragma unroll 2
    for (int t0 = 0; t0 < segn; t0 += 32) {
      const int t = t0 + lane;
      int2 rg = make_int2(0, 0);
      if (t < segn) {
        const int s = g0 + t;
        // cell and stencil components are in [0, n): one conditional subtraction wraps
        int jx = ix + a.stencil[3 * s], jy = iy + a.stencil[3 * s + 1], jz = iz + a.stencil[3 * s + 2];
        jx -= jx >= n ? n : 0;
        jy -= jy >= n ? n : 0;
        jz -= jz >= n ? n : 0;
        // lower bound of the distance from this row's anchor (wrapped into the
        // box) to the cell's slab [c l - l/2, c l + l/2] on each axis, minimum image
        float dx = wi.x - (float) jx * a.lcf[0], dy = wi.y - (float) jy * a.lcf[1], dz = wi.z - (float) jz * a.lcf[2];
        dx = fmaxf(fabsf(dx - a.Lf[0] * rintf(dx * a.invLf[0])) - 0.5f * a.lcf[0], 0.f);
        dy = fmaxf(fabsf(dy - a.Lf[1] * rintf(dy * a.invLf[1])) - 0.5f * a.lcf[1], 0.f);
        dz = fmaxf(fabsf(dz - a.Lf[2] * rintf(dz * a.invLf[2])) - 0.5f * a.lcf[2], 0.f);
        if (s == 0 || dx * dx + dy * dy + dz * dz <= a.c2cull) {
          const int rj = a.cell_rank[(jx * n + jy) * n + jz];
          rg = make_int2(a.start[rj], a.start[rj + 1]);
        }
      }
      const bool keep = rg.y > rg.x;
      const unsigned kb = __ballot_sync(0xffffffffu, keep);
      if (keep)
        ranges[kept + __popc(kb & below)] = rg;
      kept += __popc(kb);
    }
    __syncwarp();
    for (int b0 = 0; b0 < kept; b0 += 32) {
      const int s0 = g0 + b0;
      int beg = 0, end = 0;
      if (b0 + lane < kept) {
        const int2 rg = ranges[b0 + lane];
        beg = rg.x;
        end = rg.y;
      }
      const int c = end - beg;
      int incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o)
          incl += v;
      }
      const int excl = incl - c;
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      // stencil entry 0 is the group's own cell: its members pair unconditionally
      const int own = s0 == 0 ? __shfl_sync(0xffffffffu, incl, 0) : 0;
      for (int base = 0; base < total; base += kCand) {
        const int lo = max(excl, base), hi = min(incl, base + kCand);
        for (int k = lo; k < hi; k++)
          cand[k - base] = beg + (k - excl);
        __syncwarp();
        const int nb = min(kCand, total - base);
        for (int k0 = 0; k0 < nb; k0 += 32) {
          const int k = k0 + lane;
          bool take = false;
          int q = 0;
          if (k < nb) {
            q = cand[k];
            if (q != p) {
              if (base + k < own) {
                take = true;
              } else {
                const float4 wj = a.anchor32[q];
                float fx = wi.x - wj.x, fy = wi.y - wj.y, fz = wi.z - wj.z;
                fx -= a.Lf[0] * rintf(fx * a.invLf[0]);
                fy -= a.Lf[1] * rintf(fy * a.invLf[1]);
                fz -= a.Lf[2] * rintf(fz * a.invLf[2]);
                const float f2 = fx * fx + fy * fy + fz * fz;
                if (f2 < a.c2lo) {
                  take = true;
                } else if (f2 <= a.c2hi) {
                  const double dx = exact_wrap(__dsub_rn(xi, a.anchor_sorted[3 * q]), a.box.L[0], a.box.invL[0]);
                  const double dy = exact_wrap(__dsub_rn(yi, a.anchor_sorted[3 * q + 1]), a.box.L[1], a.box.invL[1]);
                  const double dz = exact_wrap(__dsub_rn(zi, a.anchor_sorted[3 * q + 2]), a.box.L[2], a.box.invL[2]);
                  take = exact_sq3(dx, dy, dz) < a.cg.c2;
                }
              }
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
        __syncwarp();
      }
    }
    __syncwarp();
  }
  if (lane == 0) {
    a.nbr_count[p] = min(count, a.rowcap);
    if (count > a.rowcap) {
      atomicMax(&a.flags[kFlagOverflow], count);
      a.flags[kFlagListTrunc] = 1;
    }
    atomicMax(&a.flags[kFlagMaxRow], count);
  }
}

// The whole rebuild in one cooperative launch: cell assignment, counting-sort
// scan (block sums, then offsets), scatter, placement in group order within
// each cell, list rows, separated by grid-wide barriers.  Without a rebuild due every block returns at once (the decision
// is read from device memory, so the launch sits in a CUDA graph unchanged).
__global__ void __launch_bounds__(kRebuildThreads) k_list_rebuild(RebuildArgs a)
{
  if (!a.flags[kFlagRebuild])
    return;
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  __shared__ int warp_tot[kBuildWarps];
  __shared__ int cand[kBuildWarps * kCand];
  __shared__ int2 ranges[kBuildWarps * kSeg];
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (int g = tid; g < a.ngroup; g += nth)
    cell_assign(a, g);
  grid.sync();
  scan_cells_sum(a, warp_tot);
  grid.sync();
  scan_cells_write(a, warp_tot);
  grid.sync();
  for (int g = tid; g < a.ngroup; g += nth)
    a.scatter[a.start[a.cell_rank[a.cell_of_group[g]]] + a.slot[g]] = g;
  grid.sync();
  for (int i = tid; i < a.ngroup; i += nth)
    place_group(a, i);
  grid.sync();
  const int lane = threadIdx.x & 31;
  for (int p = tid >> 5; p < a.ngroup; p += nth >> 5)
    build_row(a, p, lane, cand + (threadIdx.x >> 5) * kCand, ranges + (threadIdx.x >> 5) * kSeg);
}

cudaError_t launch_list_check(mmnb_handle *h, const double *d_r, int force)
{
  k_list_check<<<h->top2_blocks, kCheckThreads, 0, h->stream>>>(
      d_r, h->d_group, h->ngroup, h->d_last, h->nlw, h->first ? 1 : 0, force, h->cfg.rebuild_interval, h->d_anchor,
      h->d_top2, h->d_flags, h->d_cell_count, h->ncell3, h->water ? h->prune_margin : 0.0, h->d_rank,
      h->d_plast);
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
    h->rebuild_grid = std::min(std::min(per_sm * nsm, div_up(h->ngroup, kBuildWarps)), h->block_sum_cap);
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
  a.anchor32 = h->d_anchor32;
  a.block_sum = h->d_block_sum;
  // the rows' counts are written last, by the list build: until then they
  // hold the groups in cell order
  a.scatter = h->d_nbr_count;
  // bound of the FP32 squared-distance error: anchors wrapped into [0, L] and
  // rounded (<= 4 ulp(L) per component after the difference and the image
  // shift), propagated through |d|^2, plus the rounding of the sum; 8x margin
  double lmax = 0, lmin = 1e300;
  for (int d = 0; d < 3; d++) {
    a.Lf[d] = (float) h->box.L[d];
    a.invLf[d] = (float) h->box.invL[d];
    lmax = std::max(lmax, h->box.L[d]);
    lmin = std::min(lmin, h->box.L[d]);
  }
  const double c2 = h->cg.c2, ulp = std::ldexp(1.0, -23);
  const double tol = 8 * (2 * std::sqrt(3.0) * std::sqrt(c2) * 4 * ulp * lmax + 4 * ulp * c2);
  // the FP32 minimum image may pick another image only at |d| ~ L/2
  const bool safe = std::sqrt(c2) + 1.0 < 0.45 * lmin;
  a.c2lo = safe ? (float) (c2 - tol) : -1.0f;
  a.c2hi = safe ? (float) (c2 + tol) : 3.0e38f;
  // the cull keeps a 0.01 A margin over the FP32 rounding of the anchors and
  // cell centres (~1e-5 A here); boxes where the FP32 minimum image is not
  // safe keep every stencil cell
  for (int d = 0; d < 3; d++)
    a.lcf[d] = (float) h->cg.lc[d];
  const double cull = std::sqrt(c2) + 0.01;
  a.c2cull = safe ? (float) (cull * cull) : 3.0e38f;
  void *args[] = {&a};
  h->launches += 1;
  return cudaLaunchCooperativeKernel((const void *) k_list_rebuild, dim3(h->rebuild_grid), dim3(kRebuildThreads),
                                     args, 0, h->stream);
}

}  // namespace mmnb

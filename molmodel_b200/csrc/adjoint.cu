// Adjoint of one evaluation with respect to three uniform parameter scales:
// all charges (lambda_q), all LJ sigmas (lambda_s) and all LJ epsilons
// (lambda_e), each at 1.  For rigid water with q_H = -q_O/2 and LJ on O only
// these are the per-type parameters (q_O, sigma_O, epsilon_O) times their
// values, the parameters WeakCouple and BCIFit update (src/msimprog.cpp:855-876,
// src/bcifit.cpp:44-59, values mapped to sites by ElecLJ::types_changed,
// src/eleclj.cpp:440-503).
//
// Structure used (exact, no approximation):
//   * every electrostatic term (real space with its switch-derivative share,
//     reciprocal space, exclusions, self and neutralising terms) is a sum of
//     q_i q_j products, so E_elec(lambda_q) = lambda_q^2 E_elec and likewise the
//     electrostatic force: d/dlambda_q = 2 x (the electrostatic part);
//   * the LJ pair energy with the group switch is S (A/r^12 - B/r^6) with
//     A = 4 eps sig^12, B = 4 eps sig^6: linear in lambda_e, and its A and B
//     parts scale as lambda_s^12 and lambda_s^6; the tail correction is linear
//     in totA and totB (src/eleclj.cpp:294-308, 1247-1266).
// The backward kernel recomputes the LJ pair terms of every listed group pair
// inside the cutoff in FP64 (nothing from the forward pass is stored), splits
// energy and force into their A and B parts, and contracts the forces with the
// caller's dL/dF.  The electrostatic force is the forward force minus the LJ
// force, so the charge gradient of the loss needs no second field solve.
//
// Scope: LJ sites must be group anchors, without group exclusions or 1-4
// pairs (rigid water and united-atom-like models); other systems return
// MMNB_ERR_UNSUPPORTED.

#include <vector>

#include "mmnb_internal.cuh"

namespace mmnb {

constexpr int kBwdWarps = 8;

struct BwdArgs {
  int ngroup, rowcap, geometric;
  Box box;
  double rhi2, rlo2, inv_sw;
  const double *r;        // positions (caller's order)
  const double *dl_df;    // 3 * nsite, or null
  const int *sorted, *group, *mask, *nbr, *nbr_count;
  const double *sig, *eps;
  double *partial;        // 4 per row: E_A, E_B, g.F_A, g.F_B
};

// one warp per row group; lanes walk the row's list entries
__global__ void __launch_bounds__(kBwdWarps * 32) k_lj_backward(BwdArgs a)
{
  const int lane = threadIdx.x & 31;
  const int p = blockIdx.x * kBwdWarps + (threadIdx.x >> 5);
  if (p >= a.ngroup)
    return;
  const int ai = a.group[2 * a.sorted[p]];
  double ea = 0, eb = 0, ga = 0, gb = 0;
  if (a.mask[ai] & MMNB_SITE_HAS_LJ) {
    const double4 ri = make_double4(a.r[3 * ai], a.r[3 * ai + 1], a.r[3 * ai + 2], 0);
    double gx = 0, gy = 0, gz = 0;
    if (a.dl_df) {
      gx = a.dl_df[3 * ai];
      gy = a.dl_df[3 * ai + 1];
      gz = a.dl_df[3 * ai + 2];
    }
    const double si = a.sig[ai], ei = a.eps[ai];
    const int cnt = a.nbr_count[p];
    const int *row = a.nbr + (size_t) p * a.rowcap;
    for (int e = lane; e < cnt; e += 32) {
      const int aj = a.group[2 * a.sorted[row[e]]];
      if (!(a.mask[aj] & MMNB_SITE_HAS_LJ))
        continue;
      const double4 rj = make_double4(a.r[3 * aj], a.r[3 * aj + 1], a.r[3 * aj + 2], 0);
      double x, y, z, sx, sy, sz;
      const double r2 = anchor_disp(a.box, ri, rj, x, y, z, sx, sy, sz);
      if (r2 > a.rhi2)
        continue;
      double s = 1, ds = 0;
      if (r2 > a.rlo2) {
        const double zz = (r2 - a.rlo2) * a.inv_sw;
        s = 1 + zz * zz * zz * (-10 + zz * (15 - 6 * zz));
        ds = ((60 * zz - 120) * zz + 60) * zz * zz * a.inv_sw;
      }
      const double sj = a.sig[aj], ej = a.eps[aj];
      const double sg = a.geometric ? sqrt(si * sj) : 0.5 * (si + sj);
      const double s6 = sg * sg * sg * sg * sg * sg;
      const double b = 4 * sqrt(ei * ej) * s6;
      const double ir2 = 1 / r2, ir6 = ir2 * ir2 * ir2;
      const double bi6 = b * ir6, ai12 = b * s6 * ir6 * ir6;
      ea += 0.5 * s * ai12;
      eb += 0.5 * s * bi6;
      // force on the row's anchor from each part, switch derivative included:
      // -grad(S u) = (S du/dr2 * (-2) + u * ds) d
      const double fa = 12 * ai12 * ir2 * s + ds * ai12;
      const double fb = 6 * bi6 * ir2 * s + ds * bi6;
      const double gd = gx * x + gy * y + gz * z;
      ga += fa * gd;
      gb += fb * gd;
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    ea += __shfl_xor_sync(0xffffffffu, ea, o);
    eb += __shfl_xor_sync(0xffffffffu, eb, o);
    ga += __shfl_xor_sync(0xffffffffu, ga, o);
    gb += __shfl_xor_sync(0xffffffffu, gb, o);
  }
  if (lane == 0) {
    double *o = a.partial + 4 * (size_t) p;
    o[0] = ea;
    o[1] = eb;
    o[2] = ga;
    o[3] = gb;
  }
}

}  // namespace mmnb

using namespace mmnb;

static int bwd_fail(mmnb_handle *h, int code, const std::string &msg)
{
  if (h)
    h->err = msg;
  return code;
}

extern "C" int mmnb_backward(mmnb_handle *h, const double *r, const double *dl_df, double *f, double *u,
                             double grad_u[3], double grad_l[3])
{
  if (!h || !r || !grad_u)
    return bwd_fail(h, MMNB_ERR_ARG, "null handle, positions or gradient output");
  if (!h->params_set)
    return bwd_fail(h, MMNB_ERR_STATE, "mmnb_set_params has not been called");
  if (!h->lj_on_anchors_only || h->any_gexcl || h->use_14)
    return bwd_fail(h, MMNB_ERR_UNSUPPORTED,
                "the backward pass covers LJ sites that are group anchors, without group exclusions or 1-4 pairs");
  const size_t n3 = 3 * (size_t) h->nsite;
  // forward pass (also brings the neighbour list up to date for r)
  std::vector<double> fw(n3, 0.0);
  mmnb_energy en;
  int s = mmnb_compute(h, r, fw.data(), nullptr, &en, nullptr, nullptr);
  if (s)
    return s;
  double gF = 0;
  if (dl_df)
    for (size_t k = 0; k < n3; k++)
      gF += dl_df[k] * fw[k];
  // LJ pair terms in FP64 over the current list; scratch kept by the handle
  const size_t np = 4 * (size_t) h->ngroup;
  if (h->bwd_cap < np + n3) {
    if (h->d_bwd)
      cudaFree(h->d_bwd);
    h->d_bwd = nullptr;
    h->bwd_cap = 0;
    const cudaError_t ea = cudaMalloc(&h->d_bwd, (np + n3) * sizeof(double));
    if (ea != cudaSuccess)
      return bwd_fail(h, MMNB_ERR_CUDA, std::string("backward scratch: ") + cudaGetErrorString(ea));
    h->bwd_cap = np + n3;
  }
  double *d_part = h->d_bwd, *d_g = dl_df ? h->d_bwd + np : nullptr;
  std::vector<double> part(np);
  BwdArgs a;
  a.ngroup = h->ngroup;
  a.rowcap = h->rowcap;
  a.geometric = h->cfg.geometric_combining_for_sigma;
  a.box = h->box;
  a.rhi2 = h->rhi2;
  a.rlo2 = h->rlo2;
  a.inv_sw = h->inv_sw;
  a.r = h->d_r;  // mmnb_compute left this evaluation's positions here
  a.dl_df = d_g;
  a.sorted = h->d_sorted;
  a.group = h->d_group;
  a.mask = h->d_mask;
  a.nbr = h->d_nbr;
  a.nbr_count = h->d_nbr_count;
  a.sig = h->d_sig;
  a.eps = h->d_eps;
  a.partial = d_part;
  cudaError_t e = cudaSuccess;
  if (d_g)
    e = cudaMemcpyAsync(d_g, dl_df, n3 * sizeof(double), cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    k_lj_backward<<<div_up(h->ngroup, kBwdWarps), kBwdWarps * 32, 0, h->stream>>>(a);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(part.data(), d_part, np * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess)
    return bwd_fail(h, MMNB_ERR_CUDA, std::string("backward pass: ") + cudaGetErrorString(e));
  // fixed-order sums
  double ea = 0, eb = 0, ga = 0, gb = 0;
  for (int p = 0; p < h->ngroup; p++) {
    ea += part[4 * p];
    eb += part[4 * p + 1];
    ga += part[4 * p + 2];
    gb += part[4 * p + 3];
  }
  const bool tail = h->cfg.include_lj_correction != 0;
  const double ta = tail ? lj_tail_ab(h, h->totA, 0) : 0, tb = tail ? lj_tail_ab(h, 0, h->totB) : 0;
  grad_u[0] = 2 * en.elec;
  grad_u[1] = 12 * (ea + ta) - 6 * eb + 6 * tb;
  grad_u[2] = ea - eb + ta + tb;
  if (grad_l) {
    grad_l[0] = dl_df ? 2 * (gF - (ga - gb)) : 0;
    grad_l[1] = dl_df ? 12 * ga - 6 * gb : 0;
    grad_l[2] = dl_df ? ga - gb : 0;
  }
  if (f)
    for (size_t k = 0; k < n3; k++)
      f[k] += fw[k];
  if (u)
    *u += en.total;
  return MMNB_OK;
}

"""Virial (mmnb_virial): dU/ds along the reference's volume-move path -- box x s,
every molecule moved rigidly with its centre of mass x s (MSys::scale,
src/msys.cpp:416-421), eta / s and the P3M influence function / s with rc and
the mesh counts kept (ElecLJ::scale, src/eleclj.cpp:1268-1280) -- against
central differences of the energy:

* of the reference's own code (oracle/_ref, or the oracle's restatement where
  that was not built) evaluated at s = 1 +- h with the scaled box, eta / s and
  a grid spacing x s, the energy on both sides of the step that
  MSimProgram::test_scale (src/msimprog.cpp:379-400) takes;
* of this library's own energy through mmnb_scale (FP64 form).

The FP64 energy reads the reference's Chebyshev table, which is refitted for
each eta; the virial includes that table's own eta derivative (a second fit of
-eta d/d(eta) erfc(eta r)/r with the same nodes), so it is the derivative of
the reference's energy, not of exact Ewald sums.  That energy is a different
cubic on each r^2 segment of the table, so it jumps by ~1e-9 of a site pair's
energy where a site pair crosses a segment join (or r^2 = 4, below which erfc
is evaluated directly): a difference quotient whose two sides straddle a join
measures the jump, not the derivative.  The jumps the box's site pairs cross
between s = 1 - h and 1 + h are therefore summed from the table's cubics and
taken out of the difference; bound 5e-8 of |W|.  The mixed form's erfc depends on
eta r only, so it has no table term; its forces and energies carry ~4e-6
relative error, and the reference's table term is ~6e-6 of |W| on these
boxes: bound 2e-5 of |W|.
"""
import numpy as np
import pytest

from molmodel_b200 import ElecLJ, water_box
from molmodel_b200.water import SITE_HAS_LJ, SITE_HAS_Q
from oracle.oracle import make_config, port, reference

pytestmark = pytest.mark.gpu

H = 1e-6
ETA, RC = 0.35, 9.0


def scaled_positions(wb, s):
    r = wb.positions.reshape(-1, 3, 3)
    m = wb.masses.reshape(-1, 3)
    com = (r * m[:, :, None]).sum(1) / m.sum(1)[:, None]
    return (r + (s - 1) * com[:, None, :]).reshape(-1, 3)


def table_segment(i, eta=ETA, rc=RC):
    """Cubic i of the erfc(eta r)/r table in r^2 (src/rspace.c:25-37,
    src/cheby.c:7-45: 512 segments over [4, 1.2 rc^2], 50-node Chebyshev fit),
    continued past segment 511 by the same construction."""
    from math import cos, erfc, pi, sqrt
    mx = 1.2 * rc * rc
    dx = (mx - 4.0) / 512
    a, b = i * dx + 4.0, (i + 1) * dx + 4.0
    bma, bpa = 0.5 * (b - a), 0.5 * (b + a)
    g = []
    for k in range(50):
        r = sqrt(cos(pi * (k + 0.5) / 50) * bma + bpa)
        g.append(erfc(eta * r) / r)
    c = [2 / 50 * sum(g[k] * cos(pi * j * (k + 0.5) / 50) for k in range(50)) for j in range(4)]
    return np.array([c[0] / 2 - c[1] + c[2] - c[3], 2 * c[1] - 8 * c[2] + 18 * c[3], 8 * c[2] - 48 * c[3],
                     32 * c[3]])


def pieces(r2, continued, rc=RC):
    """Piece of the real-space Coulomb term a site pair's r^2 is in: -1 below
    the table (direct erfc), the segment index inside it, and past its end
    either 512 (direct erfc, the reference) or the continued segment index."""
    mn, mx = 4.0, 1.2 * rc * rc
    k = np.floor((r2 - mn) * (512 / (mx - mn))).astype(np.int64)
    k = np.where(r2 <= mn, -1, k)
    return k if continued else np.minimum(k, 512)


def piece_value(k, r2, continued, eta=ETA, rc=RC):
    from math import erfc, sqrt
    if k < 0 or (k >= 512 and not continued):
        r = sqrt(r2)
        return erfc(eta * r) / r
    mn, mx = 4.0, 1.2 * rc * rc
    f = (r2 - mn) * (512 / (mx - mn)) - k
    c = table_segment(k, eta, rc)
    return ((c[3] * f + c[2]) * f + c[1]) * f + c[0]


def site_pair_r2(wb, s, pairs):
    """r^2 of the nine site pairs of each listed group pair at scale s (the
    anchors' image), and the switch of each group pair."""
    r = scaled_positions(wb, s).reshape(-1, 3, 3)
    L = wb.box * s
    d = r[pairs[:, 0], 0] - r[pairs[:, 1], 0]
    d -= L * np.floor(d / L + 0.5)
    oi = r[pairs[:, 0]] - r[pairs[:, 0], :1]
    oj = r[pairs[:, 1]] - r[pairs[:, 1], :1]
    dv = d[:, None, None, :] + oi[:, :, None, :] - oj[:, None, :, :]
    R2 = (d ** 2).sum(-1)
    rlo2, rhi2 = (RC - 1.0) ** 2, RC ** 2
    z = np.clip((R2 - rlo2) / (rhi2 - rlo2), 0.0, None)
    S = np.where(R2 <= rhi2, ((-6 * z + 15) * z - 10) * z ** 3 + 1, 0.0)
    return (dv ** 2).sum(-1), S


def jump_sum(wb, pairs, h, continued, q=None):
    """Sum of the jumps of the piecewise real-space energy that the site pairs
    cross between s = 1 - h and s = 1 + h (each segment is its own fit, so the
    energy is discontinuous by ~1e-10 of a site pair's energy at a join)."""
    q = (wb.q if q is None else q).reshape(-1, 3)
    r2m, S = site_pair_r2(wb, 1 - h, pairs)
    r2p, _ = site_pair_r2(wb, 1 + h, pairs)
    pm, pp = pieces(r2m, continued), pieces(r2p, continued)
    mn, mx = 4.0, 1.2 * RC * RC
    dx = (mx - mn) / 512
    total = 0.0
    for g, a, b in zip(*np.nonzero(pm != pp)):
        qq = q[pairs[g, 0], a] * q[pairs[g, 1], b] * S[g]
        lo, hi = sorted((int(pm[g, a, b]), int(pp[g, a, b])))
        sign = 1.0 if pp[g, a, b] > pm[g, a, b] else -1.0
        for k in range(lo, hi):
            B = mn + (k + 1) * dx  # the join between piece k and piece k + 1
            total += sign * qq * (piece_value(k + 1, B, continued) - piece_value(k, B, continued))
    return total


def c1_cfg(box, s=1.0):
    return dict(rspace_cutoff=9.0, ewald_screening=0.35 / s, kspace_cutoff=7.0)


def c2_cfg(box, s=1.0):
    return dict(rspace_cutoff=9.0, ewald_screening=0.35 / s, use_p3m=True, p3m_grid_spacing=s * box / 48,
                p3m_assignment_order=5, neighbor_list_width=1.5)


def oracle_at(wb, cfg_of, s, site_mask=None, sigma=None, epsilon=None):
    lib = reference() or port()
    box = wb.box * s
    c = make_config(box, **cfg_of(wb.box, s))
    o = lib.eleclj(c, wb.nsite, wb.groups, wb.exclusions, wb.site_mask if site_mask is None else site_mask, wb.q,
                   wb.sigma if sigma is None else sigma, wb.epsilon if epsilon is None else epsilon, wb.rscreen)
    return o, o.eval(scaled_positions(wb, s))["total"]


def oracle_energy(wb, cfg_of, s, site_mask=None, sigma=None, epsilon=None):
    return oracle_at(wb, cfg_of, s, site_mask, sigma, epsilon)[1]


def oracle_difference(wb, cfg_of, site_mask=None, sigma=None, epsilon=None):
    """U at s = 1 and the central difference of U over s = 1 +- H, less the
    table's jumps crossed in between."""
    o, u0 = oracle_at(wb, cfg_of, 1.0, site_mask, sigma, epsilon)
    du = oracle_energy(wb, cfg_of, 1 + H, site_mask, sigma, epsilon) - \
        oracle_energy(wb, cfg_of, 1 - H, site_mask, sigma, epsilon)
    du -= jump_sum(wb, o.nbrlist().pairs(), H, continued=False)
    return u0, du / (2 * H), H


CASES = [
    ("c1-ksum", 6, c1_cfg),
    ("c2-p3m", 16, c2_cfg),
]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name,n,cfg_of", CASES, ids=[c[0] for c in CASES])
def test_virial_matches_central_difference_of_reference_energy(name, n, cfg_of, precision):
    wb = water_box(n, seed=4)
    p = ElecLJ(precision=precision, **cfg_of(wb.box)).init(wb)
    w, e, f = p.virial(wb.positions, wb.masses)
    p.close()
    u0, fd, h = oracle_difference(wb, cfg_of)
    tol = 5e-8 if precision == "fp64" else 2e-5
    assert abs(w - fd) < tol * abs(w), (w, fd, u0, h)
    assert abs(e["total"] - u0) < (1e-10 if precision == "fp64" else 5e-5) * abs(u0)


@pytest.mark.parametrize("name,n,cfg_of", CASES, ids=[c[0] for c in CASES])
def test_virial_matches_central_difference_through_mmnb_scale(name, n, cfg_of):
    wb = water_box(n, seed=5)
    cfg = cfg_of(wb.box)
    p0 = ElecLJ(precision="fp64", **cfg).init(wb)
    w, e, _ = p0.virial(wb.positions, wb.masses)
    pairs = p0.pairlist()
    p0.close()
    h = H
    us = []
    for s in (1 + h, 1 - h):
        p = ElecLJ(precision="fp64", **cfg).init(wb)
        p.compute(wb.positions)
        p.scale(s)
        us.append(p.compute(scaled_positions(wb, s))["total"])
        p.close()
    # the rigid-water FP64 kernel continues the table past 1.2 rc^2
    fd = (us[0] - us[1] - jump_sum(wb, pairs, h, continued=True)) / (2 * h)
    assert abs(w - fd) < 5e-8 * abs(w), (w, fd, h)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_virial_general_kernels(precision):
    """LJ on the H sites too (a tiny epsilon): not the rigid-water topology, so
    the general pair kernels and their virial sums run."""
    wb = water_box(6, seed=6)
    mask = np.full(wb.nsite, SITE_HAS_Q | SITE_HAS_LJ, dtype=np.int32)
    sig = np.where(np.arange(wb.nsite) % 3 == 0, wb.sigma, 1.0)
    eps = np.where(np.arange(wb.nsite) % 3 == 0, wb.epsilon, 0.01)
    p = ElecLJ(precision=precision, **c1_cfg(wb.box)).init(wb)
    p.set_params(mask, wb.q, sig, eps)
    w, e, _ = p.virial(wb.positions, wb.masses)
    p.close()
    u0, fd, h = oracle_difference(wb, c1_cfg, mask, sig, eps)
    tol = 5e-8 if precision == "fp64" else 2e-5
    assert abs(w - fd) < tol * abs(w), (w, fd, u0, h)


def test_virial_refuses_screened_charges():
    from molmodel_b200._lib import MmnbError
    wb = water_box(6, seed=1)
    p = ElecLJ(precision="fp64", **c1_cfg(wb.box)).init(wb)
    p.set_params(wb.site_mask, wb.q, wb.sigma, wb.epsilon, np.full(wb.nsite, 0.5))
    with pytest.raises(MmnbError) as ex:
        p.virial(wb.positions, wb.masses)
    assert ex.value.status == 3
    p.close()

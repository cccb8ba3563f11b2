"""Adjoint (mmnb_forward, then mmnb_site_gradients): per-site gradients of the
energy U and of a force-matching loss L = sum_i |F_i - F_i^target|^2 with
respect to site charges, sigmas and epsilons, against central differences of
the oracle's energy and forces.

Directional checks: for a seeded direction v over the sites, sum_i v_i dX/dp_i
against (X(p + h v) - X(p - h v)) / 2h, Richardson-extrapolated over h and 2h,
with X = U or L and p = q, sigma or epsilon.  The charge directions are
non-uniform (random per site, or on one site type only), which a gradient with
respect to a uniform charge scale could not answer.  Positions do not move, so
no table segment join is crossed.  The sigma and epsilon steps are multiples of
1e-4 and 1e-5, exact in the six significant digits the reference's LJ tail
keys on (src/eleclj.cpp:283-308).

Systems: rigid water with the Ewald k-sum, P3M with real-space and with ik
differentiation, and a water box with cross-group exclusions, screening
radii, 1-4 pairs (O-O and O-H, scaled) and LJ on the H sites, so that every
term of the backward pass runs.  The C5 case (512 waters, 64 frames 1 ps apart
from FP64 dynamics at 300 K) checks the water-parameter gradients
d/d(q_O, sigma_O, epsilon_O) and a force-matching fit driven by them.
"""
import numpy as np
import pytest

from molmodel_b200 import ElecLJ, maxwell_boltzmann, water_box
from molmodel_b200._lib import MmnbError
from molmodel_b200.adjoint import (backward, fit_water, type_gradients, water_fit_gradients, water_site_params,
                                   water_site_types)
from molmodel_b200.md import MDyn
from molmodel_b200.water import EPSILON_O, Q_O_E, SIGMA_O
from oracle.oracle import make_config, port

from adjoint_cases import CASES, CFG, System, directional_fd, directions, grad_key, oracle_eval  # noqa: F401

pytestmark = pytest.mark.gpu

MMNB_ERR_STATE = 6


@pytest.fixture(scope="module", params=CASES, ids=[c[0] for c in CASES])
def case(request):
    name, extra, cfg = request.param
    wb = water_box(6, seed=11)
    s = System(wb, extra)
    # targets: the forces with every charge x 1.04 and the O sigmas + 0.03
    tq = s.q * 1.04
    tsig = np.where(np.arange(s.nsite) % 3 == 0, s.sigma + 0.03, s.sigma)
    targets = oracle_eval(s, cfg, q=tq, sig=tsig)["f"]
    rng = np.random.default_rng(5)
    checks = []
    for label, which, v, h in directions(s, rng):
        fd_u, fd_l = directional_fd(s, cfg, which, v, h, targets)
        checks.append((label, which, v, fd_u, fd_l))
    return name, s, cfg, targets, checks


def site_grads(s, cfg, precision, targets, dl_df=None):
    p = ElecLJ(precision=precision, **cfg).init(s, pairs14=s.pairs14)
    out = p.forward(s.positions)
    g = p.site_gradients(2 * (out["f"] - targets) if dl_df is None else dl_df)
    p.close()
    return out, g


def test_fp64_site_gradients_match_finite_differences(case):
    name, s, cfg, targets, checks = case
    out, g = site_grads(s, cfg, "fp64", targets)
    for label, which, v, fd_u, fd_l in checks:
        k = grad_key(which)
        pu = float(v @ g["du_" + k])
        pl = float(v @ g["dl_" + k])
        assert abs(pu - fd_u) <= 3e-8 * abs(fd_u) + 1e-9, (name, label, pu, fd_u)
        assert abs(pl - fd_l) <= 3e-8 * abs(fd_l) + 1e-9, (name, label, pl, fd_l)


KSUM = [c for c in CASES if "kspace_cutoff" in c[2]]


@pytest.mark.parametrize("name,extra,cfg", KSUM, ids=[c[0] for c in KSUM])
def test_fp64_site_gradients_match_the_restated_oracle_gradients(name, extra, cfg):
    """Site by site against oracle/adjoint_oracle.py (the FP64 CPU restatement,
    itself pinned to central differences on the CPU): 1e-10 of each array's
    largest entry."""
    from oracle.adjoint_oracle import site_gradients as oracle_site_gradients
    wb = water_box(6, seed=11)
    s = System(wb, extra)
    targets = oracle_eval(s, cfg, q=s.q * 1.04)["f"]
    out, g = site_grads(s, cfg, "fp64", targets)
    dl_df = 2 * (out["f"] - targets)
    o = oracle_site_gradients(port(), s, cfg, s.positions, dl_df, pairs14=s.pairs14)
    for key in ("du_dq", "du_dsig", "du_deps", "dl_dq", "dl_dsig", "dl_deps"):
        scale = np.abs(o[key]).max()
        assert np.abs(g[key] - o[key]).max() <= 1e-10 * scale, (name, key)


def test_mixed_site_gradients_match_fp64_for_the_same_loss_gradient(case):
    """The mixed form's backward, given the same dL/dF, differs from the FP64
    one only through the forward's site potentials and fields (FP32 pair
    arithmetic): 2e-5 of the largest term."""
    name, s, cfg, targets, checks = case
    out64, g64 = site_grads(s, cfg, "fp64", targets)
    dl_df = 2 * (out64["f"] - targets)
    _, gm = site_grads(s, cfg, "mixed", targets, dl_df=dl_df)
    for key in ("du_dq", "du_dsig", "du_deps", "dl_dq", "dl_dsig", "dl_deps"):
        scale = np.abs(g64[key]).max()
        assert np.abs(gm[key] - g64[key]).max() <= 2e-5 * scale, (name, key)


def test_uniform_scale_backward_is_the_contracted_site_gradients():
    wb = water_box(6, seed=12)
    s = System(wb)
    cfg = CASES[1][2]
    targets = oracle_eval(s, cfg, q=s.q * 1.02)["f"]
    p = ElecLJ(precision="fp64", **cfg).init(s)
    out = p.forward(s.positions)
    dl_df = 2 * (out["f"] - targets)
    g = p.site_gradients(dl_df)
    f, u, gu, gl = backward(p, s.positions, dl_df)
    p.close()
    assert abs(gu[0] - 2 * out["elec"]) <= 1e-10 * abs(out["elec"])
    for k, (par, key) in enumerate(((s.q, "dq"), (s.sigma, "dsig"), (s.epsilon, "deps"))):
        # bounded by the sum of the terms' sizes (the targets move only the
        # charges, so the loss's sigma sum nearly cancels)
        assert abs(gu[k] - par @ g["du_" + key]) <= 1e-12 * (np.abs(par * g["du_" + key]).sum())
        assert abs(gl[k] - par @ g["dl_" + key]) <= 1e-12 * (np.abs(par * g["dl_" + key]).sum())
    # the same forward again (the FP64 mesh is summed with atomic adds, so to rounding)
    assert np.abs(f - out["f"]).max() <= 1e-12 * np.abs(out["f"]).max()
    assert abs(u - out["total"]) <= 1e-12 * abs(out["total"])


def test_site_gradients_need_the_forward_of_the_same_state():
    wb = water_box(6, seed=13)
    p = ElecLJ(precision="fp64", **CASES[1][2]).init(wb)
    with pytest.raises(MmnbError) as ex:
        p.site_gradients()
    assert ex.value.status == MMNB_ERR_STATE
    p.forward(wb.positions)
    p.site_gradients()
    p.compute(wb.positions)  # another evaluation discards the forward's state
    with pytest.raises(MmnbError) as ex:
        p.site_gradients()
    assert ex.value.status == MMNB_ERR_STATE
    p.forward(wb.positions)
    p.set_params(wb.site_mask, wb.q, wb.sigma, wb.epsilon)
    with pytest.raises(MmnbError) as ex:
        p.site_gradients()
    assert ex.value.status == MMNB_ERR_STATE
    p.close()


# ---- C5: the water parameters over 64 frames ---------------------------------

C5_CFG = dict(rspace_cutoff=9.0, ewald_screening=0.35, use_p3m=True, p3m_assignment_order=5,
              neighbor_list_width=1.0)


def _water_oracle(wb, cfg, theta):
    q, sig, eps = water_site_params(theta, wb.nwater)
    return port().eleclj(make_config(wb.box, **cfg), wb.nsite, wb.groups, wb.exclusions, wb.site_mask, q, sig,
                         eps, wb.rscreen)


@pytest.fixture(scope="module")
def c5():
    """512 waters (L 24.86 A), P3M 24^3; 64 frames 1 ps apart from FP64
    dynamics at 300 K (1 fs steps); targets from the perturbed parameters
    (q_O x 1.05, sigma_O + 0.02 A, epsilon_O x 0.95)."""
    wb = water_box(8, seed=3)
    cfg = dict(C5_CFG, p3m_grid_spacing=wb.box / 24)
    pot = ElecLJ(precision="fp64", **cfg).init(wb)
    md = MDyn(pot, wb.masses, timestep=0.001)
    md.set_state(wb.positions, maxwell_boltzmann(wb, 300.0, seed=5))
    frames = []
    for _ in range(64):
        md.run(1000)
        frames.append(md.state()[0])
    md.close()
    pot.close()
    theta0 = np.array([Q_O_E, SIGMA_O, EPSILON_O])
    target_theta = np.array([Q_O_E * 1.05, SIGMA_O + 0.02, EPSILON_O * 0.95])
    ot = _water_oracle(wb, cfg, target_theta)
    targets = [ot.eval(r)["f"] for r in frames]

    def lu(theta):
        o = _water_oracle(wb, cfg, theta)
        L = U = 0.0
        for r, ft in zip(frames, targets):
            out = o.eval(r)
            L += float(((out["f"] - ft) ** 2).sum())
            U += out["total"]
        return L, U

    # relative steps of about 1e-4 (and twice that, Richardson-extrapolated),
    # rounded to one significant digit so theta +- h stays exact in the six
    # digits the LJ tail keys on
    steps = [float(f"{1e-4 * abs(t):.0e}") for t in theta0]
    fd_l, fd_u = np.zeros(3), np.zeros(3)
    for k in range(3):
        d = []
        for h in (steps[k], 2 * steps[k]):
            tp, tm = theta0.copy(), theta0.copy()
            tp[k] += h
            tm[k] -= h
            (lp, up), (lm, um) = lu(tp), lu(tm)
            d.append(((lp - lm) / (2 * h), (up - um) / (2 * h)))
        fd_l[k] = (4 * d[0][0] - d[1][0]) / 3
        fd_u[k] = (4 * d[0][1] - d[1][1]) / 3
    L0, U0 = lu(theta0)
    return wb, cfg, frames, targets, theta0, target_theta, fd_l, fd_u, L0, U0


# the mixed forward's forces carry ~4e-6 relative error, and the loss
# gradient inherits it through dL/dF = 2 (F - F^target), where F - F^target
# is ~5% of F: ~1e-4 relative
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-7), ("mixed", 3e-4)])
def test_c5_water_parameter_gradients(c5, precision, tol):
    wb, cfg, frames, targets, theta0, _, fd_l, fd_u, L0, U0 = c5
    pot = ElecLJ(precision=precision, **cfg).init(wb)
    L, dl, U, du = water_fit_gradients(pot, frames, targets)
    pot.close()
    assert abs(L - L0) < (1e-8 if precision == "fp64" else 1e-3) * L0
    assert abs(U - U0) < (1e-10 if precision == "fp64" else 5e-5) * abs(U0)
    for k in range(3):
        assert abs(du[k] - fd_u[k]) <= tol * abs(fd_u[k]), (k, du, fd_u)
        assert abs(dl[k] - fd_l[k]) <= tol * abs(fd_l[k]), (k, dl, fd_l)


def test_c5_one_evaluation_per_frame(c5):
    wb, cfg, frames, targets = c5[:4]
    pot = ElecLJ(precision="fp64", **cfg).init(wb)
    pot.compute(frames[0])
    before = pot.counters()
    water_fit_gradients(pot, frames[:8], targets[:8])
    after = pot.counters()
    pot.close()
    assert after[1] - before[1] == 8  # evaluations counted by the device


def test_c5_type_gradients_sum_the_sites(c5):
    wb, cfg, frames, targets = c5[:4]
    pot = ElecLJ(precision="fp64", **cfg).init(wb)
    out = pot.forward(frames[0])
    g = pot.site_gradients(2 * (out["f"] - targets[0]))
    pot.close()
    t = type_gradients(g, water_site_types(wb.nwater), "du")
    assert set(t) == {"O", "H"}
    assert t["H"][1] == 0 and t["H"][2] == 0  # no LJ on H
    # dU/dq_type . q_type over the types = 2 U_elec (charges in e)
    q_o, q_h = Q_O_E, -Q_O_E / 2
    assert abs(t["O"][0] * q_o + t["H"][0] * q_h - 2 * out["elec"]) <= 1e-10 * abs(out["elec"])


def test_c5_force_matching_fit_recovers_the_target_parameters(c5):
    """L-BFGS on the adjoint gradients from theta0 to the parameters the
    targets were made with (8 of the 64 frames)."""
    wb, cfg, frames, targets, theta0, target_theta = c5[:6]
    pot = ElecLJ(precision="fp64", **cfg).init(wb)
    theta, L, calls = fit_water(pot, wb.site_mask, frames[:8], targets[:8], theta0, maxiter=60)
    pot.close()
    assert np.abs(theta / target_theta - 1).max() < 1e-6, (theta, target_theta, L, calls)

"""Adjoint (mmnb_backward) for the water parameters (q_O, sigma_O, epsilon_O):
gradients of the total energy and of a force-matching loss against central
finite differences of the FP64 oracle (relative step 1e-4), for the FP64 and
the mixed forward."""
import numpy as np
import pytest

from molmodel_b200 import ElecLJ, maxwell_boltzmann, water_box
from molmodel_b200.adjoint import water_fit_gradients
from molmodel_b200.md import MDyn
from molmodel_b200.units import e_to_charge_unit
from molmodel_b200.water import EPSILON_O, Q_O_E, SIGMA_O
from oracle.oracle import make_config, port

pytestmark = pytest.mark.gpu


def _params(wb, theta):
    q_o, s_o, e_o = theta
    q = np.tile([q_o, -q_o / 2, -q_o / 2], wb.nwater)
    sig = np.zeros(wb.nsite)
    eps = np.zeros(wb.nsite)
    sig[0::3] = s_o
    eps[0::3] = e_o
    return e_to_charge_unit(q), sig, eps


def _oracle(wb, cfg, theta):
    q, sig, eps = _params(wb, theta)
    return port().eleclj(make_config(wb.box, **cfg), wb.nsite, wb.groups, wb.exclusions, wb.site_mask, q, sig, eps,
                         wb.rscreen)


@pytest.fixture(scope="module")
def case():
    """512 waters (L 24.86 A), P3M 24^3; three frames 40 fs apart from FP64
    dynamics at 300 K; targets from the perturbed parameters (q_O x 1.05,
    sigma_O + 0.02 A, epsilon_O x 0.95)."""
    wb = water_box(8, seed=3)
    cfg = dict(rspace_cutoff=9.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=wb.box / 24,
               p3m_assignment_order=5, neighbor_list_width=1.0)
    pot = ElecLJ(precision="fp64", **cfg).init(wb)
    md = MDyn(pot, wb.masses, timestep=0.001)
    md.set_state(wb.positions, maxwell_boltzmann(wb, 300.0, seed=5))
    frames = []
    for _ in range(3):
        md.run(40)
        frames.append(md.state()[0])
    md.close()
    pot.close()
    theta0 = np.array([Q_O_E, SIGMA_O, EPSILON_O])
    target_theta = np.array([Q_O_E * 1.05, SIGMA_O + 0.02, EPSILON_O * 0.95])
    ot = _oracle(wb, cfg, target_theta)
    targets = [ot.eval(r)["f"] for r in frames]
    # central differences of L and U on the oracle
    def lu(theta):
        o = _oracle(wb, cfg, theta)
        L = U = 0.0
        for r, ft in zip(frames, targets):
            out = o.eval(r)
            L += float(((out["f"] - ft) ** 2).sum())
            U += out["total"]
        return L, U
    # central differences with relative steps of about 1e-4 (and twice that,
    # combined by Richardson extrapolation so the O(h^2) truncation error of
    # the quadratic loss drops out), rounded to one significant digit: the
    # reference keys the LJ tail on sigma and epsilon printed with %12.6g
    # (src/eleclj.cpp:283-308), so theta +- h must stay exact in six digits
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
    return wb, cfg, frames, targets, theta0, fd_l, fd_u, L0, U0


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-6), ("mixed", 2e-3)])
def test_gradients_match_finite_differences(case, precision, tol):
    wb, cfg, frames, targets, theta0, fd_l, fd_u, L0, U0 = case
    pot = ElecLJ(precision=precision, **cfg).init(wb)
    L, dl, U, du = water_fit_gradients(pot, frames, targets, theta0)
    pot.close()
    assert abs(L - L0) < 1e-6 * L0 if precision == "fp64" else abs(L - L0) < 1e-3 * L0
    assert abs(U - U0) < 1e-9 * abs(U0) if precision == "fp64" else abs(U - U0) < 1e-4 * abs(U0)
    for k in range(3):
        assert abs(du[k] - fd_u[k]) <= tol * abs(fd_u[k]) + 1e-9 * abs(U0), (k, du, fd_u)
        assert abs(dl[k] - fd_l[k]) <= tol * abs(fd_l[k]), (k, dl, fd_l)

"""Parameter gradients for force-field fitting (mmnb_forward, then
mmnb_site_gradients), and a force-matching fit driven by them.

The reference fits per-type parameters: WeakCouple::update
(src/msimprog.cpp:855-876) rescales the sigma and epsilon of named types by
feedback on density and energy per molecule, and BCIFit (src/bcifit.cpp:44-123)
fits bond charge increments by Nelder-Mead; ElecLJ::types_changed
(src/eleclj.cpp:440-503) maps each type's fixed charge (in e), sigma and
epsilon to its sites.  The library returns per-site gradients of the energy
and of any loss of the forces; type_gradients sums them over each type's
sites through that map, so a fit can take gradient steps (fit_water below
runs L-BFGS on them) instead of simplex or feedback moves.

For the rigid 3-site water model the fitted parameters are
theta = (q_O [e], sigma_O [A], epsilon_O [kcal/mol]) with q_H = -q_O/2 and LJ
on O only.
"""
import ctypes

import numpy as np

from ._lib import check, load
from .units import e_to_charge_unit

_dp = ctypes.POINTER(ctypes.c_double)


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def backward(pot, r, dl_df=None):
    """mmnb_backward: one forward pass and the gradients with respect to
    uniform scales of all charges, sigmas and epsilons.  Returns forces,
    energy, dU/dscales and sum_i dl_df_i . dF_i/dscales."""
    r = np.ascontiguousarray(r, dtype=np.float64)
    g = None if dl_df is None else np.ascontiguousarray(dl_df, dtype=np.float64)
    f = np.zeros((pot.nsite, 3))
    u = ctypes.c_double(0.0)
    gu = np.zeros(3)
    gl = np.zeros(3)
    check(load().mmnb_backward(pot._h, _d(r), _d(g), _d(f), ctypes.byref(u), _d(gu), _d(gl)), pot._h)
    return f, u.value, gu, gl


def type_gradients(grads, site_types, of="du"):
    """Per-type gradients from per-site ones, for parameters mapped to sites as
    ElecLJ::types_changed maps them (a site takes its type's charge, sigma and
    epsilon).  grads: site_gradients()'s dict; of: "du" (energy) or "dl"
    (loss).  Returns {type: array([d/dcharge (per e), d/dsigma, d/depsilon])}."""
    types = np.asarray(site_types)
    cu = e_to_charge_unit(1.0)
    out = {}
    for t in np.unique(types):
        m = types == t
        out[t.item() if hasattr(t, "item") else t] = np.array(
            [cu * grads[of + "_dq"][m].sum(), grads[of + "_dsig"][m].sum(), grads[of + "_deps"][m].sum()])
    return out


def water_site_types(nwater):
    return np.array(["O", "H", "H"] * nwater)


def water_theta_gradient(per_type):
    """d/d(q_O, sigma_O, epsilon_O) from the O and H type gradients, with the
    tie q_H = -q_O/2."""
    o, hh = per_type["O"], per_type.get("H", np.zeros(3))
    return np.array([o[0] - 0.5 * hh[0], o[1], o[2]])


def water_site_params(theta, nwater):
    """Site charges (charge units), sigmas and epsilons of rigid water at
    theta = (q_O [e], sigma_O, epsilon_O)."""
    q_o, s_o, e_o = theta
    q = e_to_charge_unit(np.tile([q_o, -q_o / 2, -q_o / 2], nwater))
    sig = np.zeros(3 * nwater)
    eps = np.zeros(3 * nwater)
    sig[0::3] = s_o
    eps[0::3] = e_o
    return q, sig, eps


def water_fit_gradients(pot, frames, targets):
    """Force-matching loss L = sum_frames sum_i |F_i(theta) - F_i^target|^2 and
    total energy U = sum_frames U, with their gradients with respect to
    theta = (q_O, sigma_O, epsilon_O) at the potential's current parameters.
    One evaluation per frame: mmnb_forward gives F, and the backward pass
    (mmnb_site_gradients) takes dL/dF = 2 (F - F^target).  Returns
    (L, dL/dtheta, U, dU/dtheta)."""
    types = water_site_types(pot.nsite // 3)
    L = U = 0.0
    dl = np.zeros(3)
    du = np.zeros(3)
    for r, ft in zip(frames, targets):
        out = pot.forward(r)
        diff = out["f"] - ft
        g = pot.site_gradients(2 * diff)
        L += float((diff ** 2).sum())
        U += out["total"]
        dl += water_theta_gradient(type_gradients(g, types, "dl"))
        du += water_theta_gradient(type_gradients(g, types, "du"))
    return L, dl, U, du


def fit_water(pot, site_mask, frames, targets, theta0, maxiter=50, gtol=1e-10):
    """Force matching of theta = (q_O, sigma_O, epsilon_O) by L-BFGS on the
    adjoint gradients (scipy.optimize, relative coordinates theta / theta0).
    Leaves the potential at the fitted parameters; returns (theta, L, the
    number of evaluations of L and its gradient)."""
    from scipy.optimize import minimize
    theta0 = np.asarray(theta0, dtype=np.float64)
    nwater = pot.nsite // 3
    calls = [0]

    def fun(x):
        theta = theta0 * x
        q, sig, eps = water_site_params(theta, nwater)
        pot.set_params(site_mask, q, sig, eps)
        L, dl, _, _ = water_fit_gradients(pot, frames, targets)
        calls[0] += 1
        return L, dl * theta0

    res = minimize(fun, np.ones(3), jac=True, method="L-BFGS-B",
                   options=dict(maxiter=maxiter, gtol=gtol, ftol=1e-15))
    theta = theta0 * res.x
    pot.set_params(site_mask, *water_site_params(theta, nwater))
    return theta, float(res.fun), calls[0]

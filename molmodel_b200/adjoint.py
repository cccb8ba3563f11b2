"""Gradients for water force-field fitting through mmnb_backward.

The reference fits per-type parameters (WeakCouple, src/msimprog.cpp:855-876;
BCIFit, src/bcifit.cpp:44-123).  For the rigid 3-site water model the fitted
parameters are theta = (q_O [e], sigma_O [A], epsilon_O [kcal/mol]) with
q_H = -q_O/2 and LJ on O only; every site charge is proportional to q_O and
every LJ sigma/epsilon is sigma_O/epsilon_O, so d/dtheta_k = (d/dscale_k) /
theta_k with the scale gradients the library returns.
"""
import ctypes

import numpy as np

from ._lib import check, load

_dp = ctypes.POINTER(ctypes.c_double)


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def backward(pot, r, dl_df=None):
    """One forward + backward pass: returns forces, energy, dU/dscales and
    sum_i dl_df_i . dF_i/dscales (scales of all charges, sigmas, epsilons)."""
    r = np.ascontiguousarray(r, dtype=np.float64)
    g = None if dl_df is None else np.ascontiguousarray(dl_df, dtype=np.float64)
    f = np.zeros((pot.nsite, 3))
    u = ctypes.c_double(0.0)
    gu = np.zeros(3)
    gl = np.zeros(3)
    check(load().mmnb_backward(pot._h, _d(r), _d(g), _d(f), ctypes.byref(u), _d(gu), _d(gl)), pot._h)
    return f, u.value, gu, gl


def water_fit_gradients(pot, frames, targets, theta):
    """Force-matching loss L = sum_frames sum_i |F_i(theta) - F_i^target|^2 and
    total energy U = sum_frames U, with their gradients with respect to
    theta = (q_O, sigma_O, epsilon_O) at the potential's current parameters
    (which must be theta).  Returns (L, dL/dtheta, U, dU/dtheta)."""
    theta = np.asarray(theta, dtype=np.float64)
    L = 0.0
    U = 0.0
    dl = np.zeros(3)
    du = np.zeros(3)
    for r, ft in zip(frames, targets):
        f, _, _, _ = backward(pot, r)          # forces at theta
        diff = f - ft
        f2, u, gu, gl = backward(pot, r, 2 * diff)
        L += float((diff ** 2).sum())
        U += u
        dl += gl
        du += gu
    return L, dl / theta, U, du / theta

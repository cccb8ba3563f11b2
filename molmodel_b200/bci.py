"""Bond charge increments solved self-consistently with the GPU potential.

Restates ElecLJ::update_q and ElecLJ::solve_for_bci (src/eleclj.cpp:809-866):
each bond (a, b) moves q0 + dq from site b to site a; dq is iterated as
    dq = (phi_b - phi_a) / k      (phi: site potentials, minus E_ext . r)
with all bonds updated from the same potentials and the charges rebuilt
after each sweep, until every dq changes by less than `tolerance` (relative
when |dq| > tolerance), at most `max_iterations` sweeps.  Bonds with k = 0
keep dq = 0.  The self energy of the increments is sum 0.5 k dq^2
(BondChargeIncrement::self_energy, include/eleclj.hpp:282).  Units are the
reference's internal ones (charges in sqrt(kcal A/mol)).
"""
import numpy as np

from ._lib import MmnbError


def site_charges(q_site0, bonds, q0, dq):
    """ElecLJ::update_q: base charges plus each bond's increment."""
    q = np.array(q_site0, dtype=np.float64)
    for (a, b), c in zip(bonds, np.asarray(q0) + np.asarray(dq)):
        q[a] += c
        q[b] -= c
    return q


def solve_for_bci(potential, system, r, bonds, k, q0, dq=None, external_field=None, tolerance=1e-10,
                  max_iterations=1000, site_phi=None):
    """Iterate the increments to self-consistency on `potential` (an ElecLJ
    bound to `system`, whose charges it resets each sweep).  Returns (dq,
    charges, sweeps).  `site_phi(q)` may replace the GPU evaluation (for
    checks against another implementation of the potentials)."""
    bonds = [tuple(b) for b in bonds]
    k = np.asarray(k, dtype=np.float64)
    q0 = np.asarray(q0, dtype=np.float64)
    dq = np.zeros(len(bonds)) if dq is None else np.array(dq, dtype=np.float64)
    r = np.asarray(r, dtype=np.float64).reshape(-1, 3)
    q_base = np.asarray(system.q, dtype=np.float64)
    q = site_charges(q_base, bonds, q0, dq)

    def phi_of(q):
        if site_phi is not None:
            return site_phi(q)
        potential.set_params(system.site_mask, q, system.sigma, system.epsilon, system.rscreen)
        return potential.compute(r, want_fields=True)["phi"]

    converged = False
    it = 0
    while not converged and it < max_iterations:
        converged = True
        phi = np.array(phi_of(q))
        if external_field is not None and np.linalg.norm(external_field) > 0:
            phi -= r @ np.asarray(external_field, dtype=np.float64)
        for i, (a, b) in enumerate(bonds):
            if abs(k[i]) < 1e-10:
                dq[i] = 0
                continue
            last = dq[i]
            dq[i] = (phi[b] - phi[a]) / k[i]
            if not np.isfinite(dq[i]):
                raise MmnbError(1, "solve_for_bci: NaN detected")
            if abs(dq[i]) > tolerance:
                if abs(last - dq[i]) / abs(dq[i]) > tolerance:
                    converged = False
            elif abs(last - dq[i]) > tolerance:
                converged = False
        q = site_charges(q_base, bonds, q0, dq)
        it += 1
    if not converged:
        raise MmnbError(1, f"solve_for_bci: did not converge to tolerance of {tolerance} within "
                           f"{max_iterations} iterations")
    return dq, q, it


def self_energy(k, dq):
    return float(0.5 * np.sum(np.asarray(k) * np.asarray(dq) ** 2))

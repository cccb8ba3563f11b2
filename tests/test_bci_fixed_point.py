"""Bond charge increments (molmodel_b200/bci.py, restating ElecLJ::update_q and
ElecLJ::solve_for_bci, src/eleclj.cpp:809-866) pinned on the CPU by what the
reference's iteration converges to, with the oracle's site potentials:

- at convergence every bond satisfies the reference's update
  dq = (phi_b - phi_a) / k (src/eleclj.cpp:834-836), phi evaluated afresh at
  the final charges, which are the base charges plus update_q's increments;
- that fixed point is the solution of the linear system the iteration solves:
  the site potentials are linear in the charges (pair terms, self and
  neutralising terms), phi = G q - E.r, so with C the bonds' +-1 incidence
  (k I + C^T G C) dq = C^T (G q_base - E.r), G built column by column from
  unit-charge evaluations.
"""
import numpy as np

from molmodel_b200.bci import site_charges, solve_for_bci
from molmodel_b200.water import water_box
from oracle.oracle import make_config, port

CFG = dict(rspace_cutoff=5.5, ewald_screening=0.45, kspace_cutoff=5.0)


def oracle_phi(wb, q):
    o = port().eleclj(make_config(wb.box, **CFG), wb.nsite, wb.groups, wb.exclusions, wb.site_mask, q,
                      wb.sigma, wb.epsilon, wb.rscreen)
    return o.eval(wb.positions)["phi"]


def test_bci_converges_to_the_references_fixed_point():
    wb = water_box(4, seed=21)
    bonds = [(3 * w, 3 * w + h) for w in range(wb.nwater) for h in (1, 2)]
    rng = np.random.default_rng(3)
    k = rng.uniform(300.0, 500.0, len(bonds))
    k[5] = 0.0  # a bond with no stiffness keeps dq = 0
    q0 = rng.normal(scale=0.05, size=len(bonds))
    field = np.array([0.02, -0.01, 0.05])
    r = wb.positions
    dq, q, it = solve_for_bci(None, wb, r, bonds, k, q0, external_field=field, tolerance=1e-12,
                              site_phi=lambda qq: oracle_phi(wb, qq))
    assert it > 3 and dq[5] == 0.0 and np.abs(dq).max() > 1e-4
    # update_q's charges
    assert np.array_equal(q, site_charges(wb.q, bonds, q0, dq))
    # the reference's update holds at the final charges
    phi = oracle_phi(wb, q) - r @ field
    a = np.array([b[0] for b in bonds])
    b = np.array([b[1] for b in bonds])
    stiff = k > 0
    resid = dq[stiff] - (phi[b] - phi[a])[stiff] / k[stiff]
    assert np.abs(resid).max() < 1e-9 * np.abs(dq).max()

    # the same increments from the linear system, G from unit charges
    n = wb.nsite
    G = np.empty((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        G[:, j] = oracle_phi(wb, e)
    C = np.zeros((n, len(bonds)))
    C[a, np.arange(len(bonds))] = 1.0
    C[b, np.arange(len(bonds))] = -1.0
    q_base = site_charges(wb.q, bonds, q0, np.zeros(len(bonds)))
    rhs = -(C.T @ (G @ q_base - r @ field))
    A = np.diag(k) + C.T @ G @ C
    # a bond with k = 0 is held at dq = 0: its row and column leave the system
    keep = np.flatnonzero(stiff)
    dq_lin = np.zeros(len(bonds))
    dq_lin[keep] = np.linalg.solve(A[np.ix_(keep, keep)], rhs[keep])
    assert np.abs(dq - dq_lin).max() < 1e-8 * np.abs(dq_lin).max()

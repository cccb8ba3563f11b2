"""Bond charge increments (ElecLJ::solve_for_bci restated in
molmodel_b200/bci.py) solved with the GPU site potentials against the same
iteration on the oracle's potentials."""
import numpy as np
import pytest

from molmodel_b200 import ElecLJ, water_box
from molmodel_b200.bci import self_energy, solve_for_bci
from oracle.oracle import make_config, port

pytestmark = pytest.mark.gpu


def test_bci_matches_the_oracle_iteration():
    wb = water_box(6, seed=8)
    cfg = dict(rspace_cutoff=9.0, ewald_screening=0.35, kspace_cutoff=7.0)
    bonds = [(3 * w, 3 * w + h) for w in range(wb.nwater) for h in (1, 2)]
    k = np.full(len(bonds), 400.0)
    q0 = np.zeros(len(bonds))
    field = np.array([0.0, 0.0, 0.05])
    pot = ElecLJ(precision="fp64", **cfg).init(wb)
    dq, q, it = solve_for_bci(pot, wb, wb.positions, bonds, k, q0, external_field=field, tolerance=1e-10)
    pot.close()

    def oracle_phi(qq):
        o = port().eleclj(make_config(wb.box, **cfg), wb.nsite, wb.groups, wb.exclusions, wb.site_mask, qq,
                          wb.sigma, wb.epsilon, wb.rscreen)
        return o.eval(wb.positions)["phi"]

    dq_o, q_o, it_o = solve_for_bci(None, wb, wb.positions, bonds, k, q0, external_field=field, tolerance=1e-10,
                                    site_phi=oracle_phi)
    assert it == it_o and it > 2
    assert np.abs(dq - dq_o).max() < 1e-9 * np.abs(dq_o).max()
    assert abs(self_energy(k, dq) - self_energy(k, dq_o)) < 1e-9 * self_energy(k, dq_o)
    # the increments respond to the field: H sites along +z gain charge
    assert np.abs(dq).max() > 0

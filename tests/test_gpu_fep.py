"""FEP (molmodel_b200/fep.py): the energy difference of FEP::update against
the oracle's, and lambda windows run as one batch."""
import numpy as np
import pytest

from molmodel_b200 import ElecLJ, water_box
from molmodel_b200.fep import energy_difference, lambda_params, run_windows
from oracle.oracle import make_config, port

pytestmark = pytest.mark.gpu


def _states(wb):
    p1 = dict(q=wb.q, sigma=wb.sigma, epsilon=wb.epsilon, rscreen=wb.rscreen, site_mask=wb.site_mask)
    p2 = dict(p1, q=wb.q * 0.9, sigma=wb.sigma * 1.01, epsilon=wb.epsilon * 1.1)
    return p1, p2


def test_energy_difference_matches_oracle():
    wb = water_box(6, seed=4)
    cfg = dict(rspace_cutoff=9.0, ewald_screening=0.35, kspace_cutoff=7.0)
    p1, p2 = _states(wb)
    pot = ElecLJ(precision="fp64", **cfg).init(wb)
    du = energy_difference(pot, p1, p2, wb.positions, 0.25, 0.5)
    pot.close()
    us = []
    for lam in (0.25, 0.5):
        p = lambda_params(p1, p2, lam)
        o = port().eleclj(make_config(wb.box, **cfg), wb.nsite, wb.groups, wb.exclusions, p["site_mask"], p["q"],
                          p["sigma"], p["epsilon"], p["rscreen"])
        us.append(o.eval(wb.positions)["total"])
    assert abs(du - (us[1] - us[0])) < 1e-9 * abs(us[0])


def test_windows_run_as_one_batch():
    wb = water_box(6, seed=5)
    cfg = dict(rspace_cutoff=9.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=wb.box / 18,
               p3m_assignment_order=5, neighbor_list_width=0.3)
    p1, p2 = _states(wb)
    res = run_windows(wb, p1, p2, [0.0, 0.5, 1.0], cfg, steps=200, sample_every=50, dt=0.001)
    assert res["samples_per_window"] == 4
    assert np.isfinite(res["total_forward"]) and np.isfinite(res["total_backward"])

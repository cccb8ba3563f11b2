"""Launch tuning (mmnb_autotune / mmnb_set_tuning) changes no result: every
combination of the choices gives bitwise the same mixed-form forces and
energy, and the tuner keeps valid choices."""
import itertools

import numpy as np
import pytest

from molmodel_b200 import ElecLJ, water_box

pytestmark = pytest.mark.gpu


def _pot(wb):
    return ElecLJ(precision="mixed", rspace_cutoff=9.0, ewald_screening=0.35, use_p3m=True,
                  p3m_grid_spacing=wb.box / 32, p3m_assignment_order=5, neighbor_list_width=1.5).init(wb)


def test_every_tuning_gives_the_same_result():
    wb = water_box(10, seed=6)
    p = _pot(wb)
    ref = p.compute(wb.positions)
    for combo in itertools.product((4, 5), (0, 1, 2), (1, 0)):
        p.tuning = combo
        assert p.tuning == combo
        g = p.compute(wb.positions)   # host call: graph replay with these choices
        g2 = p.compute(wb.positions)
        assert np.array_equal(g["f"], ref["f"]) and np.array_equal(g2["f"], ref["f"]), combo
        assert g["total"] == ref["total"], combo
    p.close()


def test_autotune_keeps_valid_choices():
    wb = water_box(8, seed=7)
    p = _pot(wb)
    before = p.compute(wb.positions)
    t = p.autotune(wb.positions, iters=5)
    assert t[0] in (4, 5) and t[1] in (0, 1, 2) and t[2] in (0, 1)
    after = p.compute(wb.positions)
    assert np.array_equal(before["f"], after["f"])
    p.close()

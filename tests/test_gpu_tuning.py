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
        assert p.tuning[:3] == combo
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
    assert t[0] in (4, 5) and t[1] in (0, 1, 2) and t[2] in (0, 1) and t[3] in (8, 10, 12)
    after = p.compute(wb.positions)
    assert np.array_equal(before["f"], after["f"])
    p.close()


def test_fp64_water_warps_give_the_same_result():
    """The FP64 rigid-water kernel's rows are summed in a fixed order whichever
    warp takes them: every warps-per-block choice gives the same bits.  (The
    Ewald k-sum, whose sums run in a fixed order too; the FP64 P3M mesh is summed
    with atomic adds, which differ from run to run at rounding.)"""
    wb = water_box(10, seed=8)
    p = ElecLJ(precision="fp64", rspace_cutoff=9.0, ewald_screening=0.35, kspace_cutoff=6.0,
               neighbor_list_width=1.5).init(wb)
    ref = None
    for warps in (12, 10, 8):
        p.tuning = (5, 2, 0, warps)
        assert p.tuning[3] == warps
        g = p.compute(wb.positions, want_fields=True)
        if ref is None:
            ref = g
        assert np.array_equal(g["f"], ref["f"]) and np.array_equal(g["phi"], ref["phi"]), warps
        assert g["total"] == ref["total"], warps
    p.close()

"""Pruned rows of the rigid-water kernel: between list builds the kernel reads
rows cut to rc + width/3 and makes them again from the full rows whenever the
two largest anchor moves since the last prune exceed width/3.  Every pair
within rc stays listed, so the mixed form's fixed-point results are bitwise
those of evaluating the full rows.  Checked along a trajectory of growing
rigid-body moves against a handle that rebuilds (and so re-prunes) at every
evaluation."""
import numpy as np
import pytest

from molmodel_b200 import ElecLJ, water_box

pytestmark = pytest.mark.gpu


def _cfg(wb, **kw):
    d = dict(rspace_cutoff=9.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=wb.box / 24,
             p3m_assignment_order=5, neighbor_list_width=1.5)
    d.update(kw)
    return d


def test_pruned_rows_give_the_full_rows_bits():
    wb = water_box(8, seed=11)
    rng = np.random.default_rng(3)
    lazy = ElecLJ(precision="mixed", **_cfg(wb)).init(wb)
    eager = ElecLJ(precision="mixed", rebuild_interval=1, **_cfg(wb)).init(wb)
    r = wb.positions.copy()
    nw = wb.nwater
    for step in range(40):
        if step:
            # every molecule moves rigidly by up to 0.17 A per step (a random
            # walk): the pruned rows are remade every few steps, the list
            # rebuilt every ten or so
            shift = rng.uniform(-0.1, 0.1, size=(nw, 1, 3))
            r = (r.reshape(nw, 3, 3) + shift).reshape(-1, 3)
        a = lazy.compute(r)
        b = eager.compute(r)
        assert np.array_equal(a["f"], b["f"]), step
        assert a["total"] == b["total"], step
    rebuilds, evals = lazy.counters()
    assert evals == 40 and 1 < rebuilds < 40
    lazy.close()
    eager.close()

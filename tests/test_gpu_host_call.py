"""The host-array call (mmnb_compute, Potential::add_to_energy_and_forces) after
its first evaluation replays a graph of its own, with the positions copied in
pieces on a stream of their own and the mixed charge assignment of each piece
started as it lands.  Along a trajectory -- new positions every call, list
rebuilds on the way -- every call must give what a fresh potential gives at
those positions: bitwise in the mixed form (fixed-point sums), to 1e-12 in the
FP64 form (its mesh sums are FP64 atomics)."""
import numpy as np
import pytest

from conftest import rel_max
from molmodel_b200 import ElecLJ, water_box

pytestmark = pytest.mark.gpu


def p3m(box, mesh, **kw):
    d = dict(rspace_cutoff=9.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=box / mesh,
             p3m_assignment_order=5, neighbor_list_width=1.0)
    d.update(kw)
    return d


@pytest.mark.parametrize("side", [1, 0])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_host_call_reads_each_calls_positions(precision, side):
    wb = water_box(8, seed=11)
    cfg = p3m(wb.box, 24)
    p = ElecLJ(precision=precision, rebuild_interval=3, **cfg).init(wb)
    t = p.tuning
    p.tuning = (t[0], t[1], side)
    rng = np.random.default_rng(5)
    r = wb.positions.copy()
    for _ in range(7):
        r = r + rng.normal(scale=0.03, size=r.shape)
        f = np.zeros_like(r)
        u = p.add_to_energy_and_forces(0.0, f, r)
        fresh = ElecLJ(precision=precision, **cfg).init(wb).compute(r)
        if precision == "mixed":
            assert np.array_equal(f, fresh["f"])
            assert u == fresh["total"]
        else:
            assert rel_max(f, fresh["f"]) < 1e-12
            assert abs(u - fresh["total"]) <= 1e-12 * abs(fresh["total"])
    rebuilds, evaluations = p.counters()
    assert evaluations == 7 and rebuilds >= 3


def test_host_call_with_the_ewald_sum_and_without_kspace():
    """The paths without a mesh branch wait for every piece before the list check."""
    wb = water_box(6, seed=12)
    rng = np.random.default_rng(6)
    for cfg in (dict(rspace_cutoff=8.0, ewald_screening=0.35, kspace_cutoff=6.0),
                dict(rspace_cutoff=8.0, ewald_screening=0.35, include_kspace=False)):
        p = ElecLJ(precision="mixed", **cfg).init(wb)
        r = wb.positions.copy()
        for _ in range(4):
            r = r + rng.normal(scale=0.03, size=r.shape)
            f = np.zeros_like(r)
            u = p.add_to_energy_and_forces(0.0, f, r)
            fresh = ElecLJ(precision="mixed", **cfg).init(wb).compute(r)
            assert np.array_equal(f, fresh["f"]) and u == fresh["total"]

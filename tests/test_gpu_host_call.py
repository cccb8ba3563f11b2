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


def test_host_call_after_an_asynchronous_device_evaluation():
    """A device-array evaluation still in flight on the handle's stream (energy
    left in the handle's own buffer) does not stand in for the host call that
    follows it: the host call returns its own positions' energy and forces."""
    import torch
    wb = water_box(8, seed=13)
    cfg = p3m(wb.box, 24)
    p = ElecLJ(precision="mixed", **cfg).init(wb)
    s = torch.cuda.Stream()
    p.set_stream(s.cuda_stream)
    rng = np.random.default_rng(7)
    r1 = wb.positions + rng.normal(scale=0.03, size=wb.positions.shape)
    r2 = wb.positions + rng.normal(scale=0.03, size=wb.positions.shape)
    p.compute(r1)  # the host call's graph exists from here on
    d_r = torch.tensor(r2.reshape(-1), dtype=torch.float64, device="cuda")
    d_f = torch.zeros(3 * wb.nsite, dtype=torch.float64, device="cuda")
    fresh = ElecLJ(precision="mixed", **cfg).init(wb).compute(r1)
    other = ElecLJ(precision="mixed", **cfg).init(wb).compute(r2)
    assert other["total"] != fresh["total"]
    for _ in range(3):
        for _ in range(4):
            p.compute_device(d_r.data_ptr(), d_f.data_ptr(), 0)
        f = np.zeros_like(r1)
        u = p.add_to_energy_and_forces(0.0, f, r1)
        assert u == fresh["total"]
        assert np.array_equal(f, fresh["f"])
    torch.cuda.synchronize()

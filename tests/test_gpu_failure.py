"""Failure paths, each made on the host: a box crowded past the neighbour rows'
capacity, a non-finite coordinate, and a volume move the cutoff no longer
fits.  The reference calls die() or grows its rows on the host (src/pbin.c:41-50,
src/eleclj.cpp:168-182); here the host call retries or returns a status, the
device path reports through mmnb_check, and the handle stays usable.

Every device index stays in range whatever the coordinates (float-to-int
conversions give 0 for NaN and saturate; cell and mesh indices are wrapped
into range; row writes stop at the capacity), so these cases fault nothing.
"""
import numpy as np
import pytest

from conftest import rel_max
from molmodel_b200 import ElecLJ, water_box
from molmodel_b200._lib import MmnbError
from oracle.oracle import make_config, port, reference

pytestmark = pytest.mark.gpu

TOL = 1e-10
MMNB_ERR_CUTOFF, MMNB_ERR_OVERFLOW, MMNB_ERR_STATE, MMNB_ERR_DEVICE = 4, 5, 6, 8


def cfg(wb):
    return dict(rspace_cutoff=9.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=wb.box / 24,
                p3m_assignment_order=5, neighbor_list_width=1.0)


def crowded(wb, f=0.6):
    """Molecules moved rigidly so their centres sit in a cube f times the box
    edge around the box centre: about 1/f^3 the density there, rows several
    times longer than the capacity sized for the uniform box."""
    r = wb.positions.reshape(-1, 3, 3)
    m = wb.masses.reshape(-1, 3)
    com = (r * m[:, :, None]).sum(1) / m.sum(1)[:, None]
    c = 0.5 * wb.box
    return (r + ((c + f * (com - c)) - com)[:, None, :]).reshape(-1, 3)


def oracle_eval(wb, r, cfgd):
    lib = reference() or port()
    o = lib.eleclj(make_config(wb.box, **cfgd), wb.nsite, wb.groups, wb.exclusions, wb.site_mask, wb.q, wb.sigma,
                   wb.epsilon, wb.rscreen)
    return o.eval(r)


def test_row_overflow_host_call_grows_rows_and_evaluates_again():
    wb = water_box(8, seed=7)
    c = cfg(wb)
    r = crowded(wb)
    p = ElecLJ(precision="fp64", **c).init(wb)
    g = p.compute(r)
    o = oracle_eval(wb, r, c)
    assert rel_max(g["f"], o["f"]) < TOL
    assert abs(g["total"] - o["total"]) <= TOL * abs(o["total"])
    rebuilds, _ = p.counters()
    assert rebuilds == 2  # the list cut at the capacity, then the full one
    truncated, _ = p.check()
    assert truncated == 0  # the evaluation on cut rows was not returned
    p.close()


def test_row_overflow_on_the_device_path_is_reported_and_repaired():
    import torch
    wb = water_box(8, seed=7)
    c = cfg(wb)
    p = ElecLJ(precision="fp64", **c).init(wb)
    p.compute(wb.positions)  # rows sized for the uniform box
    dev = torch.device("cuda", 0)
    d_r = torch.tensor(wb.positions.reshape(-1), dtype=torch.float64, device=dev)
    d_f = torch.zeros(3 * wb.nsite, dtype=torch.float64, device=dev)
    d_e = torch.zeros(8, dtype=torch.float64, device=dev)
    p.graph_capture(d_r.data_ptr(), d_f.data_ptr(), d_e.data_ptr())
    r = crowded(wb)
    d_r.copy_(torch.from_numpy(r.reshape(-1)))
    torch.cuda.synchronize(dev)
    p.compute_device(d_r.data_ptr(), d_f.data_ptr(), d_e.data_ptr())  # rebuilds onto cut rows
    with pytest.raises(MmnbError) as ex:
        p.check()
    assert ex.value.status == MMNB_ERR_OVERFLOW
    # the graph captured before holds the old rows
    with pytest.raises(MmnbError) as ex:
        p.graph_launch()
    assert ex.value.status == MMNB_ERR_STATE
    d_f.zero_()
    p.compute_device(d_r.data_ptr(), d_f.data_ptr(), d_e.data_ptr())  # complete rows
    truncated, max_row = p.check()
    assert truncated == 0 and max_row > 0
    torch.cuda.synchronize(dev)
    o = oracle_eval(wb, r, c)
    assert rel_max(d_f.cpu().numpy().reshape(-1, 3), o["f"]) < TOL
    assert abs(float(d_e[3]) - o["total"]) <= TOL * abs(o["total"])
    # captured again, the graph replays
    p.graph_capture(d_r.data_ptr(), d_f.data_ptr(), d_e.data_ptr())
    d_f.zero_()
    p.graph_launch()
    torch.cuda.synchronize(dev)
    assert rel_max(d_f.cpu().numpy().reshape(-1, 3), o["f"]) < TOL
    p.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nonfinite_coordinate_is_reported_and_the_handle_stays_usable(precision):
    import torch
    wb = water_box(6, seed=8)
    c = dict(rspace_cutoff=9.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=wb.box / 18,
             p3m_assignment_order=5)
    p = ElecLJ(precision=precision, **c).init(wb)
    bad = wb.positions.copy()
    bad[100, 1] = np.nan
    f = np.zeros((wb.nsite, 3))
    with pytest.raises(MmnbError) as ex:
        p.add_to_energy_and_forces(0.0, f, bad)
    assert ex.value.status == MMNB_ERR_DEVICE
    assert not f.any()  # nothing added
    # device path: reported by mmnb_check
    dev = torch.device("cuda", 0)
    d_r = torch.tensor(bad.reshape(-1), dtype=torch.float64, device=dev)
    d_f = torch.zeros(3 * wb.nsite, dtype=torch.float64, device=dev)
    p.compute_device(d_r.data_ptr(), d_f.data_ptr(), 0)
    with pytest.raises(MmnbError) as ex:
        p.check()
    assert ex.value.status == MMNB_ERR_DEVICE
    # the handle is still usable
    g = p.compute(wb.positions)
    o = oracle_eval(wb, wb.positions, c)
    tol = TOL if precision == "fp64" else 1e-4
    assert rel_max(g["f"], o["f"]) < tol
    p.close()


def test_volume_move_past_the_cutoff_is_refused_with_the_handle_unchanged():
    wb = water_box(6, seed=9)
    c = dict(rspace_cutoff=9.0, ewald_screening=0.35, kspace_cutoff=7.0)
    p = ElecLJ(precision="fp64", **c).init(wb)
    p.compute(wb.positions)
    with pytest.raises(MmnbError) as ex:
        p.scale(0.9)  # 0.49 x 16.78 A < 9 A
    assert ex.value.status == MMNB_ERR_CUTOFF
    g = p.compute(wb.positions)
    o = oracle_eval(wb, wb.positions, c)
    assert rel_max(g["f"], o["f"]) < TOL
    p.close()

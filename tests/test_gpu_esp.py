"""Potential at points away from the sites (mmnb_phi_at_points) against the
reference's ElecLJ::electrostatic_potential_at_gridpoints (src/eleclj.cpp:1302-1340):
the golden fixture made by the reference's own RSpaceEwaldPhiAtGridpoints and
kspace_phi, and the oracle's restatement on larger and orthorhombic boxes.
The call is FP64 in both precision forms; tolerance 1e-10 relative (max error
over points divided by the RMS potential)."""
import ctypes
import json
import os

import numpy as np
import pytest

from conftest import rel_max
from molmodel_b200 import ElecLJ, load_library, water_box
from oracle.oracle import make_config, port

pytestmark = pytest.mark.gpu

TOL = 1e-10
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "esp_points.npz")


def gpu(wb, cfg, q=None, rscreen=None, precision="fp64", bctype=1):
    p = ElecLJ(precision=precision, **cfg).init(wb, bctype=bctype)
    if q is not None or rscreen is not None:
        p.set_params(wb.site_mask, wb.q if q is None else q, wb.sigma, wb.epsilon,
                     wb.rscreen if rscreen is None else rscreen)
    return p


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("tag", ["ksum", "p3m"])
def test_phi_at_points_golden(tag, precision):
    g = np.load(GOLDEN)
    wb = water_box(int(g[tag + "_n"]), seed=int(g[tag + "_seed"]))
    cfg = json.loads(str(g[tag + "_config"]))
    p = gpu(wb, cfg, q=g[tag + "_q"], rscreen=g[tag + "_rscreen"], precision=precision)
    phi = p.electrostatic_potential_at_gridpoints(wb.positions, g[tag + "_points"])
    assert rel_max(phi, g[tag + "_phi"]) < TOL
    # a second call on the same handle gives the same bits (scratch is per call)
    assert np.array_equal(phi, p.electrostatic_potential_at_gridpoints(wb.positions, g[tag + "_points"]))


def test_phi_at_points_4096_waters_vs_oracle():
    wb = water_box(16, seed=4)
    cfg = dict(rspace_cutoff=9.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=wb.box / 48,
               p3m_assignment_order=5, kspace_cutoff=6.0)
    rng = np.random.default_rng(2)
    pts = rng.uniform(0, wb.box, size=(1000, 3))
    phi = gpu(wb, cfg).electrostatic_potential_at_gridpoints(wb.positions, pts)
    o = port().eleclj(make_config(wb.box, **cfg), wb.nsite, wb.groups, wb.exclusions, wb.site_mask, wb.q,
                      wb.sigma, wb.epsilon, wb.rscreen)
    assert rel_max(phi, o.phi_at_points(wb.positions, pts)) < TOL


class _System:
    """An orthorhombic view of a water box (the box is three edge lengths)."""

    def __init__(self, wb, box, q):
        for k in ("nsite", "groups", "exclusions", "site_mask", "sigma", "epsilon", "rscreen"):
            setattr(self, k, getattr(wb, k))
        self.q = q
        self.box = box


@pytest.mark.parametrize("flags", [dict(), dict(include_kspace=0), dict(include_rspace=0), dict(include_self=0)])
def test_phi_at_points_orthorhombic_terms(flags):
    wb = water_box(5, seed=6)
    stretch = np.array([1.0, 1.1, 0.95])
    r = wb.positions * stretch
    box = wb.box * stretch
    q = wb.q.copy()
    q[3] -= 0.3 * q[4]   # net charge: the neutralising term is on unless include_self is off
    s = _System(wb, box, q)
    cfg = dict(rspace_cutoff=6.5, ewald_screening=0.4, kspace_cutoff=5.0, **flags)
    o = port().eleclj(make_config(box, bctype=2, **cfg), s.nsite, s.groups, s.exclusions, s.site_mask, q,
                      s.sigma, s.epsilon, s.rscreen)
    rng = np.random.default_rng(3)
    pts = rng.uniform(0, 1, size=(200, 3)) * box
    ref = o.phi_at_points(r, pts)
    g = ElecLJ(**cfg).init(s, bctype=2)
    assert rel_max(g.electrostatic_potential_at_gridpoints(r, pts), ref) < TOL


def test_phi_at_points_empty_and_bad_args():
    wb = water_box(3, seed=1)
    p = gpu(wb, dict(rspace_cutoff=4.0, ewald_screening=0.5))
    assert p.electrostatic_potential_at_gridpoints(wb.positions, np.zeros((0, 3))).shape == (0,)
    # a null positions array or a negative count is rejected before any work
    lib = load_library()
    pts = np.zeros((4, 3))
    phi = np.zeros(4)
    dp = ctypes.POINTER(ctypes.c_double)
    assert lib.mmnb_phi_at_points(p._h, None, 4, pts.ctypes.data_as(dp), phi.ctypes.data_as(dp)) == 1
    r = np.ascontiguousarray(wb.positions)
    assert lib.mmnb_phi_at_points(p._h, r.ctypes.data_as(dp), -1, pts.ctypes.data_as(dp),
                                  phi.ctypes.data_as(dp)) == 1

"""The mixed form's P3M mesh path (FP32 B-spline weights, 64-bit fixed-point
charge mesh, FP32 R2C/C2R transforms and interpolation) against the FP64
form, whose mesh path matches the reference's CPU code to 1e-10.

Only the reciprocal-space force is compared (real space and self terms off),
so the bound measures the mesh path alone.  Mesh sizes cover the factors 2,
3, 5 and 7 of the reference's mesh sizes, odd lengths (an odd half
spectrum along z) and an orthorhombic box with three different lengths."""
import dataclasses

import numpy as np
import pytest

from conftest import rel_max, rel_rms
from molmodel_b200 import ElecLJ, water_box
from molmodel_b200 import _lib

pytestmark = pytest.mark.gpu

# RMS relative error of the reciprocal-space force, mixed vs FP64
KSPACE_RMS_TOL = 1e-5
KSPACE_MAX_TOL = 1e-4


def kspace_forces(system, spacing, precision, bctype=_lib.MMNB_CUBIC):
    cfg = dict(rspace_cutoff=9.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=spacing,
               p3m_assignment_order=5, include_rspace=False, include_self=False)
    pot = ElecLJ(precision=precision, **cfg).init(system, bctype=bctype)
    out = pot.compute(system.positions)
    st = pot.settings()
    pot.close()
    return out, st


@pytest.mark.parametrize("mesh", [24, 21, 35, 49, 96, 140])
def test_mesh_path_vs_fp64(mesh):
    wb = water_box(6, seed=5)
    g, st = kspace_forces(wb, wb.box / mesh, "mixed")
    o, _ = kspace_forces(wb, wb.box / mesh, "fp64")
    assert st["mesh"] == (mesh, mesh, mesh)
    err, emax = rel_rms(g["f"], o["f"]), rel_max(g["f"], o["f"])
    print(f"mesh {mesh}: RMS {err:.2e}, max {emax:.2e}")
    assert err < KSPACE_RMS_TOL
    assert emax < KSPACE_MAX_TOL
    assert abs(g["elec"] - o["elec"]) < 1e-5 * abs(o["elec"])


def test_mesh_path_orthorhombic():
    """Three different mesh lengths: the axes are not mixed up."""
    wb = water_box(6, seed=6)
    box = np.array([wb.box, 1.3 * wb.box, 1.6 * wb.box])
    sysb = dataclasses.replace(wb, box=box)
    g, st = kspace_forces(sysb, wb.box / 20, "mixed", _lib.MMNB_ORTHORHOMBIC)
    o, _ = kspace_forces(sysb, wb.box / 20, "fp64", _lib.MMNB_ORTHORHOMBIC)
    assert len(set(st["mesh"])) == 3
    err = rel_rms(g["f"], o["f"])
    print(f"mesh {st['mesh']}: RMS {err:.2e}")
    assert err < KSPACE_RMS_TOL


def test_mesh_path_bitwise_repeatable():
    """Two evaluations of the same positions give the same bits (the
    fixed-point mesh is cleared for the next step)."""
    wb = water_box(8, seed=7)
    cfg = dict(rspace_cutoff=9.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=wb.box / 28,
               p3m_assignment_order=5)
    pot = ElecLJ(precision="mixed", **cfg).init(wb)
    a = pot.compute(wb.positions)
    b = pot.compute(wb.positions)
    pot.close()
    assert np.array_equal(a["f"], b["f"])
    assert a["total"] == b["total"]

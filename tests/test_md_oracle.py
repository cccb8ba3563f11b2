"""The CPU restatement of the reference's MD step (oracle/md_oracle.py):
constraint solves and the integrator on forces simple enough to check by
hand.  The GPU integrator is compared with it in test_gpu_md.py."""
import numpy as np
import pytest

from molmodel_b200 import maxwell_boltzmann, water_box
from oracle import md_oracle
from oracle.oracle import reference

needs_reference = pytest.mark.skipif(reference() is None or not reference().has_constraints,
                                     reason="the reference build (oracle/_ref) is not present")

MASS_UNIT = 1.0 / 418.4


def _molecules(n=4, seed=2):
    wb = water_box(n, seed=seed)
    m = (wb.masses * MASS_UNIT).reshape(-1, 3)
    return wb, wb.positions.reshape(-1, 3, 3).copy(), m


def test_water_box_geometry_matches_the_constraints():
    wb, x, m = _molecules()
    _, dist = md_oracle._derivs(x)
    assert np.allclose(dist, md_oracle.water_lengths()[None, :], atol=1e-12)


def test_position_constraint_restores_geometry_and_momentum():
    wb, x0, m = _molecules()
    rng = np.random.default_rng(0)
    v = rng.normal(size=x0.shape) * 5.0
    x = x0 + 0.002 * v
    p_before = (m[..., None] * v).sum((0, 1))
    md_oracle.constrain_positions(x0, x, v, 1 / m, md_oracle.water_lengths(), 0.002)
    _, dist = md_oracle._derivs(x)
    assert np.abs(dist - md_oracle.water_lengths()[None, :]).max() < 1e-12
    # constraint forces are internal: total momentum is unchanged
    assert np.allclose((m[..., None] * v).sum((0, 1)), p_before, rtol=0, atol=1e-9)


def test_velocity_constraint_removes_bond_stretching():
    wb, x, m = _molecules()
    v = np.random.default_rng(1).normal(size=x.shape)
    md_oracle.constrain_velocities(x, v, 1 / m)
    g, _ = md_oracle._derivs(x)
    assert np.abs(np.einsum("mcak,mak->mc", g, v)).max() < 1e-12


def test_free_rigid_waters_keep_their_kinetic_energy():
    """No forces: the constrained motion is free rigid-body rotation and
    translation, whose kinetic energy the integrator keeps to O(dt^2)."""
    wb = water_box(3, seed=5)
    v = maxwell_boltzmann(wb, 300.0, seed=7)
    masses = wb.masses * MASS_UNIT
    _, _, e = md_oracle.run(lambda r: (np.zeros_like(r), 0.0), wb.positions, v, masses, 0.0005, 200,
                            md_oracle.water_lengths())
    assert np.abs(e[:, 0] / e[0, 0] - 1).max() < 1e-4


@needs_reference
def test_constraint_solves_match_the_reference_constraint_group():
    """The restated solves (three distances) against the reference's own
    ConstraintGroup (two O-H lengths and the H-O-H angle, src/constraint.cpp:
    295-358): the same converged positions and velocities."""
    wb, x0, m = _molecules(n=5, seed=3)
    rng = np.random.default_rng(5)
    v = rng.normal(size=x0.shape) * 8.0
    x = x0 + 0.002 * v
    xr, vr = x.copy(), v.copy()
    md_oracle.constrain_positions(x0, xr, vr, 1 / m, md_oracle.water_lengths(), 0.002)
    xf, vf = reference().water_constrain_positions(x0, x, v, m[0], 0.002, tol=1e-13)
    assert np.abs(xf.reshape(x.shape) - xr).max() < 1e-11
    assert np.abs(vf.reshape(v.shape) - vr).max() < 1e-11 / 0.002
    w = rng.normal(size=x0.shape)
    wr = w.copy()
    md_oracle.constrain_velocities(xr, wr, 1 / m)
    wf = reference().water_constrain_velocities(xr, w, m[0])
    assert np.abs(wf.reshape(w.shape) - wr).max() < 1e-12


@needs_reference
def test_md_step_with_the_reference_constraints():
    """200 steps of free rigid waters: the restated step with the reference's
    constraint solver and with the restated one give the same trajectory."""
    wb = water_box(3, seed=5)
    v = maxwell_boltzmann(wb, 300.0, seed=7)
    masses = wb.masses * MASS_UNIT
    free = lambda r: (np.zeros_like(r), 0.0)
    ra, va, ea = md_oracle.run(free, wb.positions, v, masses, 0.0005, 200, md_oracle.water_lengths())
    rb, vb, eb = md_oracle.run(free, wb.positions, v, masses, 0.0005, 200, md_oracle.water_lengths(),
                               constraints=md_oracle.ReferenceConstraints(reference()))
    assert np.abs(ra - rb).max() < 1e-10
    assert np.abs(ea - eb).max() < 1e-10 * np.abs(ea).max()

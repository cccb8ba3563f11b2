"""Device MD (mmnb_md_*): velocity Verlet with SETTLE against the CPU
restatement of the reference's MD step with SHAKE/RATTLE, rigid geometry
and energy conservation."""
import numpy as np
import pytest

from molmodel_b200 import ElecLJ, maxwell_boltzmann, water_box
from molmodel_b200.md import MDyn, nve_drift
from oracle import md_oracle
from oracle.oracle import make_config, port, reference

pytestmark = pytest.mark.gpu

MASS_UNIT = 1.0 / 418.4


def _ksum_cfg():
    return dict(rspace_cutoff=9.0, ewald_screening=0.35, kspace_cutoff=7.0)


def _bond_errors(r, nmol):
    x = r.reshape(nmol, 3, 3)
    _, dist = md_oracle._derivs(x)
    return np.abs(dist - md_oracle.water_lengths()[None, :]).max()


@pytest.mark.parametrize("solver", ["restated", "reference"])
def test_fp64_md_follows_the_reference_step(solver):
    """216 waters, ordinary Ewald (kc 7), 1 fs, 10 steps: SETTLE + the 3x3
    velocity solve against the reference's step with its constraint solves
    iterated to convergence -- restated (three distances), or the reference's
    own ConstraintGroup (two O-H lengths and the H-O-H angle,
    src/constraint.cpp:295-358) with the reference's own energies, where the
    reference build is present."""
    ref = reference()
    if solver == "reference" and (ref is None or not ref.has_constraints):
        pytest.skip("the reference build (oracle/_ref) is not present")
    wb = water_box(6, seed=1)
    cfg = _ksum_cfg()
    v0 = maxwell_boltzmann(wb, 300.0, seed=3)
    pot = ElecLJ(precision="fp64", **cfg).init(wb)
    md = MDyn(pot, wb.masses, timestep=0.001)
    md.set_state(wb.positions, v0)
    e_gpu = md.run(10)
    r_gpu, v_gpu = md.state()
    md.close()

    lib = ref if solver == "reference" else port()
    o = lib.eleclj(make_config(wb.box, **cfg), wb.nsite, wb.groups, wb.exclusions, wb.site_mask, wb.q,
                   wb.sigma, wb.epsilon, wb.rscreen)

    def evaluate(r):
        out = o.eval(r)
        return out["f"], out["total"]

    cs = md_oracle.ReferenceConstraints(ref) if solver == "reference" else None
    r_o, v_o, e_o = md_oracle.run(evaluate, wb.positions, v0, wb.masses * MASS_UNIT, 0.001, 10,
                                  md_oracle.water_lengths(), constraints=cs)
    assert np.abs(r_gpu - r_o).max() < 1e-9
    assert np.abs(v_gpu - v_o).max() < 1e-6 * np.abs(v_o).max()
    assert np.abs(e_gpu - e_o).max() < 1e-8 * np.abs(e_o[:, 2]).max()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_md_keeps_rigid_geometry_and_conserves_energy(precision):
    """512 waters, P3M 24^3, 1 fs, 400 steps: bonds stay at their lengths and
    the conserved energy drifts by far less than its fluctuations allow."""
    wb = water_box(8, seed=2)
    cfg = dict(rspace_cutoff=9.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=wb.box / 24,
               p3m_assignment_order=5, neighbor_list_width=1.0)
    pot = ElecLJ(precision=precision, **cfg).init(wb)
    md = MDyn(pot, wb.masses, timestep=0.001)
    md.set_state(wb.positions, maxwell_boltzmann(wb, 300.0, seed=4))
    e = md.run(400)
    r, v = md.state()
    md.close()
    assert _bond_errors(r, wb.nwater) < 1e-9
    # drift of the conserved energy in kcal/mol per ns per molecule
    drift = abs(nve_drift(e, 0.001, wb.nwater))
    assert drift < 5.0, drift
    # it is a conserved quantity: its spread is small next to the kinetic energy's
    assert e[:, 2].std() < 0.05 * e[:, 0].std()

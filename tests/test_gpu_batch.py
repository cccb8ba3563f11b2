"""Replica batch (mmnb_md_batch): replicas of uneven size advanced by one graph
launch per step give exactly what each replica gives on its own, and a
temperature swap rescales velocities as asked."""
import numpy as np
import pytest

from molmodel_b200 import ElecLJ, maxwell_boltzmann, water_box_n
from molmodel_b200.md import MDyn, ReplicaBatch

pytestmark = pytest.mark.gpu


def _replica(nw, i):
    wb = water_box_n(nw, seed=40 + i)
    pot = ElecLJ(precision="mixed", rspace_cutoff=9.0, ewald_screening=0.35, neighbor_list_width=1.5,
                 use_p3m=True, p3m_grid_spacing=1.04, p3m_assignment_order=5).init(wb)
    md = MDyn(pot, wb.masses, timestep=0.002)
    md.set_state(wb.positions, maxwell_boltzmann(wb, 300.0 + 20 * i, seed=70 + i))
    return wb, pot, md


def test_batch_equals_replicas_run_alone():
    sizes = [256, 300, 517]
    batched = [_replica(n, i) for i, n in enumerate(sizes)]
    alone = [_replica(n, i) for i, n in enumerate(sizes)]
    b = ReplicaBatch([r[2] for r in batched])
    eb = b.run(25)
    eb2 = b.run(5)
    b.close()
    for k, (rb, ra) in enumerate(zip(batched, alone)):
        ea = ra[2].run(25)
        ea2 = ra[2].run(5)
        xb, vb = rb[2].state()
        xa, va = ra[2].state()
        # mixed form: fixed-point sums, so the branch order cannot matter
        assert np.array_equal(xb, xa) and np.array_equal(vb, va), k
        assert np.array_equal(eb[k], ea) and np.array_equal(eb2[k], ea2), k
    for r in batched + alone:
        r[2].close()
        r[1].close()


def test_velocity_rescale():
    wb, pot, md = _replica(256, 0)
    _, v0 = md.state()
    md.scale_velocities(1.1)
    _, v1 = md.state()
    assert np.allclose(v1, 1.1 * v0, rtol=1e-15, atol=0)
    md.close()
    pot.close()

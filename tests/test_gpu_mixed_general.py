"""The mixed form's general pair kernel (any group size, screening radii,
group exclusions, 1-4 pairs) against the FP64 oracle."""
import numpy as np
import pytest

from conftest import rel_max, rel_rms
from molmodel_b200 import ElecLJ, water_box
from oracle.oracle import make_config, port
from test_gpu_parity import C1, Custom

pytestmark = pytest.mark.gpu

RMS_TOL = 1e-5
ENERGY_TOL = 5e-5


class Paired:
    """Waters grouped two by two: groups of six sites (anchor = the first O),
    each water's own pairs excluded, the two waters of a group not."""

    def __init__(self, wb):
        self.nsite, self.box, self.positions = wb.nsite, wb.box, wb.positions
        self.site_mask, self.q, self.sigma, self.epsilon, self.rscreen = (wb.site_mask, wb.q, wb.sigma, wb.epsilon,
                                                                          wb.rscreen)
        g = np.arange(0, wb.nsite, 6, dtype=np.int32)
        self.groups = np.stack([g, np.minimum(g + 6, wb.nsite)], axis=1).astype(np.int32)
        self.exclusions = wb.exclusions


def _oracle(s, cfg, pairs14=None):
    c = make_config(s.box, **cfg)
    return port().eleclj(c, s.nsite, s.groups, s.exclusions, s.site_mask, s.q, s.sigma, s.epsilon, s.rscreen,
                         pairs14=pairs14)


@pytest.mark.parametrize("fields", [False, True])
def test_mixed_screening_group_exclusions_and_14(fields):
    cs = Custom(water_box(6, seed=1), np.random.default_rng(3))
    cfg = dict(C1, elec_1_4_scale_factor=0.5, lj_1_4_scale_factor=0.7)
    p = ElecLJ(precision="mixed", **cfg).init(cs, pairs14=cs.pairs14)
    g = p.compute(cs.positions, want_fields=fields)
    o = _oracle(cs, cfg, cs.pairs14).eval(cs.positions)
    assert rel_rms(g["f"], o["f"]) < RMS_TOL
    assert abs(g["total"] - o["total"]) < ENERGY_TOL * abs(o["total"])
    if fields:
        assert rel_max(g["phi"], o["phi"]) < 1e-4


def test_mixed_six_site_groups():
    s = Paired(water_box(6, seed=2))
    p3m = dict(rspace_cutoff=9.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=s.box / 20,
               p3m_assignment_order=5)
    g = ElecLJ(precision="mixed", **p3m).init(s).compute(s.positions)
    o = _oracle(s, p3m).eval(s.positions)
    assert rel_rms(g["f"], o["f"]) < RMS_TOL
    assert abs(g["total"] - o["total"]) < ENERGY_TOL * abs(o["total"])
    g64 = ElecLJ(precision="fp64", **p3m).init(s).compute(s.positions)
    assert rel_max(g64["f"], o["f"]) < 1e-10

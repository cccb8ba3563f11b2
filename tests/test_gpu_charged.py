"""A system with a net charge: the neutralising background term
(src/eleclj.cpp:965-975: -pi / (eta^2 V) times the total charge on every site
potential) reaches the energies for P3M and for the k-sum, in both forms,
against the oracle; and it follows a charge change through set_params, on the
host call's first evaluation after the change and on its graph replays."""
import numpy as np
import pytest

from conftest import rel_max, rel_rms
from molmodel_b200 import ElecLJ, water_box
from molmodel_b200.water import WaterBox
from oracle.oracle import make_config, port, reference

pytestmark = pytest.mark.gpu

RMS_TOL = 1e-5
ENERGY_TOL = 5e-5

CFGS = {
    "p3m": dict(rspace_cutoff=7.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=0.8,
                p3m_assignment_order=5),
    "ksum": dict(rspace_cutoff=7.0, ewald_screening=0.35, kspace_cutoff=6.0),
}


def charged(wb, dq_e):
    q = wb.charges_e.copy()
    q[0] += dq_e  # one O site: the box now carries dq_e elementary charges
    return WaterBox(nwater=wb.nwater, box=wb.box, positions=wb.positions, masses=wb.masses, seed=wb.seed,
                    charges_e=q)


def oracle_eval(lib, s, cfg, r=None):
    o = lib.eleclj(make_config(s.box, **cfg), s.nsite, s.groups, s.exclusions, s.site_mask, s.q, s.sigma,
                   s.epsilon, s.rscreen)
    return o.eval(s.positions if r is None else r)


@pytest.mark.parametrize("kind", sorted(CFGS))
def test_net_charge_fp64(kind):
    wb = charged(water_box(5, seed=14), 0.8)
    assert abs(wb.charges_e.sum()) > 0.5
    cfg = CFGS[kind]
    g = ElecLJ(**cfg).init(wb).compute(wb.positions, want_fields=True)
    o = oracle_eval(port(), wb, cfg)
    assert rel_max(g["f"], o["f"]) < 1e-10
    assert rel_max(g["phi"], o["phi"]) < 1e-10
    for k in ("elec", "lj", "total"):
        assert abs(g[k] - o[k]) <= 1e-10 * abs(o[k]), k
    ref = reference()
    if ref is not None:
        r = oracle_eval(ref, wb, cfg)
        assert abs(g["total"] - r["total"]) <= 1e-10 * abs(r["total"])
    # the background term is there: the neutral box's site potentials differ by it
    n = water_box(5, seed=14)
    gn = ElecLJ(**cfg).init(n).compute(n.positions, want_fields=True)
    assert np.abs(g["phi"][1:] - gn["phi"][1:]).min() > 0


@pytest.mark.parametrize("kind", sorted(CFGS))
def test_net_charge_mixed_after_set_params(kind):
    base = water_box(5, seed=15)
    wb = charged(base, 0.8)
    cfg = CFGS[kind]
    p = ElecLJ(precision="mixed", **cfg).init(base)
    p.compute(base.positions)
    p.compute(base.positions)  # the host call's graph exists from here on
    p.set_params(wb.site_mask, wb.q, wb.sigma, wb.epsilon, wb.rscreen)
    rng = np.random.default_rng(4)
    r = wb.positions.copy()
    for _ in range(3):  # the first evaluation after the change, then graph replays
        r = r + rng.normal(scale=0.02, size=r.shape)
        g = p.compute(r)
        o = oracle_eval(port(), wb, cfg, r)
        assert rel_rms(g["f"], o["f"]) < RMS_TOL
        assert abs(g["elec"] - o["elec"]) <= ENERGY_TOL * abs(o["elec"])
        assert abs(g["total"] - o["total"]) <= ENERGY_TOL * abs(o["total"])

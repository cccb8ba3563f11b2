"""FP64 GPU form vs the CPU oracle on the same seeded inputs.

The FP64 form must match the reference's eleclj + rspace + pppm/kspace results
to 1e-10 relative (forces, site potentials and fields: max over sites of the
vector error divided by the RMS vector; energies: relative), and its cell
assignment and neighbour list must be identical to the reference's.
"""
import numpy as np
import pytest

from conftest import rel_max
from molmodel_b200 import ElecLJ, water_box
from molmodel_b200.water import WaterBox
from oracle.oracle import make_config, port, reference

pytestmark = pytest.mark.gpu

TOL = 1e-10

C1 = dict(rspace_cutoff=9.0, smoothing_width=1.0, ewald_screening=0.35, kspace_cutoff=7.0)


def p3m_cfg(box, mesh, order=5, **kw):
    d = dict(rspace_cutoff=9.0, smoothing_width=1.0, ewald_screening=0.35, use_p3m=True,
             p3m_grid_spacing=box / mesh, p3m_assignment_order=order)
    d.update(kw)
    return d


def oracle_for(lib, system, cfg, bctype=1, box=None, pairs14=None):
    c = make_config(system.box if box is None else box, bctype=bctype, **cfg)
    return lib.eleclj(c, system.nsite, system.groups, system.exclusions, system.site_mask, system.q,
                      system.sigma, system.epsilon, system.rscreen, pairs14=pairs14)


def gpu_for(system, cfg, bctype=1, pairs14=None, precision="fp64"):
    p = ElecLJ(precision=precision, **cfg)
    return p.init(system, bctype=bctype, pairs14=pairs14)


def assert_parity(g, o, tol=TOL):
    assert rel_max(g["f"], o["f"]) < tol
    assert rel_max(g["phi"], o["phi"]) < tol
    assert rel_max(g["evec"], o["evec"]) < tol
    for k in ("elec", "lj", "lj_correction", "total"):
        assert abs(g[k] - o[k]) <= tol * max(abs(o[k]), 1e-300), k


def canon_pairs(p):
    p = np.sort(np.asarray(p, dtype=np.int64), axis=1)
    return np.unique(p[:, 0] * (1 << 32) + p[:, 1])


@pytest.fixture(scope="module")
def c1():
    return water_box(6, seed=1)


def test_c1_ewald_fp64(c1):
    g = gpu_for(c1, C1).compute(c1.positions, want_fields=True)
    o = oracle_for(port(), c1, C1).eval(c1.positions)
    assert_parity(g, o)
    ref = reference()
    if ref is not None:
        assert_parity(g, oracle_for(ref, c1, C1).eval(c1.positions))


@pytest.mark.parametrize("order", [2, 3, 4, 5, 6, 7])
def test_p3m_orders_fp64(order):
    wb = water_box(5, seed=3)
    cfg = dict(rspace_cutoff=7.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=0.8,
               p3m_assignment_order=order)
    g = gpu_for(wb, cfg).compute(wb.positions, want_fields=True)
    o = oracle_for(port(), wb, cfg).eval(wb.positions)
    assert_parity(g, o)


def test_p3m_ik_fp64():
    wb = water_box(5, seed=4)
    cfg = dict(rspace_cutoff=7.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=0.8,
               p3m_assignment_order=5, p3m_ik_differentiate=True)
    g = gpu_for(wb, cfg).compute(wb.positions, want_fields=True)
    o = oracle_for(port(), wb, cfg).eval(wb.positions)
    assert_parity(g, o)


@pytest.fixture(scope="module")
def c2():
    return water_box(16, seed=2)


def test_c2_p3m_fp64_and_list(c2):
    cfg = p3m_cfg(c2.box, 48, neighbor_list_width=1.5)
    p = gpu_for(c2, cfg)
    g = p.compute(c2.positions, want_fields=True)
    o = oracle_for(port(), c2, cfg)
    oo = o.eval(c2.positions)
    assert_parity(g, oo)
    assert p.settings()["mesh"] == (48, 48, 48)
    # neighbour list and cells are the reference's, exactly
    assert np.array_equal(canon_pairs(p.pairlist()), canon_pairs(o.nbrlist().pairs()))
    cells, n = p.cells(c2.ngroup)
    assert n == o.nbrlist().ncell()
    assert np.array_equal(cells, o.nbrlist().cells(c2.ngroup))


def test_rebuild_sequence_matches_reference(c1):
    """Displace molecules step by step: rebuild decisions and lists follow
    NeighborList::coordinates_changed exactly."""
    cfg = dict(C1, neighbor_list_width=0.3)
    p = gpu_for(c1, cfg)
    o = oracle_for(port(), c1, cfg)
    nl = port().nbrlist(c1.ngroup, 9.0, o.nlw, c1.box)
    rng = np.random.default_rng(7)
    r = c1.positions.copy()
    rebuilds = 0
    for step in range(25):
        rebuilds += nl.update(r[0::3])
        o.eval(r)
        p.compute(r)
        rb, ev = p.counters()
        assert ev == step + 1
        assert rb == rebuilds
        assert np.array_equal(canon_pairs(p.pairlist()), canon_pairs(nl.pairs()))
        r = r + rng.normal(scale=0.05, size=r.shape)
    assert rebuilds >= 3  # the 0.3 A skin is crossed several times in 25 steps


def test_unwrapped_coordinates(c1):
    """Molecules moved by whole box vectors: same forces, reference cells and list."""
    rng = np.random.default_rng(11)
    shift = rng.integers(-3, 4, size=(c1.nwater, 3)) * c1.box
    r = (c1.positions.reshape(-1, 3, 3) + shift[:, None, :]).reshape(-1, 3)
    g0 = gpu_for(c1, C1).compute(c1.positions)
    p = gpu_for(c1, C1)
    g = p.compute(r, want_fields=True)
    o = oracle_for(port(), c1, C1)
    assert_parity(g, o.eval(r))
    assert rel_max(g["f"], g0["f"]) < TOL
    assert np.array_equal(canon_pairs(p.pairlist()), canon_pairs(o.nbrlist().pairs()))
    assert np.array_equal(p.cells(c1.ngroup)[0], o.nbrlist().cells(c1.ngroup))


def test_orthorhombic():
    wb = water_box(6, seed=5)
    stretch = np.array([1.0, 1.1, 0.95])
    r = wb.positions * stretch
    sysx = WaterBox(nwater=wb.nwater, box=wb.box, positions=r, masses=wb.masses, seed=5,
                    charges_e=wb.charges_e)
    box = wb.box * stretch

    class Ortho:
        pass
    s = Ortho()
    for k in ("nsite", "groups", "exclusions", "site_mask", "q", "sigma", "epsilon", "rscreen"):
        setattr(s, k, getattr(sysx, k))
    s.box = box
    cfg = dict(rspace_cutoff=8.5, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=0.9,
               p3m_assignment_order=4)
    g = gpu_for(s, cfg, bctype=2).compute(r, want_fields=True)
    o = oracle_for(port(), s, cfg, bctype=2, box=box).eval(r)
    assert_parity(g, o)


class Custom:
    """A water box with extra cross-group exclusions, screening radii and 1-4
    pairs, to exercise group_excluded, the screening function and the 1-4 path."""

    def __init__(self, wb, rng):
        self.nsite, self.box, self.positions = wb.nsite, wb.box, wb.positions
        self.groups, self.site_mask, self.q = wb.groups, wb.site_mask, wb.q
        self.sigma, self.epsilon = wb.sigma, wb.epsilon
        k = rng.choice(wb.nwater - 1, size=wb.nwater // 4, replace=False)
        extra = np.stack([3 * k, 3 * (k + 1)], axis=1)           # O(k) - O(k+1)
        extra2 = np.stack([3 * k + 1, 3 * (k + 1) + 2], axis=1)  # H(k) - H(k+1)
        self.exclusions = np.concatenate([wb.exclusions, extra, extra2]).astype(np.int32)
        self.rscreen = np.where(np.arange(wb.nsite) % 3 == 0, 1.6, 0.0)
        j = rng.choice(wb.nwater - 2, size=wb.nwater // 5, replace=False)
        self.pairs14 = np.stack([3 * j, 3 * (j + 2) + 1], axis=1).astype(np.int32)


def test_group_exclusions_screening_and_14(c1):
    cs = Custom(c1, np.random.default_rng(3))
    cfg = dict(C1, elec_1_4_scale_factor=0.5, lj_1_4_scale_factor=0.7)
    g = gpu_for(cs, cfg, pairs14=cs.pairs14).compute(cs.positions, want_fields=True)
    o = oracle_for(port(), cs, cfg, pairs14=cs.pairs14).eval(cs.positions)
    assert_parity(g, o)
    ref = reference()
    if ref is not None:
        assert_parity(g, oracle_for(ref, cs, cfg, pairs14=cs.pairs14).eval(cs.positions))


def test_scale_matches_fresh_setup():
    """ElecLJ::scale: eta / s, table, influence function and stencil follow."""
    wb = water_box(5, seed=8)
    s = 1.02
    cfg = dict(rspace_cutoff=7.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=0.8,
               p3m_assignment_order=5)
    p = gpu_for(wb, cfg)
    p.compute(wb.positions)
    p.scale(s)
    r = wb.positions * s
    g = p.compute(r, want_fields=True)
    cfg2 = dict(cfg, ewald_screening=0.35 / s, p3m_grid_spacing=0.8 * s)
    o = oracle_for(port(), wb, cfg2, box=wb.box * s).eval(r)
    assert_parity(g, o, tol=1e-9)


def test_energy_conservation_fd(c1):
    """Forces are the negative gradient of the energy (central differences)."""
    p = gpu_for(c1, C1)
    r = c1.positions.copy()
    g = p.compute(r)
    rng = np.random.default_rng(1)
    d = rng.normal(size=r.shape)
    d /= np.linalg.norm(d)
    h = 1e-5
    ep = p.compute(r + h * d)["total"]
    em = p.compute(r - h * d)["total"]
    fd = -(ep - em) / (2 * h)
    an = float((g["f"] * d).sum())
    assert abs(fd - an) < 1e-6 * max(1.0, abs(an))


def test_orthorhombic_list_with_cell_cull():
    """A box large enough that the list build skips stencil cells per row
    (different cell edges on the three axes, molecules also outside the box):
    the pair list is still exactly the reference's, before and after a rebuild."""
    wb = water_box(13, seed=21)
    stretch = np.array([1.0, 1.12, 0.9])
    r = wb.positions * stretch
    r[0:30] += np.array([1.0, -2.0, 1.0]) * (wb.box * stretch)   # ten molecules one image away
    box = wb.box * stretch

    class Ortho:
        pass
    s = Ortho()
    for k in ("nsite", "groups", "exclusions", "site_mask", "q", "sigma", "epsilon", "rscreen"):
        setattr(s, k, getattr(wb, k))
    s.box = box
    cfg = dict(rspace_cutoff=9.0, ewald_screening=0.35, neighbor_list_width=1.5, use_p3m=True,
               p3m_grid_spacing=1.2, p3m_assignment_order=4)
    p = gpu_for(s, cfg, bctype=2)
    o = oracle_for(port(), s, cfg, bctype=2, box=box)
    rng = np.random.default_rng(4)
    for step in range(3):
        g = p.compute(r, want_fields=True)
        oo = o.eval(r)
        assert_parity(g, oo)
        assert np.array_equal(canon_pairs(p.pairlist()), canon_pairs(o.nbrlist().pairs())), step
        # whole molecules moved past the skin: the next evaluation rebuilds
        r = (r.reshape(-1, 3, 3) + rng.normal(scale=0.2, size=(wb.nwater, 1, 3))).reshape(-1, 3)

"""Parity on the headline configuration: the 98,304-site water box that
bench.py times (32,768 rigid waters, L = 99.437 A, P3M 96^3 order 5, eta 0.35,
rc 9 A with a 1 A switch, skin 1.5 A).

* FP64 form against the reference's own code (oracle/_ref, compiled from the
  reference's sources; the oracle's restatement where that was not built):
  forces, site potentials and fields to 1e-10 relative, energies to 1e-10,
  cell of every group and the neighbour pair set identical, after the first
  build and again after a rebuild that the reference's displacement criterion
  triggers (src/nbrlist.cpp:51-77, 222-251; src/eleclj.cpp:785-807).
* Mixed form against the same FP64 results on two seeds: RMS relative force
  error <= 1e-5.
"""
import numpy as np
import pytest

from conftest import rel_max, rel_rms
from molmodel_b200 import ElecLJ, water_box
from oracle.oracle import make_config, port, reference

pytestmark = pytest.mark.gpu

TOL = 1e-10
RMS_TOL = 1e-5
NSIDE, MESH = 32, 96


def cfg_for(box):
    return dict(rspace_cutoff=9.0, smoothing_width=1.0, neighbor_list_width=1.5, ewald_screening=0.35,
                use_p3m=True, p3m_grid_spacing=box / MESH, p3m_assignment_order=5, p3m_alias_sum_limit=2)


def oracle_lib():
    return reference() or port()


def oracle_for(lib, wb, cfg):
    c = make_config(wb.box, **cfg)
    return lib.eleclj(c, wb.nsite, wb.groups, wb.exclusions, wb.site_mask, wb.q, wb.sigma, wb.epsilon,
                      wb.rscreen)


def canon_pairs(p):
    p = np.sort(np.asarray(p, dtype=np.int64), axis=1)
    return np.unique(p[:, 0] * (1 << 32) + p[:, 1])


def assert_fp64_parity(g, o):
    assert rel_max(g["f"], o["f"]) < TOL
    assert rel_max(g["phi"], o["phi"]) < TOL
    assert rel_max(g["evec"], o["evec"]) < TOL
    for k in ("elec", "lj", "lj_correction", "total"):
        assert abs(g[k] - o[k]) <= TOL * abs(o[k]), k


def assert_same_list(p, o, wb):
    nl = o.nbrlist()
    assert np.array_equal(canon_pairs(p.pairlist()), canon_pairs(nl.pairs()))
    cells, n = p.cells(wb.ngroup)
    assert n == nl.ncell() == 25
    assert np.array_equal(cells, nl.cells(wb.ngroup))


def test_c3_fp64_matches_reference_with_identical_lists():
    wb = water_box(NSIDE, seed=1)
    cfg = cfg_for(wb.box)
    p = ElecLJ(precision="fp64", **cfg).init(wb)
    o = oracle_for(oracle_lib(), wb, cfg)
    g = p.compute(wb.positions, want_fields=True)
    assert p.settings()["mesh"] == (MESH, MESH, MESH)
    assert_fp64_parity(g, o.eval(wb.positions))
    assert_same_list(p, o, wb)
    # every molecule jiggled, two of them carried 0.8 A: the two largest anchor
    # moves add up to more than the 1.5 A skin, so both sides rebuild
    rng = np.random.default_rng(11)
    r = wb.positions + rng.normal(scale=0.02, size=wb.positions.shape)
    for g_ in (5, 20000):
        r[3 * g_:3 * g_ + 3] += np.array([0.8, -0.1, 0.05])
    g = p.compute(r, want_fields=True)
    assert p.counters()[0] == 2  # rebuilds: the first build and this one
    assert_fp64_parity(g, o.eval(r))
    assert_same_list(p, o, wb)
    p.close()


@pytest.mark.parametrize("seed", [1, 2])
def test_c3_mixed_error_vs_fp64_oracle(seed):
    wb = water_box(NSIDE, seed=seed)
    cfg = cfg_for(wb.box)
    p = ElecLJ(precision="mixed", **cfg).init(wb)
    g = p.compute(wb.positions)
    o = oracle_for(oracle_lib(), wb, cfg).eval(wb.positions)
    assert rel_rms(g["f"], o["f"]) < RMS_TOL
    assert abs(g["total"] - o["total"]) < 5e-5 * abs(o["total"])
    p.close()

"""The Ewald screening the library chooses for P3M when none is given
(p3m_optimize, src/pppm.c:666-716), the grid-density rule for the mesh
(src/eleclj.cpp:195-200) and the error estimates ElecLJ::init reports
(src/eleclj.cpp:129-138, 225, 233-243), each against the reference's own code.

The reference minimises chi_r^2 + chi_k^2 with GSL's simplex and stops once the
simplex size (mean distance of its vertices from their centre) is below 1e-4.
The library runs a Nelder-Mead simplex from the same start with the same step,
size test and iteration limit.  Both end within a few sizes of the objective's
minimum, which the oracle finds by golden-section search on the reference's own
objective, so eta is compared with that minimum to ETA_TOL, and the objective
at the library's eta must be within OBJ_TOL (relative) of its minimum.  The mesh
estimate itself is compared to CHI_TOL, which its cancellation sets.
"""
import numpy as np
import pytest

from conftest import rel_max
from molmodel_b200 import ElecLJ, water_box
from molmodel_b200._lib import MmnbError
from oracle.oracle import make_config, port, reference

pytestmark = pytest.mark.gpu

ETA_TOL = 5e-4
OBJ_TOL = 1e-4
# chi_k^2 is the difference of two sums over the mesh (sum_p g^2 k^2 and
# numerator^2 / denominator) that agree to 8 digits for ik at order 4 on 18^3
# and to 10 digits for order 5 on 30^3, so last-bit differences of the device's
# exp, pow and sin from the host's are amplified 1e8-1e10 times
CHI_TOL = 1e-6

CASES = {
    "order5": (6, dict(rspace_cutoff=9.0, p3m_grid_spacing=0.5, p3m_assignment_order=5)),
    "order3_alias1": (5, dict(rspace_cutoff=7.0, p3m_grid_spacing=0.8, p3m_assignment_order=3,
                              p3m_alias_sum_limit=1)),
    "order4_ik": (5, dict(rspace_cutoff=7.0, p3m_grid_spacing=0.8, p3m_assignment_order=4,
                          p3m_ik_differentiate=True)),
}


def oracle_lib():
    ref = reference()
    return ref if ref is not None else port()


def mesh_args(cfg):
    return (cfg["p3m_grid_spacing"], cfg["p3m_assignment_order"])


def mesh_kw(cfg):
    return dict(nalias=cfg.get("p3m_alias_sum_limit", 2), ik=cfg.get("p3m_ik_differentiate", False))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_optimised_eta_matches_the_reference_objective(case, precision):
    n, cfg = CASES[case]
    wb = water_box(n, seed=5)
    p = ElecLJ(precision=precision, ewald_screening=-1.0, use_p3m=True, **cfg).init(wb)
    s = p.settings()
    lib = oracle_lib()
    latv = np.eye(3) * wb.box
    sp, order = mesh_args(cfg)
    eta_star = lib.p3m_optimize(latv, sp, order, s["rc"], **mesh_kw(cfg))
    assert abs(s["eta"] - eta_star) < ETA_TOL, (s["eta"], eta_star)
    obj = lambda e: lib.p3m_optimize_objective(latv, sp, order, s["rc"], e, **mesh_kw(cfg))
    assert obj(s["eta"]) <= obj(eta_star) * (1 + OBJ_TOL)
    # the estimates at the chosen eta: the mesh's is p3m_init's, the real-space
    # one estimated_dimensionless_rspace_error's
    rs, ks = p.error_estimates()
    chi, mesh = lib.p3m_chi(latv, sp, order, s["eta"], **mesh_kw(cfg))
    assert mesh == s["mesh"]
    assert abs(ks - chi) <= CHI_TOL * chi
    rc, v = s["rc"], wb.box ** 3
    rs_ref = 2 / np.sqrt(rc / np.cbrt(v)) * np.exp(-(rc * s["eta"]) ** 2)
    assert abs(rs - rs_ref) <= 1e-13 * rs_ref


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_optimised_eta_gives_the_explicit_eta_result(precision):
    """A potential whose eta was optimised evaluates as one given that eta: the
    real-space table, the influence function and the self term all follow it."""
    n, cfg = CASES["order3_alias1"]
    wb = water_box(n, seed=6)
    p = ElecLJ(precision=precision, ewald_screening=-1.0, use_p3m=True, **cfg).init(wb)
    eta = p.settings()["eta"]
    q = ElecLJ(precision=precision, ewald_screening=eta, use_p3m=True, **cfg).init(wb)
    a = p.compute(wb.positions, want_fields=True)
    b = q.compute(wb.positions, want_fields=True)
    if precision == "mixed":
        # fixed-point sums: the same inputs give the same bits
        assert np.array_equal(a["f"], b["f"]) and a["total"] == b["total"]
    else:
        assert rel_max(a["f"], b["f"]) < 1e-12
        assert abs(a["total"] - b["total"]) <= 1e-12 * abs(b["total"])
    if precision == "fp64":
        o = port().eleclj(make_config(wb.box, ewald_screening=eta, use_p3m=True, **cfg), wb.nsite, wb.groups,
                          wb.exclusions, wb.site_mask, wb.q, wb.sigma, wb.epsilon, wb.rscreen).eval(wb.positions)
        assert rel_max(a["f"], o["f"]) < 1e-10
        assert abs(a["total"] - o["total"]) <= 1e-10 * abs(o["total"])


def test_grid_density_sets_the_mesh():
    wb = water_box(5, seed=7)
    density = 2.0
    p = ElecLJ(ewald_screening=0.35, use_p3m=True, p3m_grid_density=density, rspace_cutoff=7.0).init(wb)
    sp = wb.box / np.cbrt(density * wb.box ** 3)
    _, mesh = oracle_lib().p3m_chi(np.eye(3) * wb.box, sp, 3, 0.35)
    assert p.settings()["mesh"] == mesh
    # a spacing other than the default beside a density is an error, as in the reference
    with pytest.raises(MmnbError):
        ElecLJ(ewald_screening=0.35, use_p3m=True, p3m_grid_density=density, p3m_grid_spacing=0.8,
               rspace_cutoff=7.0).init(wb)


def test_kspace_sum_error_estimate_and_automatic_eta():
    wb = water_box(5, seed=8)
    kc, rc = 7.0, 7.0
    p = ElecLJ(kspace_cutoff=kc, rspace_cutoff=rc).init(wb)
    s = p.settings()
    eta = np.sqrt(np.pi * kc / (rc * wb.box))
    assert abs(s["eta"] - eta) <= 1e-15 * eta
    rs, ks = p.error_estimates()
    l = np.cbrt(wb.box ** 3)
    ks_ref = eta * l / np.pi * np.sqrt(8 / kc) * np.exp(-(np.pi * kc / (eta * l)) ** 2)
    assert abs(ks - ks_ref) <= 1e-13 * ks_ref
    assert abs(rs - 2 / np.sqrt(rc / l) * np.exp(-(rc * eta) ** 2)) <= 1e-13 * rs
    # no k-space, no real space: zero estimates
    z = ElecLJ(kspace_cutoff=kc, rspace_cutoff=rc, include_kspace=False, include_rspace=False,
               ewald_screening=0.3).init(wb)
    assert z.error_estimates() == (0.0, 0.0)

"""The oracle's restated per-site gradients (oracle/adjoint_oracle.py) against
central differences of the oracle's own energy and forces, on the CPU: the
Ewald k-sum on a water box, and a box with cross-group exclusions, screening
radii, scaled 1-4 pairs and LJ on the H sites.  Directional derivatives along
seeded non-uniform directions (per-site charges, H charges only, one site,
integer sigma and epsilon patterns), Richardson-extrapolated central
differences; the same bound the GPU gradients meet against these differences."""
import numpy as np
import pytest

from molmodel_b200 import water_box
from oracle.adjoint_oracle import site_gradients
from oracle.oracle import port

from adjoint_cases import CASES, System, directional_fd, directions, grad_key, oracle_eval

KSUM = [c for c in CASES if "kspace_cutoff" in c[2]]


@pytest.mark.parametrize("name,extra,cfg", KSUM, ids=[c[0] for c in KSUM])
def test_restated_gradients_match_finite_differences(name, extra, cfg):
    wb = water_box(6, seed=11)
    s = System(wb, extra)
    tq = s.q * 1.04
    tsig = np.where(np.arange(s.nsite) % 3 == 0, s.sigma + 0.03, s.sigma)
    targets = oracle_eval(s, cfg, q=tq, sig=tsig)["f"]
    f0 = oracle_eval(s, cfg)["f"]
    g = site_gradients(port(), s, cfg, s.positions, 2 * (f0 - targets), pairs14=s.pairs14)
    rng = np.random.default_rng(5)
    for label, which, v, h in directions(s, rng):
        fd_u, fd_l = directional_fd(s, cfg, which, v, h, targets)
        k = grad_key(which)
        pu, pl = float(v @ g["du_" + k]), float(v @ g["dl_" + k])
        assert abs(pu - fd_u) <= 3e-8 * abs(fd_u) + 1e-9, (name, label, pu, fd_u)
        assert abs(pl - fd_l) <= 3e-8 * abs(fd_l) + 1e-9, (name, label, pl, fd_l)

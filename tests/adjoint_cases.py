"""Cases shared by the adjoint tests: water boxes with and without the extra
terms (cross-group exclusions, screening radii, 1-4 pairs, LJ on H), the
oracle's energy and forces at changed parameters, and Richardson-extrapolated
central differences along seeded directions."""
import numpy as np

from molmodel_b200.water import SITE_HAS_LJ, SITE_HAS_Q
from oracle.oracle import make_config, port


class System:
    """Site arrays of a water box, optionally with the extra terms."""

    def __init__(self, wb, extra=False, seed=3):
        self.nsite, self.box, self.positions = wb.nsite, wb.box, wb.positions
        self.groups, self.exclusions = wb.groups, wb.exclusions
        self.site_mask = wb.site_mask.copy()
        self.q, self.sigma, self.epsilon = wb.q.copy(), wb.sigma.copy(), wb.epsilon.copy()
        self.rscreen = np.zeros(wb.nsite)
        self.pairs14 = None
        if extra:
            rng = np.random.default_rng(seed)
            n = wb.nwater
            k = rng.choice(n - 1, size=n // 4, replace=False)
            more = np.concatenate([np.stack([3 * k, 3 * (k + 1)], 1), np.stack([3 * k + 1, 3 * (k + 1) + 2], 1)])
            self.exclusions = np.concatenate([wb.exclusions, more]).astype(np.int32)
            self.rscreen = np.where(np.arange(wb.nsite) % 3 == 0, 1.6, 0.0)
            j = rng.choice(n - 3, size=n // 5, replace=False)
            self.pairs14 = np.concatenate([np.stack([3 * j, 3 * (j + 2)], 1),
                                           np.stack([3 * j, 3 * (j + 3) + 1], 1)]).astype(np.int32)
            h = np.arange(wb.nsite) % 3 != 0
            self.site_mask = np.full(wb.nsite, SITE_HAS_Q | SITE_HAS_LJ, dtype=np.int32)
            self.sigma = np.where(h, 1.0, self.sigma)
            self.epsilon = np.where(h, 0.01, self.epsilon)


def oracle_eval(s, cfg, q=None, sig=None, eps=None):
    o = port().eleclj(make_config(s.box, **cfg), s.nsite, s.groups, s.exclusions, s.site_mask,
                      s.q if q is None else q, s.sigma if sig is None else sig, s.epsilon if eps is None else eps,
                      s.rscreen, pairs14=s.pairs14)
    return o.eval(s.positions)


def directional_fd(s, cfg, which, v, h, targets):
    """Richardson-extrapolated central differences of U and L along v."""
    base = dict(q=s.q, sig=s.sigma, eps=s.epsilon)

    def at(t):
        p = dict(base)
        p[which] = base[which] + t * v
        out = oracle_eval(s, cfg, **p)
        return out["total"], float(((out["f"] - targets) ** 2).sum())

    d = []
    for hh in (h, 2 * h):
        (up, lp), (um, lm) = at(hh), at(-hh)
        d.append(((up - um) / (2 * hh), (lp - lm) / (2 * hh)))
    return tuple((4 * d[0][k] - d[1][k]) / 3 for k in range(2))


def directions(s, rng):
    """(name, parameter, direction, step) for the checks."""
    qm = (s.site_mask & SITE_HAS_Q) != 0
    lm = (s.site_mask & SITE_HAS_LJ) != 0
    hsite = np.arange(s.nsite) % 3 != 0
    out = [
        ("q-random", "q", np.where(qm, rng.normal(size=s.nsite), 0.0), 1e-3),
        ("q-H-only", "q", np.where(qm & hsite, rng.normal(size=s.nsite), 0.0), 1e-3),
        ("q-one-site", "q", np.eye(s.nsite)[4], 1e-3),
        ("sigma", "sig", np.where(lm, rng.integers(-2, 3, size=s.nsite), 0).astype(float), 1e-4),
        ("epsilon", "eps", np.where(lm, rng.integers(-2, 3, size=s.nsite), 0).astype(float), 1e-5),
    ]
    return out


CFG = dict(rspace_cutoff=9.0, smoothing_width=1.0, ewald_screening=0.35)
CASES = [
    ("ksum", False, dict(CFG, kspace_cutoff=7.0)),
    ("p3m", False, dict(CFG, use_p3m=True, p3m_grid_spacing=18.63 / 20, p3m_assignment_order=5)),
    ("p3m-ik", False, dict(CFG, use_p3m=True, p3m_grid_spacing=18.63 / 20, p3m_assignment_order=4,
                           p3m_ik_differentiate=True)),
    ("general", True, dict(CFG, kspace_cutoff=7.0, elec_1_4_scale_factor=0.5, lj_1_4_scale_factor=0.7)),
    ("general-p3m", True, dict(CFG, use_p3m=True, p3m_grid_spacing=18.63 / 20, p3m_assignment_order=5,
                               elec_1_4_scale_factor=0.5, lj_1_4_scale_factor=0.7)),
]


def grad_key(which):
    return {"q": "dq", "sig": "dsig", "eps": "deps"}[which]

"""ctypes wrapper over the two CPU oracles — TEST INFRASTRUCTURE ONLY.

``port()`` loads the oracle's own C restatement (oracle/_build/liborc.so);
``reference()`` loads the reference's own sources compiled by oracle/Makefile
(oracle/_ref/libref.so).  Both export the interface of oracle/oracle_api.h.
Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline and
reference legs may import this module; the product never does.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_build", "liborc.so")
REF_LIB = os.path.join(HERE, "_ref", "libref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p


class Config(ctypes.Structure):
    """orc_config (oracle/oracle_api.h)."""
    _fields_ = [
        ("bctype", ctypes.c_int),
        ("box", ctypes.c_double * 3),
        ("rspace_cutoff", ctypes.c_double),
        ("smoothing_width", ctypes.c_double),
        ("neighbor_list_width", ctypes.c_double),
        ("kspace_cutoff", ctypes.c_double),
        ("ewald_screening", ctypes.c_double),
        ("use_p3m", ctypes.c_int),
        ("p3m_grid_spacing", ctypes.c_double),
        ("p3m_assignment_order", ctypes.c_int),
        ("p3m_alias_sum_limit", ctypes.c_int),
        ("p3m_ik_differentiate", ctypes.c_int),
        ("include_lj_correction", ctypes.c_int),
        ("geometric_combining_for_sigma", ctypes.c_int),
        ("include_rspace", ctypes.c_int),
        ("include_kspace", ctypes.c_int),
        ("include_self", ctypes.c_int),
        ("elec_1_4_scale_factor", ctypes.c_double),
        ("lj_1_4_scale_factor", ctypes.c_double),
    ]


class Energy(ctypes.Structure):
    _fields_ = [("elec", ctypes.c_double), ("lj", ctypes.c_double),
                ("lj_correction", ctypes.c_double), ("total", ctypes.c_double)]


def make_config(box, bctype=1, rspace_cutoff=9.0, smoothing_width=1.0, neighbor_list_width=0.0,
                kspace_cutoff=5.0, ewald_screening=0.35, use_p3m=False, p3m_grid_spacing=0.5,
                p3m_assignment_order=3, p3m_alias_sum_limit=2, p3m_ik_differentiate=False,
                include_lj_correction=True, geometric_combining_for_sigma=False,
                include_rspace=True, include_kspace=True, include_self=True,
                elec_1_4_scale_factor=1.0, lj_1_4_scale_factor=1.0):
    c = Config()
    c.bctype = bctype
    b = np.broadcast_to(np.asarray(box, dtype=np.float64), (3,))
    c.box = (ctypes.c_double * 3)(*b)
    c.rspace_cutoff = rspace_cutoff
    c.smoothing_width = smoothing_width
    c.neighbor_list_width = neighbor_list_width
    c.kspace_cutoff = kspace_cutoff
    c.ewald_screening = ewald_screening
    c.use_p3m = int(use_p3m)
    c.p3m_grid_spacing = p3m_grid_spacing
    c.p3m_assignment_order = p3m_assignment_order
    c.p3m_alias_sum_limit = p3m_alias_sum_limit
    c.p3m_ik_differentiate = int(p3m_ik_differentiate)
    c.include_lj_correction = int(include_lj_correction)
    c.geometric_combining_for_sigma = int(geometric_combining_for_sigma)
    c.include_rspace = int(include_rspace)
    c.include_kspace = int(include_kspace)
    c.include_self = int(include_self)
    c.elec_1_4_scale_factor = elec_1_4_scale_factor
    c.lj_1_4_scale_factor = lj_1_4_scale_factor
    return c


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class OracleLib:
    def __init__(self, path):
        self.path = path
        L = self.lib = ctypes.CDLL(path)
        L.orc_chebyshev.argtypes = [ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp]
        L.orc_kspace_field.argtypes = [ctypes.c_double, ctypes.c_int, _dp, _dp, _dp, ctypes.c_double,
                                       _dp, _dp, _ip]
        L.orc_p3m_new.restype = _vp
        L.orc_p3m_new.argtypes = [ctypes.c_int, _dp, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_double, _ip, _dp]
        L.orc_p3m_field.argtypes = [_vp, _dp, _dp, _dp, _dp]
        L.orc_p3m_delete.argtypes = [_vp]
        L.orc_nbrlist_new.restype = _vp
        L.orc_nbrlist_new.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp]
        L.orc_nbrlist_update.argtypes = [_vp, _dp]
        L.orc_nbrlist_npairs.restype = ctypes.c_long
        L.orc_nbrlist_npairs.argtypes = [_vp]
        L.orc_nbrlist_pairs.argtypes = [_vp, _ip]
        L.orc_nbrlist_ncell.argtypes = [_vp]
        L.orc_nbrlist_cells.argtypes = [_vp, _ip]
        L.orc_nbrlist_ncellpairs.restype = ctypes.c_long
        L.orc_nbrlist_ncellpairs.argtypes = [_vp]
        L.orc_nbrlist_cellpairs.argtypes = [_vp, _ip]
        L.orc_nbrlist_delete.argtypes = [_vp]
        L.orc_eleclj_new.restype = _vp
        L.orc_eleclj_new.argtypes = [ctypes.POINTER(Config), ctypes.c_int, ctypes.c_int, _ip,
                                     ctypes.c_int, _ip, ctypes.c_int, _ip, _ip, _dp, _dp, _dp, _dp]
        L.orc_eleclj_eval.argtypes = [_vp, _dp, _dp, ctypes.POINTER(Energy), _dp, _dp, _dp]
        L.orc_eleclj_eta.restype = ctypes.c_double
        L.orc_eleclj_eta.argtypes = [_vp]
        L.orc_eleclj_nlw.restype = ctypes.c_double
        L.orc_eleclj_nlw.argtypes = [_vp]
        L.orc_eleclj_nbrlist.restype = _vp
        L.orc_eleclj_nbrlist.argtypes = [_vp]
        L.orc_eleclj_phi_at_points.argtypes = [_vp, _dp, ctypes.c_int, _dp, _dp]
        L.orc_eleclj_delete.argtypes = [_vp]
        L.orc_pairset_demo.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _ip, _ip]
        # the reference's constraint solver (oracle/ref_constraint.cpp; libref.so only)
        self.has_constraints = hasattr(L, "orc_water_constrain_positions")
        if self.has_constraints:
            L.orc_add_search_path.argtypes = [ctypes.c_char_p]
            L.orc_add_search_path(os.path.join(HERE, "shim").encode())
            L.orc_water_constrain_positions.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double,
                                                        ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                        ctypes.c_int]
            L.orc_water_constrain_velocities.argtypes = [ctypes.c_int, _dp, _dp, _dp, ctypes.c_double,
                                                         ctypes.c_double]

    # --- component entry points -------------------------------------------
    def chebyshev(self, rc, eta):
        mn, mx, inv = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        coeff = np.zeros((512, 7))
        self.lib.orc_chebyshev(rc, eta, ctypes.byref(mn), ctypes.byref(mx), ctypes.byref(inv), _d(coeff))
        return mn.value, mx.value, inv.value, coeff

    def kspace_field(self, kc, r, q, latv, eta):
        r, q, latv = _f64(r), _f64(q), _f64(latv)
        n = len(q)
        phi = np.zeros(n)
        evec = np.zeros((n, 3))
        nk = ctypes.c_int()
        self.lib.orc_kspace_field(kc, n, _d(r), _d(q), _d(latv), eta, _d(phi), _d(evec), ctypes.byref(nk))
        return phi, evec, nk.value

    def p3m_field(self, r, q, latv, spacing, order, eta, nalias=2, ik=False):
        r, q, latv = _f64(r), _f64(q), _f64(latv)
        n = len(q)
        ngrid = np.zeros(3, dtype=np.int32)
        chi = ctypes.c_double()
        h = self.lib.orc_p3m_new(n, _d(latv), spacing, nalias, int(ik), order, eta, _i(ngrid),
                                 ctypes.byref(chi))
        phi = np.zeros(n)
        evec = np.zeros((n, 3))
        self.lib.orc_p3m_field(h, _d(r), _d(q), _d(phi), _d(evec))
        self.lib.orc_p3m_delete(h)
        return phi, evec, tuple(int(x) for x in ngrid), chi.value

    def p3m_chi(self, latv, spacing, order, eta, nalias=2, ik=False):
        """p3m_init's dimensionless RMS force error estimate (src/pppm.c:313-393)
        for the mesh p3m_new picks (src/pppm.c:395-447); returns (chi, mesh)."""
        ngrid = np.zeros(3, dtype=np.int32)
        chi = ctypes.c_double()
        h = self.lib.orc_p3m_new(0, _d(_f64(latv)), spacing, nalias, int(ik), order, eta, _i(ngrid),
                                 ctypes.byref(chi))
        self.lib.orc_p3m_delete(h)
        return chi.value, tuple(int(x) for x in ngrid)

    def p3m_optimize_objective(self, latv, spacing, order, rc, eta, nalias=2, ik=False):
        """p3m_optimize_help (src/pppm.c:672-681): chi_r^2 + chi_k^2 at eta, 1e8
        for a negative eta."""
        if eta < 0:
            return 1e8
        v = abs(np.linalg.det(_f64(latv).reshape(3, 3)))
        chi_r = 2 / np.sqrt(rc / v ** (1.0 / 3.0)) * np.exp(-(rc * eta) ** 2)
        return chi_r ** 2 + self.p3m_chi(latv, spacing, order, eta, nalias, ik)[0] ** 2

    def p3m_optimize(self, latv, spacing, order, rc, nalias=2, ik=False, tol=1e-9):
        """The minimiser of p3m_optimize's objective (src/pppm.c:682-716).  The
        reference finds it with GSL's simplex (gsl_multimin_fminimizer_nmsimplex,
        size tolerance 1e-4), which the oracle build does not have; this
        restatement brackets the minimum on a coarse scan of the same objective
        and closes the bracket by golden-section search to ``tol``, so it gives the
        point the simplex converges to, not the simplex's own last vertex."""
        f = lambda e: self.p3m_optimize_objective(latv, spacing, order, rc, e, nalias, ik)
        grid = np.linspace(0.02, 1.5, 75)
        vals = [f(e) for e in grid]
        k = int(np.argmin(vals))
        a, b = grid[max(k - 1, 0)], grid[min(k + 1, len(grid) - 1)]
        g = (np.sqrt(5) - 1) / 2
        c, d = b - g * (b - a), a + g * (b - a)
        fc, fd = f(c), f(d)
        while b - a > tol:
            if fc < fd:
                b, d, fd = d, c, fc
                c = b - g * (b - a)
                fc = f(c)
            else:
                a, c, fc = c, d, fd
                d = a + g * (b - a)
                fd = f(d)
        return 0.5 * (a + b)

    def water_constrain_positions(self, r0, r, v, mass3, dt, r_oh=1.0, angle_deg=109.47, tol=1e-12,
                                  maxit=10000):
        """ConstraintGroup::constrain_positions (src/constraint.cpp:295-335) on every
        rigid water (two O-H lengths and the H-O-H angle): returns new r, v."""
        r0, r, v = _f64(r0), _f64(r).copy(), _f64(v).copy()
        nmol = r.size // 9
        self.lib.orc_water_constrain_positions(nmol, _d(r0), _d(r), _d(v), _d(_f64(mass3)), dt, r_oh, angle_deg,
                                               tol, maxit)
        return r, v

    def water_constrain_velocities(self, r, v, mass3, r_oh=1.0, angle_deg=109.47):
        """ConstraintGroup::constrain_velocities (src/constraint.cpp:336-358): returns new v."""
        r, v = _f64(r), _f64(v).copy()
        self.lib.orc_water_constrain_velocities(r.size // 9, _d(r), _d(v), _d(_f64(mass3)), r_oh, angle_deg)
        return v

    def pairset(self, n, adds):
        """Rows and membership matrix of a PairBinary built from ``adds``."""
        adds = _i32(adds)
        cnt = np.zeros(n, dtype=np.int32)
        rows = np.full((n, n), -1, dtype=np.int32)
        ex = np.zeros((n, n), dtype=np.int32)
        self.lib.orc_pairset_demo(n, len(adds), _i(adds), _i(cnt), _i(rows), _i(ex))
        return [list(rows[i, :cnt[i]]) for i in range(n)], ex

    def nbrlist(self, ngroup, cutoff, width, box, bctype=1):
        return NbrList(self, self.lib.orc_nbrlist_new(ngroup, cutoff, width, bctype,
                                                      _d(_f64(np.broadcast_to(box, (3,))))), own=True)

    def eleclj(self, config, nsite, groups, exclusions, site_mask, q, sig, eps, rscreen, pairs14=None):
        groups, exclusions, site_mask = _i32(groups), _i32(exclusions), _i32(site_mask)
        q, sig, eps, rscreen = _f64(q), _f64(sig), _f64(eps), _f64(rscreen)
        p14 = _i32(pairs14 if pairs14 is not None else np.zeros((0, 2)))
        h = self.lib.orc_eleclj_new(ctypes.byref(config), nsite, len(groups), _i(groups),
                                    len(exclusions), _i(exclusions), len(p14), _i(p14),
                                    _i(site_mask), _d(q), _d(sig), _d(eps), _d(rscreen))
        if not h:
            raise ValueError("oracle rejected the ElecLJ configuration")
        return ElecLJ(self, h, nsite, (config, nsite, groups, exclusions, site_mask, q, sig, eps,
                                       rscreen, p14))


class NbrList:
    def __init__(self, lib, h, own):
        self.L, self.h, self.own = lib, h, own

    def update(self, gr):
        return bool(self.L.lib.orc_nbrlist_update(self.h, _d(_f64(gr))))

    def pairs(self):
        n = self.L.lib.orc_nbrlist_npairs(self.h)
        p = np.zeros((n, 2), dtype=np.int32)
        if n:
            self.L.lib.orc_nbrlist_pairs(self.h, _i(p))
        return p

    def cells(self, ngroup):
        c = np.zeros(ngroup, dtype=np.int32)
        self.L.lib.orc_nbrlist_cells(self.h, _i(c))
        return c

    def ncell(self):
        return self.L.lib.orc_nbrlist_ncell(self.h)

    def cellpairs(self):
        n = self.L.lib.orc_nbrlist_ncellpairs(self.h)
        p = np.zeros((n, 2), dtype=np.int32)
        if n:
            self.L.lib.orc_nbrlist_cellpairs(self.h, _i(p))
        return p

    def __del__(self):
        if self.own and self.h:
            self.L.lib.orc_nbrlist_delete(self.h)
            self.h = None


class ElecLJ:
    def __init__(self, lib, h, nsite, keep):
        self.L, self.h, self.nsite, self._keep = lib, h, nsite, keep

    def eval(self, r):
        r = _f64(r)
        n = self.nsite
        f = np.zeros((n, 3))
        phi = np.zeros(n)
        evec = np.zeros((n, 3))
        ljf = np.zeros((n, 3))
        e = Energy()
        self.L.lib.orc_eleclj_eval(self.h, _d(r), _d(f), ctypes.byref(e), _d(phi), _d(evec), _d(ljf))
        return dict(f=f, phi=phi, evec=evec, ljf=ljf, elec=e.elec, lj=e.lj,
                    lj_correction=e.lj_correction, total=e.total)

    def phi_at_points(self, r, points):
        """Potential of the sites at r at the points (ElecLJ::electrostatic_potential_at_gridpoints)."""
        r, pts = _f64(r), _f64(points).reshape(-1, 3)
        phi = np.zeros(len(pts))
        self.L.lib.orc_eleclj_phi_at_points(self.h, _d(r), len(pts), _d(pts), _d(phi))
        return phi

    @property
    def eta(self):
        return self.L.lib.orc_eleclj_eta(self.h)

    @property
    def nlw(self):
        return self.L.lib.orc_eleclj_nlw(self.h)

    def nbrlist(self):
        return NbrList(self.L, self.L.lib.orc_eleclj_nbrlist(self.h), own=False)

    def __del__(self):
        if self.h:
            self.L.lib.orc_eleclj_delete(self.h)
            self.h = None


_cache = {}


def port():
    """The oracle's own restatement; raises if it has not been built."""
    if "port" not in _cache:
        if not os.path.exists(PORT_LIB):
            raise FileNotFoundError(f"{PORT_LIB} missing: run `make -C oracle port`")
        _cache["port"] = OracleLib(PORT_LIB)
    return _cache["port"]


def reference():
    """The reference's own code, or None where it was not built."""
    if "ref" not in _cache:
        _cache["ref"] = OracleLib(REF_LIB) if os.path.exists(REF_LIB) else None
    return _cache["ref"]


def water_eleclj(lib, wb, **cfg):
    """An ElecLJ oracle instance for a molmodel_b200.water.WaterBox."""
    c = make_config(wb.box, **cfg)
    return lib.eleclj(c, wb.nsite, wb.groups, wb.exclusions, wb.site_mask, wb.q, wb.sigma,
                      wb.epsilon, wb.rscreen)

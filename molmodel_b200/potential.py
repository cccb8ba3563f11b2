"""Python mirror of the reference's ElecLJ potential over libmmnb.

``ElecLJ`` keeps the reference's names and argument meanings
(include/eleclj.hpp:303-397, include/pot.hpp:6-28): the same input fields with
the same defaults (src/eleclj.cpp:13-40), ``init(system)`` to bind a system,
``add_to_energy_and_forces(u, f)`` which ADDS to the forces and returns the
energy added to ``u``, and ``scale(s)`` for volume moves.  Failures raise
``MmnbError`` where the reference would call die().
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import MmnbConfig, MmnbEnergy, check, load

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def measure_fp32_peak(device=-1):
    """FP32 FMA throughput of a GPU in TFLOP/s (mmnb_measure_fp32_peak)."""
    t = ctypes.c_double(0.0)
    check(load().mmnb_measure_fp32_peak(int(device), ctypes.byref(t)))
    return t.value


class ElecLJ:
    """Real-space Ewald + LJ with P3M or ordinary-Ewald reciprocal space."""

    def __init__(self, precision="fp64", rspace_cutoff=0.0, smoothing_width=1.0,
                 neighbor_list_width=0.0, kspace_cutoff=5.0, ewald_screening=-1.0,
                 use_p3m=False, p3m_grid_spacing=0.5, p3m_grid_density=-1.0, p3m_assignment_order=3,
                 p3m_alias_sum_limit=2, p3m_ik_differentiate=False,
                 include_lj_correction=True, geometric_combining_for_sigma=False,
                 include_rspace=True, include_kspace=True, include_self=True,
                 elec_1_4_scale_factor=1.0, lj_1_4_scale_factor=1.0,
                 rebuild_interval=0, device=-1):
        self.precision = precision
        self.rspace_cutoff = rspace_cutoff
        self.smoothing_width = smoothing_width
        self.neighbor_list_width = neighbor_list_width
        self.kspace_cutoff = kspace_cutoff
        self.ewald_screening = ewald_screening
        self.use_p3m = use_p3m
        self.p3m_grid_spacing = p3m_grid_spacing
        self.p3m_grid_density = p3m_grid_density
        self.p3m_assignment_order = p3m_assignment_order
        self.p3m_alias_sum_limit = p3m_alias_sum_limit
        self.p3m_ik_differentiate = p3m_ik_differentiate
        self.include_lj_correction = include_lj_correction
        self.geometric_combining_for_sigma = geometric_combining_for_sigma
        self.include_rspace = include_rspace
        self.include_kspace = include_kspace
        self.include_self = include_self
        self.elec_1_4_scale_factor = elec_1_4_scale_factor
        self.lj_1_4_scale_factor = lj_1_4_scale_factor
        self.rebuild_interval = rebuild_interval
        self.device = device
        self._h = None
        self._cells = None
        self.energy = None

    # ---- set-up --------------------------------------------------------------
    def _config(self, box, bctype):
        lib = load()
        c = MmnbConfig()
        lib.mmnb_config_init(ctypes.byref(c))
        c.precision = {"fp64": _lib.MMNB_FP64, "mixed": _lib.MMNB_MIXED}[self.precision]
        c.bctype = bctype
        b = np.broadcast_to(np.asarray(box, dtype=np.float64), (3,))
        c.box = (ctypes.c_double * 3)(*b)
        for name in ("rspace_cutoff", "smoothing_width", "neighbor_list_width", "kspace_cutoff",
                     "ewald_screening", "p3m_grid_spacing", "p3m_grid_density", "elec_1_4_scale_factor",
                     "lj_1_4_scale_factor"):
            setattr(c, name, float(getattr(self, name)))
        for name in ("use_p3m", "p3m_assignment_order", "p3m_alias_sum_limit", "p3m_ik_differentiate",
                     "include_lj_correction", "geometric_combining_for_sigma", "include_rspace",
                     "include_kspace", "include_self", "rebuild_interval", "device"):
            setattr(c, name, int(getattr(self, name)))
        return c

    def init(self, system, bctype=_lib.MMNB_CUBIC, pairs14=None):
        """Bind a system: anything with ``box``, ``nsite``, ``groups``,
        ``exclusions``, ``site_mask``, ``q``, ``sigma``, ``epsilon`` and
        ``rscreen`` (molmodel_b200.water.WaterBox is one)."""
        self.close()
        lib = load()
        c = self._config(system.box, bctype)
        groups = np.ascontiguousarray(system.groups, dtype=np.int32)
        excl = np.ascontiguousarray(system.exclusions, dtype=np.int32)
        p14 = np.ascontiguousarray(pairs14 if pairs14 is not None else np.zeros((0, 2)), dtype=np.int32)
        h = ctypes.c_void_p()
        st = lib.mmnb_create(ctypes.byref(c), int(system.nsite), len(groups), _i(groups), len(excl), _i(excl),
                             len(p14), _i(p14), ctypes.byref(h))
        if st:
            raise _lib.MmnbError(st, lib.mmnb_last_error(None).decode())
        self._h = h
        self._groups = groups
        self.nsite = int(system.nsite)
        self.set_params(system.site_mask, system.q, system.sigma, system.epsilon, system.rscreen)
        return self

    def set_params(self, site_mask, q, sigma, epsilon, rscreen=None):
        lib = load()
        m = np.ascontiguousarray(site_mask, dtype=np.int32)
        q = np.ascontiguousarray(q, dtype=np.float64)
        s = np.ascontiguousarray(sigma, dtype=np.float64)
        e = np.ascontiguousarray(epsilon, dtype=np.float64)
        r = None if rscreen is None else np.ascontiguousarray(rscreen, dtype=np.float64)
        check(lib.mmnb_set_params(self._h, _i(m), _d(q), _d(s), _d(e), _d(r)), self._h)

    # ---- evaluation -----------------------------------------------------------
    def compute(self, r, want_fields=False):
        """Energy and forces for positions r (nsite x 3); returns a dict."""
        lib = load()
        r = np.ascontiguousarray(r, dtype=np.float64)
        f = np.zeros((self.nsite, 3))
        e = MmnbEnergy()
        phi = np.zeros(self.nsite) if want_fields else None
        evec = np.zeros((self.nsite, 3)) if want_fields else None
        check(lib.mmnb_compute(self._h, _d(r), _d(f), None, ctypes.byref(e), _d(phi), _d(evec)), self._h)
        self.energy = dict(elec=e.elec, lj=e.lj, lj_correction=e.lj_correction, total=e.total)
        out = dict(f=f, **self.energy)
        if want_fields:
            out.update(phi=phi, evec=evec)
        return out

    # ---- adjoint --------------------------------------------------------------
    def forward(self, r):
        """mmnb_forward: compute() that keeps on the device what
        site_gradients() needs.  Returns compute()'s dict."""
        lib = load()
        r = np.ascontiguousarray(r, dtype=np.float64)
        f = np.zeros((self.nsite, 3))
        e = MmnbEnergy()
        check(lib.mmnb_forward(self._h, _d(r), _d(f), None, ctypes.byref(e)), self._h)
        self.energy = dict(elec=e.elec, lj=e.lj, lj_correction=e.lj_correction, total=e.total)
        return dict(f=f, **self.energy)

    def site_gradients(self, dl_df=None):
        """mmnb_site_gradients for the last forward(): per-site arrays du_dq,
        du_dsig, du_deps (dU/dq_i, dU/dsigma_i, dU/depsilon_i) and, given
        dl_df = dL/dF (nsite x 3), dl_dq, dl_dsig, dl_deps for that loss."""
        n = self.nsite
        out = {k: np.zeros(n) for k in ("du_dq", "du_dsig", "du_deps")}
        g = None
        if dl_df is not None:
            g = np.ascontiguousarray(dl_df, dtype=np.float64).reshape(n, 3)
            out.update({k: np.zeros(n) for k in ("dl_dq", "dl_dsig", "dl_deps")})
        check(load().mmnb_site_gradients(self._h, _d(g), _d(out["du_dq"]), _d(out["du_dsig"]),
                                         _d(out["du_deps"]), _d(out.get("dl_dq")), _d(out.get("dl_dsig")),
                                         _d(out.get("dl_deps"))), self._h)
        return out

    def electrostatic_potential_at_gridpoints(self, r, points):
        """ElecLJ::electrostatic_potential_at_gridpoints (src/eleclj.cpp:1302-1340):
        potential of the sites at r (nsite x 3) at each point (npoint x 3), in
        the units of compute()'s phi; real space, the kspace_cutoff k-sum and
        the neutralising term, each as include_rspace / include_kspace /
        include_self say."""
        lib = load()
        r = np.ascontiguousarray(r, dtype=np.float64)
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        phi = np.zeros(len(pts))
        check(lib.mmnb_phi_at_points(self._h, _d(r), len(pts), _d(pts), _d(phi)), self._h)
        return phi

    def add_to_energy_and_forces(self, u, f, r):
        """Potential::add_to_energy_and_forces: forces are added to ``f``
        (nsite x 3, float64, in place); returns ``u`` plus the energy."""
        lib = load()
        if f.dtype != np.float64 or not f.flags.c_contiguous:
            raise ValueError("f must be a C-contiguous float64 array")
        if not isinstance(r, np.ndarray) or r.dtype != np.float64 or not r.flags.c_contiguous:
            r = np.ascontiguousarray(r, dtype=np.float64)
        # per-call marshalling kept small (this is the per-step call): raw
        # addresses and the potential's own energy and u cells
        if self._cells is None:
            self._cells = (ctypes.c_double(0.0), MmnbEnergy())
        uu, e = self._cells
        uu.value = u
        check(lib.mmnb_compute(self._h, r.ctypes.data, f.ctypes.data, ctypes.addressof(uu), ctypes.addressof(e),
                               None, None), self._h)
        self.energy = dict(elec=e.elec, lj=e.lj, lj_correction=e.lj_correction, total=e.total)
        return uu.value

    def check(self):
        """mmnb_check: status of the evaluations since the last check on device
        arrays.  Returns (truncated evaluations, longest row needed); raises
        MmnbError (status MMNB_ERR_OVERFLOW or MMNB_ERR_DEVICE) when rows were
        cut at their capacity or a coordinate was not finite."""
        t = ctypes.c_long(0)
        m = ctypes.c_int(0)
        check(load().mmnb_check(self._h, ctypes.byref(t), ctypes.byref(m)), self._h)
        return t.value, m.value

    def virial(self, r, masses, molecules=None):
        """dU/ds at s = 1 along the reference's volume-move path (mmnb_virial):
        box x s, each molecule moved rigidly so its centre of mass is x s,
        eta / s.  ``molecules``: (nmol, 2) half-open site ranges (default: the
        groups).  Returns (w, energy dict, forces)."""
        lib = load()
        r = np.ascontiguousarray(r, dtype=np.float64)
        m = np.ascontiguousarray(masses, dtype=np.float64)
        mol = np.ascontiguousarray(self._groups if molecules is None else molecules, dtype=np.int32)
        f = np.zeros((self.nsite, 3))
        e = MmnbEnergy()
        w = ctypes.c_double(0.0)
        check(lib.mmnb_virial(self._h, _d(r), len(mol), _i(mol), _d(m), _d(f), None, ctypes.byref(e),
                              ctypes.byref(w)), self._h)
        return w.value, dict(elec=e.elec, lj=e.lj, lj_correction=e.lj_correction, total=e.total), f

    def autotune(self, r, iters=10):
        """Time the launch choices at positions r and keep the fastest;
        returns them (see tuning)."""
        r = np.ascontiguousarray(r, dtype=np.float64)
        check(load().mmnb_autotune(self._h, _d(r), int(iters)), self._h)
        return self.tuning

    @property
    def tuning(self):
        """(water kernel register budget code, spread layout, P3M side stream,
        FP64 water kernel warps per block), see mmnb_get_tuning."""
        t = np.zeros(4, dtype=np.int32)
        check(load().mmnb_get_tuning(self._h, _i(t)), self._h)
        return tuple(int(x) for x in t)

    @tuning.setter
    def tuning(self, values):
        values = list(values)
        if len(values) == 3:  # the FP64 choice kept
            values.append(self.tuning[3])
        t = np.ascontiguousarray(values, dtype=np.int32)
        if t.shape != (4,):
            raise ValueError("tuning takes 3 or 4 values")
        check(load().mmnb_set_tuning(self._h, _i(t)), self._h)

    def compute_device(self, d_r, d_f, d_energy):
        """Asynchronous evaluation on device pointers (ints), see mmnb_compute_device."""
        check(load().mmnb_compute_device(self._h, ctypes.c_void_p(d_r), ctypes.c_void_p(d_f),
                                         ctypes.c_void_p(d_energy)), self._h)

    def graph_capture(self, d_r, d_f, d_energy):
        """Capture one device evaluation into a CUDA graph (mmnb_graph_capture)."""
        check(load().mmnb_graph_capture(self._h, ctypes.c_void_p(d_r), ctypes.c_void_p(d_f),
                                        ctypes.c_void_p(d_energy)), self._h)

    def graph_launch(self):
        check(load().mmnb_graph_launch(self._h), self._h)

    def set_stream(self, stream_ptr):
        check(load().mmnb_set_stream(self._h, ctypes.c_void_p(stream_ptr)), self._h)

    def scale(self, s):
        """Volume move by factor s (ElecLJ::scale)."""
        check(load().mmnb_scale(self._h, float(s)), self._h)

    # ---- inspection -----------------------------------------------------------
    def pairlist(self):
        lib = load()
        n = ctypes.c_long()
        check(lib.mmnb_get_pairlist(self._h, ctypes.byref(n), None, 0), self._h)
        p = np.zeros((n.value, 2), dtype=np.int32)
        check(lib.mmnb_get_pairlist(self._h, ctypes.byref(n), _i(p), n.value), self._h)
        return p

    def cells(self, ngroup):
        c = np.zeros(ngroup, dtype=np.int32)
        nc = ctypes.c_int()
        check(load().mmnb_get_cells(self._h, _i(c), ctypes.byref(nc)), self._h)
        return c, nc.value

    def counters(self):
        rb, ev = ctypes.c_long(), ctypes.c_long()
        check(load().mmnb_get_counters(self._h, ctypes.byref(rb), ctypes.byref(ev)), self._h)
        return rb.value, ev.value

    def launches(self):
        n = ctypes.c_long()
        check(load().mmnb_get_launches(self._h, ctypes.byref(n)), self._h)
        return n.value

    def settings(self):
        rc, nlw, eta = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        mesh = np.zeros(3, dtype=np.int32)
        check(load().mmnb_get_settings(self._h, ctypes.byref(rc), ctypes.byref(nlw), ctypes.byref(eta),
                                       _i(mesh)), self._h)
        return dict(rc=rc.value, nlw=nlw.value, eta=eta.value, mesh=tuple(int(x) for x in mesh))

    def error_estimates(self):
        """(real space, reciprocal space) dimensionless RMS force error estimates,
        the two figures ElecLJ::init reports (src/eleclj.cpp:225, 233-243)."""
        rs, ks = ctypes.c_double(), ctypes.c_double()
        check(load().mmnb_get_error_estimates(self._h, ctypes.byref(rs), ctypes.byref(ks)), self._h)
        return rs.value, ks.value

    def set_timing(self, on=True):
        check(load().mmnb_set_timing(self._h, int(on)), self._h)

    def timing(self):
        ms = (ctypes.c_double * 64)()
        names = ctypes.create_string_buffer(4096)
        n = load().mmnb_get_timing(self._h, ms, 64, names, 4096)
        keys = names.value.decode().split(",") if n > 0 else []
        return dict(zip(keys, list(ms)[:n]))

    def close(self):
        if self._h is not None:
            load().mmnb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

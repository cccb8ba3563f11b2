"""Device molecular dynamics over libmmnb (the mmnb_md_* entry points).

``MDyn`` mirrors the part of the reference's MDyn (include/mdyn.hpp,
src/mdyn.cpp:120-200) that the nonbonded path drives: velocity Verlet with
the timestep in ps, rigid 3-site water constraints (the reference's
ConstraintGroup, solved here in closed form), and the per-step "Conserved
energy" (kinetic + potential) the reference prints.
"""
import ctypes

import numpy as np

from ._lib import MmnbError, load

_dp = ctypes.POINTER(ctypes.c_double)

MASS_UNIT_PER_G_MOL = 1.0 / 418.4  # include/units.h:166-168: g/mol -> mass unit


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


class MDyn:
    """Velocity Verlet on the GPU for a bound ``ElecLJ`` potential.

    masses: per-site masses in g/mol (converted to the reference's mass unit).
    timestep: ps.  rigid_water: constrain every [O, H, H] group to O-H = r_oh
    and H-O-H = hoh_angle (degrees)."""

    def __init__(self, potential, masses, timestep=0.001, rigid_water=True, r_oh=1.0, hoh_angle=109.47):
        self.potential = potential
        self.timestep = timestep
        lib = load()
        m = np.ascontiguousarray(np.asarray(masses, dtype=np.float64) * MASS_UNIT_PER_G_MOL)
        h = ctypes.c_void_p()
        st = lib.mmnb_md_create(potential._h, _d(m), float(timestep), 1 if rigid_water else 0, float(r_oh),
                                float(hoh_angle), ctypes.byref(h))
        if st:
            raise MmnbError(st, "mmnb_md_create: " + lib.mmnb_status_string(st).decode())
        self._md = h
        self.nsite = potential.nsite
        self.masses = m

    def _check(self, st):
        if st:
            raise MmnbError(st, load().mmnb_md_last_error(self._md).decode())

    def set_state(self, r, v=None):
        r = np.ascontiguousarray(r, dtype=np.float64)
        v = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        self._check(load().mmnb_md_set_state(self._md, _d(r), _d(v)))

    def run(self, steps):
        """Advance `steps` steps; returns an array (steps, 3): kinetic,
        potential and conserved energy (kcal/mol) after each step."""
        e = np.zeros((steps, 3))
        self._check(load().mmnb_md_run(self._md, int(steps), _d(e)))
        return e

    def state(self):
        r = np.zeros((self.nsite, 3))
        v = np.zeros((self.nsite, 3))
        self._check(load().mmnb_md_get_state(self._md, _d(r), _d(v)))
        return r, v

    def scale_velocities(self, factor):
        self._check(load().mmnb_md_scale_velocities(self._md, float(factor)))

    def close(self):
        if getattr(self, "_md", None):
            load().mmnb_md_destroy(self._md)
            self._md = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ReplicaBatch:
    """Several MDyn integrators (each with its own potential handle) advanced
    together: one CUDA graph launch per step with a branch per replica."""

    def __init__(self, mds):
        lib = load()
        self.mds = list(mds)
        arr = (ctypes.c_void_p * len(self.mds))(*[m._md.value for m in self.mds])
        h = ctypes.c_void_p()
        st = lib.mmnb_md_batch_create(arr, len(self.mds), ctypes.byref(h))
        if st:
            raise MmnbError(st, "mmnb_md_batch_create: " + lib.mmnb_status_string(st).decode())
        self._b = h

    def run(self, steps):
        """Advance every replica `steps` steps; returns a list of (steps, 3)
        energy arrays (kinetic, potential, conserved)."""
        out = [np.zeros((steps, 3)) for _ in self.mds]
        ptrs = (_dp * len(out))(*[_d(e) for e in out])
        st = load().mmnb_md_batch_run(self._b, int(steps), ptrs)
        if st:
            raise MmnbError(st, load().mmnb_md_batch_last_error(self._b).decode())
        return out

    def close(self):
        if getattr(self, "_b", None):
            load().mmnb_md_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def nve_drift(energies, timestep, nmolecule):
    """Linear-fit slope of the conserved energy in kcal/mol per ns per
    molecule (the drift the reference's "Conserved energy" line would show)."""
    t_ns = np.arange(1, len(energies) + 1) * timestep * 1e-3
    slope = np.polyfit(t_ns, energies[:, 2], 1)[0]
    return slope / nmolecule

"""Seeded synthetic rigid 3-site water boxes — the inputs of every workload.

The reference measures on no public dataset; all inputs here are generated by
this module from a seed, identically on every machine:

* ``n**3`` waters, one per cell of an n x n x n lattice, the oxygen at the cell
  centre ((i + 1/2) L / n) and the molecule in a uniformly random orientation
  (Shoemake's uniform quaternion from a SplitMix64 counter stream).
* O-H 1.0 A, H-O-H 109.47 degrees, qO = -0.8476 e, qH = +0.4238 e, LJ on O only
  (sigma 3.166 A, epsilon 0.1554 kcal/mol), masses O 15.9994 and H 1.00794.
* Cubic box at 0.997 g/cm^3.

Site order per water is O, H, H: the order ElecLJ::init_sites gives a heavy
atom and its terminal hydrogens (src/eleclj.cpp:668-676), so group g is the
half-open site range [3g, 3g+3) with the oxygen as anchor.  The exclusions are
the two 1-2 pairs and the 1-3 H-H pair (src/eleclj.cpp:712-724).
"""
from dataclasses import dataclass, field
import math

import numpy as np

from .units import AVOGADRO, e_to_charge_unit, K_to_kcal_mol

MASS_O = 15.9994
MASS_H = 1.00794
R_OH = 1.0
THETA_HOH = 109.47
Q_O_E = -0.8476
SIGMA_O = 3.166
EPSILON_O = 0.1554
SITE_HAS_Q = 1   # include/rspace.h:7
SITE_HAS_LJ = 2  # include/rspace.h:8

_MASK64 = (1 << 64) - 1


def splitmix64_uniform(seed, count, offset=0):
    """``count`` doubles in [0, 1) from a SplitMix64 counter stream."""
    i = np.arange(offset + 1, offset + count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed & _MASK64) + i * np.uint64(0x9E3779B97F4A7C15)
        z = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def box_length(nwater, density=0.997):
    """Cubic box edge (A) holding ``nwater`` waters at ``density`` g/cm^3."""
    mass = nwater * (MASS_O + 2 * MASS_H)  # g/mol
    return (mass / (density * AVOGADRO * 0.1)) ** (1.0 / 3.0)


def _rotations(u):
    """Rotation matrices from uniform quaternions (Shoemake 1992)."""
    u1, u2, u3 = u[:, 0], u[:, 1], u[:, 2]
    a, b = np.sqrt(1 - u1), np.sqrt(u1)
    w = a * np.sin(2 * np.pi * u2)
    x = a * np.cos(2 * np.pi * u2)
    y = b * np.sin(2 * np.pi * u3)
    z = b * np.cos(2 * np.pi * u3)
    R = np.empty((len(u), 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


@dataclass
class WaterBox:
    """A rigid-water system in the reference's units and site layout."""
    nwater: int
    box: float                      # cubic edge, A
    positions: np.ndarray           # (3N, 3) f64, A, site order O H H
    masses: np.ndarray              # (3N,) g/mol
    seed: int
    charges_e: np.ndarray = field(default=None)

    @property
    def nsite(self):
        return 3 * self.nwater

    @property
    def ngroup(self):
        return self.nwater

    @property
    def groups(self):
        g = np.arange(self.nwater, dtype=np.int32) * 3
        return np.stack([g, g + 3], axis=1)

    @property
    def exclusions(self):
        o = np.arange(self.nwater, dtype=np.int32) * 3
        return np.concatenate([np.stack([o, o + 1], 1), np.stack([o, o + 2], 1),
                               np.stack([o + 1, o + 2], 1)])

    @property
    def site_mask(self):
        m = np.full(self.nsite, SITE_HAS_Q, dtype=np.int32)
        m[0::3] |= SITE_HAS_LJ
        return m

    @property
    def q(self):
        """Charges in the reference's internal unit sqrt(kcal A/mol)."""
        return e_to_charge_unit(self.charges_e)

    @property
    def sigma(self):
        s = np.zeros(self.nsite)
        s[0::3] = SIGMA_O
        return s

    @property
    def epsilon(self):
        e = np.zeros(self.nsite)
        e[0::3] = EPSILON_O
        return e

    @property
    def rscreen(self):
        return np.zeros(self.nsite)

    @property
    def latv(self):
        """Lattice tensor in the reference's tensor_t layout (columns = vectors)."""
        return np.diag([self.box] * 3).T.reshape(-1).copy()


def water_box(n, seed, density=0.997, q_o=Q_O_E):
    """``n**3`` waters on a lattice with seeded random orientations."""
    nw = n ** 3
    L = box_length(nw, density)
    idx = np.arange(nw)
    ijk = np.stack([idx // (n * n), (idx // n) % n, idx % n], axis=1).astype(np.float64)
    centres = (ijk + 0.5) * (L / n)
    u = splitmix64_uniform(seed, 3 * nw).reshape(nw, 3)
    R = _rotations(u)
    half = math.radians(THETA_HOH) / 2
    body = np.array([[0.0, 0.0, 0.0],
                     [R_OH * math.sin(half), 0.0, R_OH * math.cos(half)],
                     [-R_OH * math.sin(half), 0.0, R_OH * math.cos(half)]])
    pos = centres[:, None, :] + np.einsum("nij,sj->nsi", R, body)
    masses = np.tile([MASS_O, MASS_H, MASS_H], nw)
    charges = np.tile([q_o, -q_o / 2, -q_o / 2], nw)
    return WaterBox(nwater=nw, box=L, positions=pos.reshape(-1, 3).copy(), masses=masses,
                    seed=seed, charges_e=charges)


def water_box_n(nwater, seed, density=0.997, q_o=Q_O_E):
    """``nwater`` waters (any count) at ``density``: the first ``nwater`` sites
    of a seeded permutation of the smallest cubic lattice that holds them,
    with seeded random orientations."""
    m = int(math.ceil(nwater ** (1.0 / 3.0) - 1e-9))
    L = box_length(nwater, density)
    pick = np.sort(np.argsort(splitmix64_uniform(seed ^ 0x9E3779B9, m ** 3))[:nwater])
    ijk = np.stack([pick // (m * m), (pick // m) % m, pick % m], axis=1).astype(np.float64)
    centres = (ijk + 0.5) * (L / m)
    u = splitmix64_uniform(seed, 3 * nwater).reshape(nwater, 3)
    R = _rotations(u)
    half = math.radians(THETA_HOH) / 2
    body = np.array([[0.0, 0.0, 0.0],
                     [R_OH * math.sin(half), 0.0, R_OH * math.cos(half)],
                     [-R_OH * math.sin(half), 0.0, R_OH * math.cos(half)]])
    pos = centres[:, None, :] + np.einsum("nij,sj->nsi", R, body)
    masses = np.tile([MASS_O, MASS_H, MASS_H], nwater)
    charges = np.tile([q_o, -q_o / 2, -q_o / 2], nwater)
    return WaterBox(nwater=nwater, box=L, positions=pos.reshape(-1, 3).copy(), masses=masses,
                    seed=seed, charges_e=charges)


def maxwell_boltzmann(wb, temperature, seed):
    """Seeded Maxwell-Boltzmann velocities (A/ps) with zero total momentum.

    Uses Box-Muller normals from the same SplitMix64 stream family; the mass
    unit is g/mol / 418.4 in kcal/mol ps^2/A^2 (include/units.h:166-168)."""
    n = wb.nsite
    u = splitmix64_uniform(seed ^ 0x5DEECE66D, 6 * n).reshape(2, 3 * n)
    g = np.sqrt(-2 * np.log1p(-u[0])) * np.cos(2 * np.pi * u[1])
    m = wb.masses / 418.4
    v = g.reshape(n, 3) * np.sqrt(K_to_kcal_mol(temperature) / m)[:, None]
    p = (v * m[:, None]).sum(0)
    v -= p / m.sum()
    return v

"""Physical constants and unit conversions of the reference (include/units.h).

The reference works in Angstrom, kcal/mol and picoseconds; a charge unit is
sqrt(kcal A / mol), so Coulomb's law carries no prefactor.  The constants and
the order in which they are combined are the reference's (include/units.h:23-29,
91-94, 201-204), so a charge converted here is bit-identical to one converted
by ElecLJ::types_changed (src/eleclj.cpp:445-453).
"""
import math

BOHR_RADIUS = 0.5291772108  # 1e-10 m
AVOGADRO = 6.0221415  # 1e23 / mol
HARTREE = 4.35974417  # 1e-18 J
CALORIE = 4.184  # J
BOLTZMANN = 1.3806505  # 1e-23 J/K

# e -> sqrt(kcal A / mol): include/units.h:91-94
CHARGE_UNIT = math.sqrt(BOHR_RADIUS * HARTREE * AVOGADRO * 100 / CALORIE)


def e_to_charge_unit(x):
    return x * CHARGE_UNIT


def charge_unit_to_e(x):
    return x / CHARGE_UNIT


def K_to_kcal_mol(t):
    """kT in kcal/mol for a temperature in K (include/units.h:201-204)."""
    return t * (BOLTZMANN * AVOGADRO * 1e-3 / CALORIE)

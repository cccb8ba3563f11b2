"""molmodel_b200 — msim's nonbonded force path on B200 (sm_100a).

The product is libmmnb.so (C ABI in include/mmnb.h, CUDA sources in
molmodel_b200/csrc).  This package binds it (``ElecLJ``) and generates the
seeded synthetic water boxes every workload uses (``water_box``).
"""
from .water import WaterBox, water_box, water_box_n, box_length, maxwell_boltzmann
from .potential import ElecLJ
from ._lib import MmnbError, load as load_library, LIB_PATH

__all__ = ["WaterBox", "water_box", "water_box_n", "box_length", "maxwell_boltzmann", "ElecLJ", "MmnbError",
           "load_library", "LIB_PATH"]

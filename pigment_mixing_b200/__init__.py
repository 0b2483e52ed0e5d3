"""B200-native paint-mixing MPM step (drop-in for the reference's Simulation setup/step path).

The compute path is ``libpigment_mpm.so`` (hand-written sm_100a CUDA behind the C ABI in
``include/pigment_mpm.h``); this package is its Python binding and the seeded scene builders.
"""
from .simulation import (BC_NOSLIP, BC_SLIPFREE, BC_SLIPSTICK, DPVISC, NO_PLASTICITY, PLATE_BACK, PLATE_BOTTOM,
                         PLATE_FRONT, PLATE_LEFT, PLATE_RIGHT, PLATE_TOP, RETURN_MAP_PLAIN, RETURN_MAP_SURROGATE,
                         VMVISC, Batch, Particles, Simulation)
from . import scenes

__all__ = ["Simulation", "Batch", "Particles", "scenes", "BC_NOSLIP", "BC_SLIPFREE", "BC_SLIPSTICK", "DPVISC", "VMVISC",
           "NO_PLASTICITY", "PLATE_TOP", "PLATE_BOTTOM", "PLATE_LEFT", "PLATE_RIGHT", "PLATE_FRONT", "PLATE_BACK",
           "RETURN_MAP_PLAIN", "RETURN_MAP_SURROGATE"]

"""gasatt - B200 (sm_100a) PIC-MCC electron step of the N2 X-ray gas attenuator.

The compute runs in libgasatt.so (hand-written CUDA); this package is the
Python host mirror of the reference's MATLAB interface plus the resident
simulation driver.
"""
from . import _lib
from ._lib import FAITHFUL, FP32_SPLIT, FP64, POS_IN_CYL, GasattError
from .dropin import (REBOND, Context, default_context, electricmagneticfield6,
                     electron_collision, find_CS0, free_motion, particle_density,
                     particle_density0)
from .tables import N2Tables

__all__ = ["Context", "default_context", "electricmagneticfield6", "electron_collision",
           "find_CS0", "free_motion", "particle_density", "particle_density0", "REBOND", "N2Tables",
           "GasattError", "FAITHFUL", "POS_IN_CYL", "FP64", "FP32_SPLIT"]

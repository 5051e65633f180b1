"""gasatt - B200 (sm_100a) PIC-MCC electron step of the N2 X-ray gas attenuator.

The compute runs in libgasatt.so (hand-written CUDA); this package is the
Python host mirror of the reference's MATLAB interface plus the resident
simulation driver.

The library is loaded on first use of a name that needs it (the drop-ins,
Context, the error type).  gasatt.abi (structures, codes), gasatt.workload
(presets, births, configs) and gasatt.tables (the N2 tables) load no library,
so CPU-only code - the oracle timed beside the GPU - can build the same
inputs without it.
"""
import importlib

from .abi import FAITHFUL, FP32_SPLIT, FP64, POS_IN_CYL
from .tables import N2Tables

_LAZY = {
    "_lib": ("._lib", None),
    "GasattError": ("._lib", "GasattError"),
    "REBOND": (".dropin", "REBOND"),
    "Context": (".dropin", "Context"),
    "default_context": (".dropin", "default_context"),
    "electricmagneticfield6": (".dropin", "electricmagneticfield6"),
    "electron_collision": (".dropin", "electron_collision"),
    "find_CS0": (".dropin", "find_CS0"),
    "free_motion": (".dropin", "free_motion"),
    "particle_density": (".dropin", "particle_density"),
    "particle_density0": (".dropin", "particle_density0"),
}


def __getattr__(name):
    if name not in _LAZY:
        raise AttributeError(f"module 'gasatt' has no attribute {name!r}")
    mod, attr = _LAZY[name]
    m = importlib.import_module(mod, __name__)
    return m if attr is None else getattr(m, attr)


__all__ = ["Context", "default_context", "electricmagneticfield6", "electron_collision",
           "find_CS0", "free_motion", "particle_density", "particle_density0", "REBOND", "N2Tables",
           "GasattError", "FAITHFUL", "POS_IN_CYL", "FP64", "FP32_SPLIT"]

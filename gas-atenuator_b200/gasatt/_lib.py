"""ctypes binding of libgasatt.so (the sm_100a library built in-tree).

The library is required: importing this module on a machine where it is
missing or cannot load raises ImportError - there is no fallback path.
"""
import ctypes
import os

from .abi import *  # noqa: F401,F403  (codes, flags, structures)
from .abi import OK, Diag, SimConfig, Tables, c_d, c_i, c_i64, c_p, c_u, c_u64

_HERE = os.path.dirname(os.path.abspath(__file__))
# GASATT_LIB may point at another build of the same library (e.g. a debug build)
LIB_PATH = os.environ.get("GASATT_LIB") or os.path.join(os.path.dirname(_HERE), "libgasatt.so")

_SIGS = {
    "gasatt_create": (c_i, [ctypes.POINTER(c_p), c_i, c_u64]),
    "gasatt_destroy": (c_i, [c_p]),
    "gasatt_last_error": (ctypes.c_char_p, [c_p]),
    "gasatt_set_stream": (c_i, [c_p, c_p]),
    "gasatt_synchronize": (c_i, [c_p]),
    "gasatt_kernel_launches": (c_i64, [c_p]),
    "gasatt_version": (ctypes.c_char_p, []),
    "gasatt_find_CS0": (c_i, [c_p, ctypes.POINTER(Tables), c_p, c_i64, c_p, c_p, c_p, c_u]),
    "gasatt_free_motion": (c_i, [c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_i64, c_d,
                                 c_p, c_p, c_p, c_p, c_p]),
    "gasatt_particle_density": (c_i, [c_p, c_d, c_d, c_p, c_i, c_p, c_p, c_p, c_i64, c_i,
                                      c_p, c_p, c_i64, c_d, c_p]),
    "gasatt_particle_density_noalloc": (c_i, [c_p, c_d, c_d, c_p, c_i, c_p, c_p, c_p, c_i64,
                                              c_i, c_p, c_p, c_i64, c_d, c_p]),
    "gasatt_electricmagneticfield6": (c_i, [c_p, c_p, c_p, c_i64, c_p, c_p, c_i64, c_p, c_p,
                                            c_i64, c_p, c_p, c_p, c_i, c_i, c_d, c_d, c_d,
                                            c_d, c_d, c_d, c_i, c_p,
                                            ctypes.POINTER(c_i64), ctypes.POINTER(c_i64),
                                            ctypes.POINTER(c_i64), c_u]),
    "gasatt_electron_collision": (c_i, [c_p, c_p, c_p, c_i64, c_i64, c_p, c_p, c_i64, c_i64,
                                        ctypes.POINTER(Tables), c_p, c_p, c_i, c_i, c_p, c_p,
                                        c_i64, c_d, c_p, c_d, c_d, c_p, c_p, c_p, c_d, c_p,
                                        ctypes.POINTER(c_i64), ctypes.POINTER(c_i64), c_u]),
    "gasatt_sim_default_config": (c_i, [ctypes.POINTER(SimConfig)]),
    "gasatt_sim_create": (c_i, [c_p, ctypes.POINTER(SimConfig), ctypes.POINTER(Tables),
                                ctypes.POINTER(c_p)]),
    "gasatt_sim_destroy": (c_i, [c_p]),
    "gasatt_sim_load": (c_i, [c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_i64, c_i]),
    "gasatt_sim_read": (c_i, [c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_i64,
                              ctypes.POINTER(c_i64), c_i]),
    "gasatt_sim_set_fields": (c_i, [c_p, c_p, c_p, c_p, c_i]),
    "gasatt_sim_get_fields": (c_i, [c_p, c_p, c_p, c_p, c_i]),
    "gasatt_sim_get_current": (c_i, [c_p, c_p, c_p, c_i]),
    "gasatt_sim_step": (c_i, [c_p, c_i]),
    "gasatt_sim_sort": (c_i, [c_p]),
    "gasatt_sim_diag": (c_i, [c_p, ctypes.POINTER(Diag)]),
    "gasatt_sim_run_host": (c_i, [c_p, c_p, c_p, ctypes.POINTER(c_i64), c_i64, c_i]),
    "gasatt_sim_counts": (c_i, [c_p, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64),
                                ctypes.POINTER(c_i64)]),
    "gasatt_sim_enable_timing": (c_i, [c_p, c_i]),
    "gasatt_sim_last_timing": (c_i, [c_p, ctypes.POINTER(ctypes.c_float),
                                     ctypes.POINTER(ctypes.c_float),
                                     ctypes.POINTER(ctypes.c_float)]),
    "gasatt_sim_birth_photo": (c_i, [c_p, c_i64, c_d, c_d, c_u64, c_u64]),
    "gasatt_sim_set_gas_density": (c_i, [c_p, c_p, c_i]),
    "gasatt_sim_set_gas_temperature": (c_i, [c_p, c_p, c_i]),
    "gasatt_sim_get_config": (c_i, [c_p, c_p]),
    "gasatt_rebond": (c_i, [c_p, c_p, c_i64, c_p, c_p, c_p, c_i64, c_i64, c_d, c_d, c_p]),
    "gasatt_sim_load_ions": (c_i, [c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_i64, c_i]),
    "gasatt_sim_read_ions": (c_i, [c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_i64, c_p, c_i]),
    "gasatt_batch_create": (c_i, [c_p, c_p, c_i, c_i, c_p]),
    "gasatt_batch_step": (c_i, [c_p, c_i]),
    "gasatt_batch_destroy": (c_i, [c_p]),
}

# every entry point declared in include/gasatt.h
EXPORTS = tuple(_SIGS)


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libgasatt.so not built ({LIB_PATH}); run __graft_entry__.build()")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class GasattError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"gasatt error {code}: {msg}")
        self.code = code


def check(ctx, code):
    if code != OK:
        msg = lib.gasatt_last_error(ctx).decode() if ctx else ""
        raise GasattError(code, msg)

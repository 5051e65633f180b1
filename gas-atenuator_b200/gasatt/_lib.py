"""ctypes binding of libgasatt.so (the sm_100a library built in-tree).

The library is required: importing this module on a machine where it is
missing or cannot load raises ImportError - there is no fallback path.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# GASATT_LIB may point at another build of the same library (e.g. a debug build)
LIB_PATH = os.environ.get("GASATT_LIB") or os.path.join(os.path.dirname(_HERE), "libgasatt.so")

c_p = ctypes.c_void_p
c_i64 = ctypes.c_int64
c_i = ctypes.c_int
c_d = ctypes.c_double
c_u = ctypes.c_uint
c_u64 = ctypes.c_uint64

# status codes / flags (include/gasatt.h)
OK, E_ARG, E_CUDA, E_CAPACITY, E_NAN, E_TABLES, E_STATE, E_NODEVICE = range(8)
Q_EULER_KICK = 1 << 0
Q_ATAN_PHI = 1 << 1
Q_ER_END_COPY = 1 << 2
Q_EZ_AXIS_JSIGN = 1 << 3
Q_EZ_RSHIFT = 1 << 4
Q_XS_LINEAR_E = 1 << 5
Q_COLL_LINEAR_P = 1 << 6
Q_SEC_LAB_FRAME = 1 << 7
Q_EXC_POWF = 1 << 8
Q_XS_NAN = 1 << 9
Q_PI7 = 1 << 10
Q_CDF_NEXTBIN = 1 << 11
FAITHFUL = 0x0FFF
POS_IN_CYL = 1 << 16
MCC_NDRAW = 8
FP64, FP32_SPLIT = 0, 1


class Tables(ctypes.Structure):
    _fields_ = [("t_el", c_p), ("n_el", c_i), ("t_sel", c_p), ("n_sel", c_i),
                ("t_sel_1", c_p), ("n_sel1", c_i),
                ("t_del", c_p), ("del_rows", c_i), ("del_cols", c_i),
                ("t_sdel", c_p), ("sdel_rows", c_i), ("sdel_cols", c_i),
                ("t_ion", c_p), ("n_ion", c_i), ("t_exc", c_p), ("n_exc", c_i)]


class SimConfig(ctypes.Structure):
    _fields_ = [("n_r", c_i), ("n_z", c_i), ("dr", c_d), ("dz", c_d), ("dt", c_d),
                ("fdtd_ratio", c_i), ("PHIp", c_d), ("FN", c_d), ("gas_density", c_d),
                ("gas_temperature", c_d), ("q_e", c_d), ("m_e", c_d), ("c", c_d),
                ("eps0", c_d), ("mu0", c_d), ("kb", c_d), ("m_ion", c_d),
                ("precision", c_i), ("capacity", c_i64), ("ion_capacity", c_i64),
                ("seed", c_u64), ("flags", c_u), ("sort_period", c_i), ("secondaries", c_i),
                ("table_n", c_i), ("table_emin_ev", c_d), ("table_emax_ev", c_d),
                ("ion_subcycle", c_i)]


class Diag(ctypes.Structure):
    _fields_ = [("n_alive", c_i64), ("n_total", c_i64), ("n_ionizations", c_i64),
                ("n_elastic", c_i64), ("n_excitation", c_i64), ("n_null", c_i64),
                ("n_lost_wall", c_i64), ("n_ions", c_i64), ("kinetic_ev", c_d),
                ("field_energy_j", c_d), ("steps", c_i64), ("status_flags", ctypes.c_int32),
                ("n_ion_lost_wall", c_i64), ("ion_kinetic_ev", c_d), ("net_charge_c", c_d),
                ("collision_loss_ev", c_d), ("wall_loss_ev", c_d)]


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

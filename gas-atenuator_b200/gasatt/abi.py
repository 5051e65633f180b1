"""The C ABI's plain data: status codes, quirk flags, precision forms and the
ctypes mirrors of the structures in include/gasatt.h.  Importing this module
loads no library, so workload builders and the CPU oracle can use the same
structures without the CUDA library.
"""
import ctypes

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
# SimConfig.gather (FP32 form): automatic, packed quads, direct field loads
GATHER_AUTO, GATHER_QUADS, GATHER_FIELDS = 0, 1, 2


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
                ("ion_subcycle", c_i), ("fdtd_tile_rows", c_i), ("pass_chunk", c_i),
                ("gather", c_i)]


class Diag(ctypes.Structure):
    _fields_ = [("n_alive", c_i64), ("n_total", c_i64), ("n_ionizations", c_i64),
                ("n_elastic", c_i64), ("n_excitation", c_i64), ("n_null", c_i64),
                ("n_lost_wall", c_i64), ("n_ions", c_i64), ("kinetic_ev", c_d),
                ("field_energy_j", c_d), ("steps", c_i64), ("status_flags", ctypes.c_int32),
                ("n_ion_lost_wall", c_i64), ("ion_kinetic_ev", c_d), ("net_charge_c", c_d),
                ("collision_loss_ev", c_d), ("wall_loss_ev", c_d)]



def default_config():
    """A gasatt_sim_config holding the defaults of gasatt_sim_default_config
    (the C2 grid, 1 Torr N2 at 300 K, CODATA constants, FP32 split form)."""
    c = SimConfig()
    c.n_r, c.n_z, c.dr, c.dz, c.dt = 256, 1024, 5e-6, 5e-6, 1e-14
    c.fdtd_ratio = 1
    c.PHIp = 2 * 3.141592653589793
    c.FN = 1.0
    c.gas_temperature = 300.0
    c.kb = 1.380649e-23
    c.gas_density = 133.322368 / (c.kb * 300.0)
    c.q_e, c.m_e, c.c = 1.602176634e-19, 9.1093837015e-31, 299792458.0
    c.eps0, c.mu0 = 8.8541878128e-12, 1.25663706212e-6
    c.m_ion = 28.0134 * 1.66053906660e-27
    c.precision = FP32_SPLIT
    c.capacity = 1 << 20
    c.ion_capacity = 0
    c.ion_subcycle = 50
    c.seed = 0
    c.flags = 0
    c.sort_period = 20
    c.secondaries = 1
    c.table_n, c.table_emin_ev, c.table_emax_ev = 2048, 0.1, 30000.0
    return c

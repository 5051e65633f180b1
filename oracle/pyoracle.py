"""ctypes wrapper of the CPU oracle (liboracle.so) and of the reference-kernel
drivers (oracle/_ref/libref_*.so).

TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and bench.py's CPU
baseline leg as the checker; the product never imports it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

c_p, c_i, c_i64, c_d, c_u, c_u64 = (ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
                                    ctypes.c_double, ctypes.c_uint, ctypes.c_uint64)


def _load():
    lib = ctypes.CDLL(LIB)
    lib.orc_set_threads.argtypes = [c_i]
    lib.orc_u01.restype = c_d
    lib.orc_u01.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
    lib.orc_child_id.restype = c_u64
    lib.orc_child_id.argtypes = [c_u64, c_i64]
    lib.orc_interp1.restype = c_d
    lib.orc_interp1.argtypes = [c_p, c_i, c_p, c_i, c_i, c_d]
    lib.orc_elastic_tables.restype = c_i
    lib.orc_xs_create.restype = c_p
    lib.orc_xs_create.argtypes = [c_p, c_i, c_d, c_d, c_d, c_d, c_d, c_d]
    lib.orc_xs_free.argtypes = [c_p]
    lib.orc_xs_nu_max.restype = c_d
    lib.orc_xs_nu_max.argtypes = [c_p]
    lib.orc_xs_array.restype = ctypes.POINTER(c_d)
    lib.orc_xs_array.argtypes = [c_p, c_i]
    lib.orc_field_energy.restype = c_d
    return lib


lib = _load()


def P(a):
    return a.ctypes.data_as(c_p) if a is not None else None


def philox(ctr, key):
    c = (ctypes.c_uint32 * 4)(*ctr)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    lib.orc_philox4x32_10(c, k, o)
    return list(o)


def child_id(parent, step):
    return lib.orc_child_id(parent, step)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ------------------------------------------------------------------ tables
def elastic_tables(tab):
    xI = np.zeros(64)
    yI = np.zeros(64)
    V = np.zeros(181 * 64)
    ne = lib.orc_elastic_tables(tab.ref, P(xI), P(yI), P(V))
    assert ne > 0, ne
    return xI[:ne].copy(), yI[:ne].copy(), V[:181 * ne].reshape(ne, 181).copy()


def find_cs0(tab, E_keV, flags):
    E = f64(E_keV).reshape(-1)
    out = [np.zeros_like(E) for _ in range(3)]
    lib.orc_find_cs0(tab.ref, P(E), c_i64(E.size), *map(P, out), c_u(flags))
    return out


class XS:
    """Resident-simulation tables built by the oracle."""

    def __init__(self, tab, G, emin, emax, n_gas, c, me, qe):
        self.h = lib.orc_xs_create(tab.ref, G, emin, emax, n_gas, c, me, qe)
        assert self.h
        self.G = G
        self.nu_max = lib.orc_xs_nu_max(self.h)

    def array(self, which):
        n = self.G * (181 if which == 3 else 1)
        return np.ctypeslib.as_array(lib.orc_xs_array(self.h, which), shape=(n,)).copy()

    def __del__(self):
        try:
            lib.orc_xs_free(self.h)
        except Exception:
            pass


# --------------------------------------------------------- reference kernels
def em2(x, y, z, vx, vy, vz, r, phi, vr, dele, Rp, Lp, PHIp, dt, flags):
    arrs = [x, y, z, vx, vy, vz, r, phi, vr]
    lib.orc_em2(*map(P, arrs), P(dele), c_i64(x.size), c_d(Rp), c_d(Lp), c_d(PHIp), c_d(dt),
                c_u(flags))


def em7(r, z, q, vr, vz, jr, jz, dele, nr, nz, dr, dz, FN, PHIp):
    lib.orc_em7(P(r), P(z), P(q), P(vr), P(vz), P(jr), P(jz), P(dele), c_i64(r.size), nr, nz,
                c_d(dr), c_d(dz), c_d(FN), c_d(PHIp))


def em3_1(Er, Ez, H, nr, nz, mu, dr, dz, dt):
    lib.orc_em3_1(P(Er), P(Ez), P(H), nr, nz, c_d(mu), c_d(dr), c_d(dz), c_d(dt))


def em3(Er0, Ez0, H0, Er, Ez, jr, jz, nr, nz, eps, dr, dz, dt, flags):
    lib.orc_em3(P(Er0), P(Ez0), P(H0), P(Er), P(Ez), P(jr), P(jz), nr, nz, c_d(eps), c_d(dr),
                c_d(dz), c_d(dt), c_u(flags))


def em4(x, y, z, vx, vy, vz, r, phi, vr, Er, Ez, H, q, m, E, dele, Rp, Lp, PHIp, nr, nz, mu, c,
        dr, dz, dt, flags):
    lib.orc_em4(P(x), P(y), P(z), P(vx), P(vy), P(vz), P(r), P(phi), P(vr), P(Er), P(Ez), P(H),
                P(q), P(m), P(E), P(dele), c_i64(x.size), c_d(Rp), c_d(Lp), c_d(PHIp), nr, nz,
                c_d(mu), c_d(c), c_d(dr), c_d(dz), c_d(dt), c_u(flags))


def electron_transport(x, y, z, vx, vy, vz, se, si, sx, energy, xI, yI, V, density, temperature,
                       dphi, t_exc, sum_cell0, rmax, cellnumxy, dr, dz, dt, draws, flags):
    n = x.size
    sec = np.zeros(n, np.uint8)
    out = [np.zeros(n) for _ in range(7)]
    lib.orc_electron_transport(P(x), P(y), P(z), P(vx), P(vy), P(vz), P(se), P(si), P(sx),
                               P(energy), P(xI), P(yI), P(f64(V)), c_i(xI.size), P(density),
                               P(temperature), c_i64(density.size), P(dphi),
                               P(np.asfortranarray(t_exc)), c_i(t_exc.shape[0]), P(sec),
                               *map(P, out), P(np.ascontiguousarray(sum_cell0, np.int32)),
                               c_i(rmax), c_i(cellnumxy), c_d(dr), c_d(dz), c_d(dt), c_i64(n),
                               P(draws), c_u(flags))
    return sec, out


def free_motion(vx, vy, vz, x, y, z, dt):
    n = x.size
    out = [np.zeros(n) for _ in range(5)]
    lib.orc_free_motion(*map(P, (vx, vy, vz, x, y, z)), c_i64(n), c_d(dt), *map(P, out))
    return out


def rebond(pos, r, phi, vel, Lp, PHIp, max_wraps=4096):
    """REBOND.m on (n, 3) arrays: (pos, vel, N_boundary), or N_boundary -1."""
    pos = np.asfortranarray(np.array(pos, dtype=np.float64))
    vel = np.asfortranarray(np.array(vel, dtype=np.float64))
    n = pos.shape[0]
    lib.orc_rebond.restype = c_i64
    nb = lib.orc_rebond(P(pos), c_i64(n), P(np.ascontiguousarray(r, dtype=np.float64)),
                        P(np.ascontiguousarray(phi, dtype=np.float64)), P(vel), c_i64(n),
                        c_i64(n), c_d(Lp), c_d(PHIp), c_i(max_wraps))
    return pos, vel, nb


def particle_density(dr, dz, dphi, r, phi, z, cellnumxy, sum_cell, VC, FN, ncell):
    out = np.zeros(ncell)
    lib.orc_particle_density(c_d(dr), c_d(dz), P(f64(dphi)), c_i(dphi.size), P(f64(r)),
                             P(f64(phi)), P(f64(z)), c_i64(r.size), c_i(cellnumxy),
                             P(f64(sum_cell)), P(f64(VC)), c_i64(ncell), c_d(FN), P(out))
    return out


def electricmagneticfield6(e_pos, e_vel, i1_pos, i1_vel, i2_pos, i2_vel, Er, Ez, H, delta, dt, Rp,
                           Lp, PHIp, FN, cycle_time, flags):
    """Arrays as (n,3) numpy; fields as MATLAB-shaped (n_r, n_z+1) etc.  Returns like the drop-in."""
    sp = [np.array(a, dtype=np.float64, order="F") for a in
          (e_pos, e_vel, i1_pos, i1_vel, i2_pos, i2_vel)]
    F = [np.array(a, dtype=np.float64, order="F") for a in (Er, Ez, H)]
    n_r, n_z = H.shape
    kin = np.zeros(max(len(e_pos), 1))
    outs = [c_i64() for _ in range(3)]
    lib.orc_electricmagneticfield6(P(sp[0]), P(sp[1]), c_i64(len(e_pos)), P(sp[2]), P(sp[3]),
                                   c_i64(len(i1_pos)), P(sp[4]), P(sp[5]), c_i64(len(i2_pos)),
                                   P(F[0]), P(F[1]), P(F[2]), c_i(n_r), c_i(n_z), c_d(delta),
                                   c_d(dt), c_d(Rp), c_d(Lp), c_d(PHIp), c_d(FN), c_i(cycle_time),
                                   P(kin), *[ctypes.byref(o) for o in outs], c_u(flags))
    ne, n1, n2 = (o.value for o in outs)
    return (sp[0][:ne], sp[1][:ne], sp[2][:n1], sp[3][:n1], sp[4][:n2], sp[5][:n2], F[0], F[1],
            F[2], kin[:ne])


def electron_collision(e_pos, e_vel, i1_pos, i1_vel, tab, kin, sum_cell, cellnumxy, density,
                       temperature, PHIp, phimax, dr, dz, se, si, sx, dt, draws, flags):
    n_e, n_i = len(e_pos), len(i1_pos)
    cap_e, cap_i = 2 * n_e + 1, n_i + n_e + 1
    E = np.zeros((cap_e, 3), order="F"); EV = np.zeros((cap_e, 3), order="F")
    I = np.zeros((cap_i, 3), order="F"); IV = np.zeros((cap_i, 3), order="F")
    E[:n_e] = e_pos; EV[:n_e] = e_vel; I[:n_i] = i1_pos; IV[:n_i] = i1_vel
    ne, ni = c_i64(), c_i64()
    rc = lib.orc_electron_collision(P(E), P(EV), c_i64(n_e), c_i64(cap_e), P(I), P(IV),
                                    c_i64(n_i), c_i64(cap_i), tab.ref, P(f64(kin)),
                                    P(f64(sum_cell)), c_i(len(sum_cell)), c_i(cellnumxy),
                                    P(f64(density)), P(f64(temperature)), c_i64(density.size),
                                    c_d(PHIp), P(f64(phimax)), c_d(dr), c_d(dz), P(f64(se)),
                                    P(f64(si)), P(f64(sx)), c_d(dt), P(draws), ctypes.byref(ne),
                                    ctypes.byref(ni), c_u(flags))
    assert rc == 0, rc
    return E[:ne.value], EV[:ne.value], I[:ni.value], IV[:ni.value]


# ------------------------------------------------ the MATLAB CPU path
class MatlabCpuPath:
    """electricmagneticfield3.m:111-319 (the reference's CPU push, deposit and
    field update) for electrons, one call per step (orc_mcpu_step).  Particles
    are Cartesian positions and velocities v; the grids are the reference's
    dense column-major arrays."""

    def __init__(self, nr, nz, delta, dt, PHIp=2 * np.pi, W=1.0):
        self.nr, self.nz, self.delta, self.dt, self.PHIp, self.W = nr, nz, delta, dt, PHIp, W
        self.Er = np.zeros((nr, nz + 1), order="F")
        self.Ez = np.zeros((nr + 1, nz), order="F")
        self.H = np.zeros((nr, nz), order="F")
        self.jr = np.zeros((nr, nz), order="F")
        self.jz = np.zeros((nr, nz), order="F")
        self.n = 0

    def load(self, x, y, z, vx, vy, vz):
        self.x, self.y, self.z = (np.array(a, dtype=np.float64) for a in (x, y, z))
        self.vx, self.vy, self.vz = (np.array(a, dtype=np.float64) for a in (vx, vy, vz))
        self.n = len(self.x)
        self.alive = np.ones(self.n, np.uint8)

    def step(self):
        lib.orc_mcpu_step.restype = c_i64
        return lib.orc_mcpu_step(c_i64(self.n), P(self.x), P(self.y), P(self.z), P(self.vx),
                                 P(self.vy), P(self.vz), P(self.alive), P(self.Er), P(self.Ez),
                                 P(self.H), P(self.jr), P(self.jz), c_i(self.nr), c_i(self.nz),
                                 c_d(self.delta), c_d(self.dt), c_d(self.PHIp), c_d(self.W))


# ------------------------------------------------------------ resident step
class OrcIons(ctypes.Structure):
    _fields_ = [("x", c_p), ("y", c_p), ("z", c_p), ("ux", c_p), ("uy", c_p), ("uz", c_p),
                ("id", c_p), ("alive", c_p), ("q", c_p), ("n", c_i64), ("cap", c_i64),
                ("overflow", c_i64), ("lost", c_i64)]


class Sim:
    """Oracle of the resident simulation (Cartesian u = gamma v form)."""

    def __init__(self, cfg, tab, cap):
        self.cfg = cfg                      # gasatt SimConfig (ctypes structure)
        self.tab = tab
        self.xs = XS(tab, cfg.table_n, cfg.table_emin_ev, cfg.table_emax_ev, cfg.gas_density,
                     cfg.c, cfg.m_e, cfg.q_e)
        self.gas = None
        self.gas_T = None
        self.cap = cap
        self.x = np.zeros(cap); self.y = np.zeros(cap); self.z = np.zeros(cap)
        self.ux = np.zeros(cap); self.uy = np.zeros(cap); self.uz = np.zeros(cap)
        self.id = np.zeros(cap, np.uint64)
        self.alive = np.zeros(cap, np.uint8)
        self.n = 0
        nr, nz = cfg.n_r, cfg.n_z
        self.Er = np.zeros((nr, nz + 1), order="F")
        self.Ez = np.zeros((nr + 1, nz), order="F")
        self.H = np.zeros((nr, nz), order="F")
        self.jr = np.zeros((nr, nz), order="F")
        self.jz = np.zeros((nr, nz), order="F")
        # ion, ela, exc, nul, lost, cap_overflow, then the excitation losses x 2^16 [eV]
        self._cnt = np.zeros(7, np.int64)
        self.counters = self._cnt[:6]
        self.step_index = 0
        # ions (cfg.ion_capacity > 0): store, held ion current
        ic = int(cfg.ion_capacity)
        self.ions = None
        self.jri = np.zeros((nr, nz), order="F")
        self.jzi = np.zeros((nr, nz), order="F")
        if ic > 0:
            self.ix = np.zeros(ic); self.iy = np.zeros(ic); self.iz = np.zeros(ic)
            self.iux = np.zeros(ic); self.iuy = np.zeros(ic); self.iuz = np.zeros(ic)
            self.iid = np.zeros(ic, np.uint64)
            self.ialive = np.zeros(ic, np.uint8)
            self.iq = np.zeros(ic, np.int8)
            self.ions = OrcIons(P(self.ix), P(self.iy), P(self.iz), P(self.iux), P(self.iuy),
                                P(self.iuz), P(self.iid), P(self.ialive), P(self.iq), 0, ic, 0, 0)

    def load(self, r, z, ur, ut, uz, ids):
        n = len(r)
        self.x[:n] = r; self.y[:n] = 0; self.z[:n] = z
        self.ux[:n] = ur; self.uy[:n] = ut; self.uz[:n] = uz
        self.id[:n] = ids
        self.alive[:n] = 1
        self.n = n
        if self.ions is not None:           # a new run starts without ions
            self.ions.n, self.ions.overflow, self.ions.lost = 0, 0, 0
            self.jri[:] = 0; self.jzi[:] = 0

    def set_gas_density(self, density):
        """Per-cell gas density (n_r x n_z) or None for the uniform density; the
        null-collision bound follows the largest cell."""
        cfg = self.cfg
        if density is None:
            self.gas, n_max = None, cfg.gas_density
        else:
            self.gas = np.asfortranarray(np.asarray(density, dtype=np.float64)
                                         .reshape(cfg.n_r, cfg.n_z, order="F"))
            n_max = float(self.gas.max())
        self.xs = XS(self.tab, cfg.table_n, cfg.table_emin_ev, cfg.table_emax_ev, n_max,
                     cfg.c, cfg.m_e, cfg.q_e)

    def set_gas_temperature(self, temperature):
        """Per-cell gas temperature (n_r x n_z) for the newborn ions, or None."""
        cfg = self.cfg
        self.gas_T = None if temperature is None else np.asfortranarray(
            np.asarray(temperature, dtype=np.float64).reshape(cfg.n_r, cfg.n_z, order="F"))

    def _pass(self, step, kick, mcc):
        n = c_i64(self.n)
        rc = lib.orc_sim_pass(ctypes.byref(self.cfg), c_p(self.xs.h), c_i64(step), P(self.x),
                              P(self.y), P(self.z), P(self.ux), P(self.uy), P(self.uz), P(self.id),
                              P(self.alive), ctypes.byref(n), c_i64(self.cap), P(self.Er),
                              P(self.Ez), P(self.H), P(self.jr), P(self.jz), c_i(kick), c_i(mcc),
                              None if self.gas is None else P(self.gas),
                              None if self.gas_T is None else P(self.gas_T),
                              None if self.ions is None else ctypes.byref(self.ions),
                              P(self._cnt))
        assert rc == 0
        self.n = n.value

    def prologue(self):
        self._pass(-1, 0, 0)

    def fdtd(self):
        jr, jz = self.jr, self.jz
        if self.ions is not None:
            jr, jz = np.asfortranarray(jr + self.jri), np.asfortranarray(jz + self.jzi)
        lib.orc_sim_fdtd(ctypes.byref(self.cfg), P(self.Er), P(self.Ez), P(self.H), P(jr), P(jz))

    def step(self):
        self.fdtd()
        self._pass(self.step_index, 1, 1)
        self.step_index += 1
        if self.ions is not None and self.step_index % self.cfg.ion_subcycle == 0:
            lib.orc_ion_push(ctypes.byref(self.cfg), ctypes.byref(self.ions), P(self.Er),
                             P(self.Ez), P(self.H), P(self.jri), P(self.jzi))

    @property
    def collision_loss_ev(self):
        """15.6 eV per ionization plus the excitation losses [eV]."""
        return 15.6 * float(self._cnt[0]) + float(self._cnt[6]) / 65536.0

    def load_ions(self, r, z, ur, ut, uz, ids, charge=None):
        n = len(r)
        self.ix[:n] = r; self.iy[:n] = 0; self.iz[:n] = z
        self.iux[:n] = ur; self.iuy[:n] = ut; self.iuz[:n] = uz
        self.iid[:n] = ids
        self.ialive[:n] = 1
        self.iq[:n] = 1 if charge is None else charge
        self.ions.n, self.ions.overflow, self.ions.lost = n, 0, 0
        self.jri[:] = 0; self.jzi[:] = 0

    def ion_state_rz(self):
        """(r, z, u_r, u_theta, u_z, id, alive, charge) of the ions."""
        n = self.ions.n
        x, y = self.ix[:n], self.iy[:n]
        r = np.hypot(x, y)
        ph = np.arctan2(y, x)
        cp, sp = np.cos(ph), np.sin(ph)
        ux, uy = self.iux[:n], self.iuy[:n]
        return (r, self.iz[:n].copy(), ux * cp + uy * sp, -ux * sp + uy * cp,
                self.iuz[:n].copy(), self.iid[:n].copy(), self.ialive[:n].copy(),
                self.iq[:n].copy())

    def field_energy(self):
        return lib.orc_field_energy(ctypes.byref(self.cfg), P(self.Er), P(self.Ez), P(self.H))

    def state_rz(self):
        """(r, z, u_r, u_theta, u_z, id, alive) of the first n slots."""
        n = self.n
        x, y = self.x[:n], self.y[:n]
        r = np.hypot(x, y)
        ph = np.arctan2(y, x)
        cp, sp = np.cos(ph), np.sin(ph)
        ux, uy = self.ux[:n], self.uy[:n]
        return (r, self.z[:n].copy(), ux * cp + uy * sp, -ux * sp + uy * cp, self.uz[:n].copy(),
                self.id[:n].copy(), self.alive[:n].copy())


# ------------------------------------------------- reference kernel drivers
class RefKernels:
    """The reference's own CUDA kernels (EM2/EM3/EM3_1/EM4/EM7/electron_transport)
    compiled from its sources into oracle/_ref by `make -C oracle ref`."""

    NAMES = ("EM2", "EM3", "EM3_1", "EM4", "EM7", "electron_transport")

    def __init__(self):
        self.libs = {}
        for k in self.NAMES:
            path = os.path.join(REF_DIR, f"libref_{k}.so")
            if not os.path.exists(path):
                raise FileNotFoundError(path)
            self.libs[k] = ctypes.CDLL(path)

    @staticmethod
    def available():
        return all(os.path.exists(os.path.join(REF_DIR, f"libref_{k}.so"))
                   for k in RefKernels.NAMES)

    def EM2(self, x, y, z, vx, vy, vz, r, phi, vr, dele, Rp, Lp, PHIp, dr, dz, dt):
        f = self.libs["EM2"].ref_EM2
        return f(*map(P, (x, y, z, vx, vy, vz, r, phi, vr)), P(dele), c_i(x.size), c_d(Rp),
                 c_d(Lp), c_d(PHIp), c_d(dr), c_d(dz), c_d(dt))

    def EM7(self, r, z, q, vr, vz, jr, jz, dele, nr, nz, dr, dz, FN, PHIp):
        f = self.libs["EM7"].ref_EM7
        return f(*map(P, (r, z, q, vr, vz, jr, jz)), P(dele), c_i(r.size), c_i(nr), c_i(nz),
                 c_d(dr), c_d(dz), c_d(FN), c_d(PHIp))

    def EM3_1(self, Er, Ez, H, nr, nz, mu, dr, dz, dt):
        f = self.libs["EM3_1"].ref_EM3_1
        return f(P(Er), P(Ez), P(H), c_i(nr), c_i(nz), c_d(mu), c_d(dr), c_d(dz), c_d(dt))

    def EM3(self, Er0, Ez0, H0, Er, Ez, jr, jz, nr, nz, mu, eps, dr, dz, dt):
        f = self.libs["EM3"].ref_EM3
        return f(*map(P, (Er0, Ez0, H0, Er, Ez, jr, jz)), c_i(nr), c_i(nz), c_d(mu), c_d(eps),
                 c_d(dr), c_d(dz), c_d(dt))

    def EM4(self, x, y, z, vx, vy, vz, r, phi, vr, Er, Ez, H, q, m, E, dele, Rp, Lp, PHIp, nr, nz,
            mu, c, dr, dz, dt):
        f = self.libs["EM4"].ref_EM4
        return f(*map(P, (x, y, z, vx, vy, vz, r, phi, vr, Er, Ez, H, q, m, E)), P(dele),
                 c_i(x.size), c_d(Rp), c_d(Lp), c_d(PHIp), c_i(nr), c_i(nz), c_d(mu), c_d(c),
                 c_d(dr), c_d(dz), c_d(dt))

    def electron_transport(self, x, y, z, vx, vy, vz, se, si, sx, energy, xI, yI, V, density,
                           temperature, dphi, t_exc, sum_cell0, cellnumxy, dr, dz, dt, draws):
        f = self.libs["electron_transport"].ref_electron_transport
        n = x.size
        sec = np.zeros(n, np.uint8)
        out = [np.zeros(n) for _ in range(7)]
        te = [np.ascontiguousarray(t_exc[:, k]) for k in range(5)]
        rc = f(*map(P, (x, y, z, vx, vy, vz, se, si, sx, energy, xI, yI, f64(V))), c_i(xI.size),
               P(density), P(temperature), c_i(density.size), P(dphi), c_i(dphi.size),
               *map(P, te), c_i(t_exc.shape[0]), P(sec), *map(P, out),
               P(np.ascontiguousarray(sum_cell0, np.int32)), c_i(cellnumxy), c_d(dr), c_d(dz),
               c_d(dt), c_i(n), P(draws))
        return rc, sec, out

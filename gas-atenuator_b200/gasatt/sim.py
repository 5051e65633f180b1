"""Resident PIC-MCC simulation: configuration presets, photoionization births,
and a thin wrapper over the gasatt_sim_* C ABI."""
import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._lib import Diag, SimConfig, check, lib
from .dropin import Context
from .tables import N2Tables

TORR = 133.322368           # Pa
KB = 1.380649e-23
ME = 9.1093837015e-31
QE = 1.602176634e-19
C = 299792458.0
K_SHELL_EV = 410.0          # N K-shell binding (EB_14.csv: 409.9 eV)
AUGER_EV = 360.0


def gas_density(torr, T=300.0):
    return torr * TORR / (KB * T)


def config(n_r, n_z, delta, dt, torr, *, precision=_lib.FP32_SPLIT, capacity=1 << 20, seed=0,
           sort_period=20, secondaries=1, FN=1.0, fdtd_ratio=1, flags=0, ion_capacity=0,
           ion_subcycle=50):
    cfg = SimConfig()
    check(None, lib.gasatt_sim_default_config(ctypes.byref(cfg)))
    cfg.n_r, cfg.n_z, cfg.dr, cfg.dz, cfg.dt = n_r, n_z, delta, delta, dt
    cfg.gas_density = gas_density(torr, cfg.gas_temperature)
    cfg.precision = precision
    cfg.capacity = int(capacity)
    cfg.seed = seed
    cfg.sort_period = sort_period
    cfg.secondaries = secondaries
    cfg.FN = FN
    cfg.fdtd_ratio = fdtd_ratio
    cfg.flags = flags
    cfg.ion_capacity = int(ion_capacity)
    cfg.ion_subcycle = int(ion_subcycle)
    return cfg


# The workloads (grids, pressures, photon energies, particle counts, steps, seeds).
PRESETS = {
    # 10,000 photoionizations at 8 keV -> 20,000 e-, 64 x 256 at 10 um, 1 Torr
    "c1": dict(n_r=64, n_z=256, delta=10e-6, dt=2e-14, torr=1.0, photo=10_000, e_keV=8.0,
               steps=500, seed=0),
    # 1,000,000 photoionizations at 8 keV -> 2,000,000 e-, 256 x 1024 at 5 um, 1 Torr
    "c2": dict(n_r=256, n_z=1024, delta=5e-6, dt=1e-14, torr=1.0, photo=1_000_000, e_keV=8.0,
               steps=2000, seed=1),
    # 8,000,000 photoionizations at 12 keV -> 16M e-, 1024 x 4096 at 5 um, 10 Torr, cap 64M
    "c4": dict(n_r=1024, n_z=4096, delta=5e-6, dt=1e-14, torr=10.0, photo=8_000_000, e_keV=12.0,
               steps=5000, seed=3, capacity=64 << 20),
    # 2,000,000 photoionizations at 8 keV -> 4M e-, 256 x 1024 at 10 um, 5 Torr
    "c5": dict(n_r=256, n_z=1024, delta=10e-6, dt=2e-14, torr=5.0, photo=2_000_000, e_keV=8.0,
               steps=20_000, seed=4),
}


def u_of_energy_ev(E_ev):
    eps = np.asarray(E_ev, dtype=np.float64) * QE / (ME * C * C)
    return C * np.sqrt(eps * (2 + eps))


def births(n_photo, photon_keV, Lp, *, seed, sigma_r=50e-6, id_base=0, Rp=None):
    """Photoionization births: per photon one photoelectron (photon energy minus
    the K-shell binding; direction density ~ (d . x)^2, x the polarisation)
    and one isotropic Auger electron, both at a Rayleigh(sigma_r) radius,
    uniform azimuth and uniform z.  Returns (r, z, u_r, u_theta, u_z, id) in SI,
    2 n_photo electrons (photoelectron 2k, Auger 2k+1)."""
    rng = np.random.default_rng(seed)
    n = int(n_photo)
    r = sigma_r * np.sqrt(-2.0 * np.log1p(-rng.random(n)))
    if Rp is not None:
        r = np.minimum(r, np.nextafter(Rp, 0))
    z = rng.random(n) * Lp
    phi = rng.random(n) * 2 * math.pi
    # photoelectron: cos(angle to x) = mu, p(mu) ~ mu^2  ->  mu = cbrt(2U - 1)
    mu = np.cbrt(2 * rng.random(n) - 1)
    psi = rng.random(n) * 2 * math.pi
    s = np.sqrt(np.maximum(0.0, 1 - mu * mu))
    d_pe = np.stack([mu, s * np.cos(psi), s * np.sin(psi)])
    # Auger: isotropic
    ct = 2 * rng.random(n) - 1
    pa = rng.random(n) * 2 * math.pi
    st = np.sqrt(np.maximum(0.0, 1 - ct * ct))
    d_au = np.stack([st * np.cos(pa), st * np.sin(pa), ct])
    u_pe = u_of_energy_ev(photon_keV * 1000 - K_SHELL_EV)
    u_au = u_of_energy_ev(AUGER_EV)
    cp, sp = np.cos(phi), np.sin(phi)

    def local(d, umag):
        return (umag * (d[0] * cp + d[1] * sp), umag * (-d[0] * sp + d[1] * cp), umag * d[2])

    pe = local(d_pe, u_pe)
    au = local(d_au, u_au)
    out_r = np.empty(2 * n); out_z = np.empty(2 * n)
    ur = np.empty(2 * n); ut = np.empty(2 * n); uz = np.empty(2 * n)
    out_r[0::2] = r; out_r[1::2] = r
    out_z[0::2] = z; out_z[1::2] = z
    ur[0::2], ut[0::2], uz[0::2] = pe
    ur[1::2], ut[1::2], uz[1::2] = au
    ids = np.arange(2 * n, dtype=np.uint64) + np.uint64(id_base)
    return out_r, out_z, ur, ut, uz, ids


class Sim:
    """One gas-cell instance resident on a GPU."""

    def __init__(self, cfg, ctx=None, tables=None, device=0):
        self.ctx = ctx or Context(device)
        self.cfg = cfg
        self.tables = tables or N2Tables()
        self.h = ctypes.c_void_p()
        check(self.ctx.handle, lib.gasatt_sim_create(self.ctx.handle, ctypes.byref(cfg),
                                                     self.tables.ref, ctypes.byref(self.h)))
        self.device = device

    def bind_stream(self, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        check(self.ctx.handle, lib.gasatt_set_stream(self.ctx.handle, ctypes.c_void_p(s.cuda_stream)))

    def load(self, r, z, ur, ut, uz, ids):
        """Load electrons (numpy arrays on the host or CUDA tensors on this device)."""
        if torch.is_tensor(r) and r.is_cuda:
            arrs = [a.to(torch.float64).contiguous() for a in (r, z, ur, ut, uz)]
            idt = ids.contiguous()
            ptrs = [ctypes.c_void_p(a.data_ptr()) for a in arrs] + [ctypes.c_void_p(idt.data_ptr())]
            check(self.ctx.handle, lib.gasatt_sim_load(self.h, *ptrs, arrs[0].numel(), 1))
            return
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (r, z, ur, ut, uz)]
        idn = np.ascontiguousarray(ids, dtype=np.uint64)
        ptrs = [a.ctypes.data_as(ctypes.c_void_p) for a in arrs] + [idn.ctypes.data_as(ctypes.c_void_p)]
        check(self.ctx.handle, lib.gasatt_sim_load(self.h, *ptrs, len(arrs[0]), 0))

    def birth_photo(self, n_photo, photon_keV, *, seed, sigma_r=50e-6, id_base=0):
        """Replace the particles by 2 n_photo photoionization births drawn on the
        GPU (the laws of births(); Philox draws keyed on seed and photon)."""
        check(self.ctx.handle, lib.gasatt_sim_birth_photo(self.h, int(n_photo), float(photon_keV),
                                                          float(sigma_r), int(seed), int(id_base)))

    def step(self, n=1):
        check(self.ctx.handle, lib.gasatt_sim_step(self.h, int(n)))

    def sort(self):
        check(self.ctx.handle, lib.gasatt_sim_sort(self.h))

    def synchronize(self):
        check(self.ctx.handle, lib.gasatt_synchronize(self.ctx.handle))

    def read(self):
        n = ctypes.c_int64()
        lib.gasatt_sim_read(self.h, None, None, None, None, None, None, 0, ctypes.byref(n), 0)
        cap = max(n.value, 1)
        out = [np.zeros(cap) for _ in range(5)]
        ids = np.zeros(cap, np.uint64)
        ptrs = [a.ctypes.data_as(ctypes.c_void_p) for a in out] + [ids.ctypes.data_as(ctypes.c_void_p)]
        check(self.ctx.handle, lib.gasatt_sim_read(self.h, *ptrs, cap, ctypes.byref(n), 0))
        k = n.value
        return dict(r=out[0][:k], z=out[1][:k], ur=out[2][:k], ut=out[3][:k], uz=out[4][:k],
                    id=ids[:k])

    def load_ions(self, r, z, ur, ut, uz, ids, charge=None):
        """Replace the ions (host arrays; charge numbers 1 or 2, default all 1).
        Needs cfg.ion_capacity > 0; call after load / birth_photo."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (r, z, ur, ut, uz)]
        idn = np.ascontiguousarray(ids, dtype=np.uint64)
        q = None if charge is None else np.ascontiguousarray(charge, dtype=np.int8)
        ptrs = [a.ctypes.data_as(ctypes.c_void_p) for a in arrs] + [idn.ctypes.data_as(ctypes.c_void_p)]
        qp = None if q is None else q.ctypes.data_as(ctypes.c_void_p)
        check(self.ctx.handle, lib.gasatt_sim_load_ions(self.h, *ptrs, qp, len(arrs[0]), 0))

    def read_ions(self):
        """Ion slots in use as a dict like read(), plus the charge numbers
        (dead ions have r = -1)."""
        n = ctypes.c_int64()
        # a first call with no room only reports the count
        lib.gasatt_sim_read_ions(self.h, None, None, None, None, None, None, None, 0,
                                 ctypes.byref(n), 0)
        cap = max(n.value, 1)
        out = [np.zeros(cap) for _ in range(5)]
        ids = np.zeros(cap, np.uint64)
        q = np.zeros(cap, np.int8)
        ptrs = [a.ctypes.data_as(ctypes.c_void_p) for a in out] + [
            ids.ctypes.data_as(ctypes.c_void_p), q.ctypes.data_as(ctypes.c_void_p)]
        if n.value:
            check(self.ctx.handle, lib.gasatt_sim_read_ions(self.h, *ptrs, cap, ctypes.byref(n), 0))
        k = n.value
        return dict(r=out[0][:k], z=out[1][:k], ur=out[2][:k], ut=out[3][:k], uz=out[4][:k],
                    id=ids[:k], charge=q[:k])

    def fields(self):
        nr, nz = self.cfg.n_r, self.cfg.n_z
        Er = np.zeros((nr, nz + 1), order="F")
        Ez = np.zeros((nr + 1, nz), order="F")
        H = np.zeros((nr, nz), order="F")
        check(self.ctx.handle, lib.gasatt_sim_get_fields(self.h, *[a.ctypes.data_as(ctypes.c_void_p)
                                                                   for a in (Er, Ez, H)], 0))
        return Er, Ez, H

    def set_fields(self, Er, Ez, H):
        arrs = [np.asfortranarray(a, dtype=np.float64) for a in (Er, Ez, H)]
        check(self.ctx.handle, lib.gasatt_sim_set_fields(self.h, *[a.ctypes.data_as(ctypes.c_void_p)
                                                                   for a in arrs], 0))

    def set_gas_density(self, density):
        """Per-cell N2 density [m^-3] of shape (n_r, n_z) for the collisions, or
        None to go back to the uniform cfg.gas_density.  Step graphs are rebuilt;
        a Batch must be created after this call."""
        if density is None:
            check(self.ctx.handle, lib.gasatt_sim_set_gas_density(self.h, None, 0))
            return
        a = np.asfortranarray(density, dtype=np.float64)
        if a.shape != (self.cfg.n_r, self.cfg.n_z):
            raise ValueError(f"gas density must have shape ({self.cfg.n_r}, {self.cfg.n_z})")
        check(self.ctx.handle, lib.gasatt_sim_set_gas_density(self.h, a.ctypes.data_as(ctypes.c_void_p), 0))

    def set_gas_temperature(self, temperature):
        """Per-cell gas temperature [K] of shape (n_r, n_z) for the newborn
        ions' Maxwellian, or None for the uniform cfg.gas_temperature."""
        if temperature is None:
            check(self.ctx.handle, lib.gasatt_sim_set_gas_temperature(self.h, None, 0))
            return
        a = np.asfortranarray(temperature, dtype=np.float64)
        if a.shape != (self.cfg.n_r, self.cfg.n_z):
            raise ValueError(f"gas temperature must have shape ({self.cfg.n_r}, {self.cfg.n_z})")
        check(self.ctx.handle, lib.gasatt_sim_set_gas_temperature(self.h, a.ctypes.data_as(ctypes.c_void_p), 0))

    def current(self):
        nr, nz = self.cfg.n_r, self.cfg.n_z
        jr = np.zeros((nr, nz), order="F")
        jz = np.zeros((nr, nz), order="F")
        check(self.ctx.handle, lib.gasatt_sim_get_current(self.h, jr.ctypes.data_as(ctypes.c_void_p),
                                                          jz.ctypes.data_as(ctypes.c_void_p), 0))
        return jr, jz

    def diag(self):
        d = Diag()
        check(self.ctx.handle, lib.gasatt_sim_diag(self.h, ctypes.byref(d)))
        return {k: getattr(d, k) for k, _ in Diag._fields_}

    def close(self):
        if self.h:
            lib.gasatt_sim_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Independent gas-cell instances (Sim objects on one context) advanced
    together: one graph launch per step runs all their step graphs side by
    side.  The instances share `sort_period`; each stays observable on its
    own (read, diag, fields)."""

    def __init__(self, sims, sort_period=20):
        self.sims = list(sims)
        ctx = self.sims[0].ctx
        if any(s.ctx is not ctx for s in self.sims):
            raise ValueError("all instances of a batch must share one Context")
        self.ctx = ctx
        arr = (ctypes.c_void_p * len(self.sims))(*[s.h.value for s in self.sims])
        self.h = ctypes.c_void_p()
        check(ctx.handle, lib.gasatt_batch_create(ctx.handle, arr, len(self.sims), int(sort_period),
                                                  ctypes.byref(self.h)))

    def step(self, n=1):
        check(self.ctx.handle, lib.gasatt_batch_step(self.h, int(n)))

    def close(self):
        if self.h:
            lib.gasatt_batch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

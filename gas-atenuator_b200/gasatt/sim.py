"""Resident PIC-MCC simulation: a thin wrapper over the gasatt_sim_* C ABI
(the workload builders - presets, births, config - live in gasatt.workload
and are re-exported here)."""
import ctypes

import numpy as np
import torch

from ._lib import Diag, check, lib
from .dropin import Context
from .tables import N2Tables
from .workload import (AUGER_EV, C, K_SHELL_EV, KB, ME, PRESETS, QE, TORR,  # noqa: F401
                       births, config, gas_density, u_of_energy_ev)


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

"""MATLAB-signature drop-ins over the C ABI.

Each function keeps the name, argument order and meaning of the reference
MATLAB function it replaces and runs on CUDA tensors through libgasatt.so:

    find_CS0                find_CS0.m:1
    free_motion             free_motion.m:1
    particle_density        particle_density.m:1   (10-argument form)
    particle_density0       particle_density0.m:1  (8-argument form)
    electricmagneticfield6  electricmagneticfield6.m:1
    electron_collision      electron_collision.m:1

Arrays that MATLAB holds as n x 3 matrices are (n, 3) float64 tensors here;
they are passed to the library in MATLAB's column-major layout.  Errors from
the library raise GasattError (MATLAB's mexErrMsgIdAndTxt in a MEX gateway).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import FAITHFUL, POS_IN_CYL, check, lib
from .tables import N2Tables

_ctx_cache = {}


class Context:
    """A gasatt context on one device (stream, seed, Philox call counter)."""

    def __init__(self, device=0, seed=0):
        self.handle = ctypes.c_void_p()
        rc = lib.gasatt_create(ctypes.byref(self.handle), device, seed)
        if rc != _lib.OK:
            raise _lib.GasattError(rc, "gasatt_create failed (no CUDA device?)")
        self.device = device

    def bind_stream(self):
        s = torch.cuda.current_stream(self.device).cuda_stream
        check(self.handle, lib.gasatt_set_stream(self.handle, ctypes.c_void_p(s)))

    @property
    def launches(self):
        return lib.gasatt_kernel_launches(self.handle)

    def close(self):
        if self.handle:
            lib.gasatt_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_context(device=0):
    if device not in _ctx_cache:
        _ctx_cache[device] = Context(device)
    ctx = _ctx_cache[device]
    ctx.bind_stream()
    return ctx


def _dev(t, device):
    t = torch.as_tensor(t, dtype=torch.float64)
    return t.to(device=f"cuda:{device}")


def _col(t, device=0):
    """(n, k) tensor -> column-major (k, n) contiguous storage, returned as the storage tensor."""
    t = _dev(t, device)
    if t.dim() == 1:
        t = t[:, None]
    return t.t().contiguous()


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _tables(**override):
    base = N2Tables()
    if override:
        return N2Tables(**{k: np.asarray(v.cpu() if torch.is_tensor(v) else v, dtype=np.float64)
                           for k, v in override.items()})
    return base


def find_CS0(t_el, t_sel, t_ion, t_exc, E_PE, *, flags=FAITHFUL, device=0):
    """[sigma_el, sigma_ion, sigma_exc] = find_CS0(t_el, t_sel, t_ion, t_exc, E_PE) (E_PE in keV)."""
    ctx = default_context(device)
    tab = _tables(t_el=t_el, t_sel=t_sel, t_ion=t_ion, t_exc=t_exc)
    E = _dev(E_PE, device).reshape(-1).contiguous()
    n = E.numel()
    se, si, sx = (torch.empty(n, dtype=torch.float64, device=E.device) for _ in range(3))
    check(ctx.handle, lib.gasatt_find_CS0(ctx.handle, tab.ref, _p(E), n, _p(se), _p(si), _p(sx),
                                          flags))
    return se, si, sx


def free_motion(vx, vy, vz, x, y, z, dt, *, device=0):
    """[xn, yn, zn, rn, phin] = free_motion(vx, vy, vz, x, y, z, dt)."""
    ctx = default_context(device)
    ins = [_dev(a, device).reshape(-1).contiguous() for a in (vx, vy, vz, x, y, z)]
    n = ins[0].numel()
    outs = [torch.empty(n, dtype=torch.float64, device=ins[0].device) for _ in range(5)]
    check(ctx.handle, lib.gasatt_free_motion(ctx.handle, *map(_p, ins), n, float(dt), *map(_p, outs)))
    return tuple(outs)


def REBOND(particle_position, particle_r, particle_phi, particle_velocity, Lp, PHIp, *, device=0):
    """[particle_position, particle_velocity, N_boundary] = REBOND(particle_position,
    particle_r, particle_phi, particle_velocity, Lp, PHIp): azimuths wrapped
    into the wedge [0, PHIp] (velocity turned with them), z reflected at Lp and 0."""
    ctx = default_context(device)
    pos, vel = _col(particle_position, device), _col(particle_velocity, device)
    r = _dev(particle_r, device).reshape(-1).contiguous()
    phi = _dev(particle_phi, device).reshape(-1).contiguous()
    n = pos.shape[1]
    nb = ctypes.c_int64()
    check(ctx.handle, lib.gasatt_rebond(ctx.handle, _p(pos), n, _p(r), _p(phi), _p(vel), n, n,
                                        float(Lp), float(PHIp), ctypes.byref(nb)))
    return pos.t(), vel.t(), nb.value


def particle_density(dr, dz, dphi, r, phi, z, cellnumxy, sum_cell, VC, FN, *, ncell=None, device=0):
    """density = particle_density(dr, dz, dphi, r, phi, z, cellnumxy, sum_cell, VC, FN).

    The result covers ncell = cellnumxy * zmax cells (zmax from the z extent
    when not given); VC is the per-cell volume of one z layer."""
    ctx = default_context(device)
    dphi = _dev(dphi, device).reshape(-1).contiguous()
    sum_cell = _dev(sum_cell, device).reshape(-1).contiguous()
    VC = _dev(VC, device).reshape(-1).contiguous()
    r, phi, z = (_dev(a, device).reshape(-1).contiguous() for a in (r, phi, z))
    if ncell is None:
        zmax = int(torch.round(z.max() / dz + 0.5).item()) if z.numel() else 1
        ncell = cellnumxy * max(zmax, 1)
    out = torch.empty(ncell, dtype=torch.float64, device=r.device)
    check(ctx.handle, lib.gasatt_particle_density(ctx.handle, float(dr), float(dz), _p(dphi),
                                                  dphi.numel(), _p(r), _p(phi), _p(z), r.numel(),
                                                  int(cellnumxy), _p(sum_cell), _p(VC), ncell,
                                                  float(FN), _p(out)))
    return out


def particle_density0(dr, dz, dphi, position, cellnumxy, sum_cell, VC, FN, *, ncell=None, device=0):
    """particle_density0.m: position columns are (r, z, phi)."""
    position = _dev(position, device)
    return particle_density(dr, dz, dphi, position[:, 0], position[:, 2], position[:, 1],
                            cellnumxy, sum_cell, VC, FN, ncell=ncell, device=device)


def electricmagneticfield6(electron_position0, electron_velocity, ion1_position0, ion1_velocity,
                           ion2_position0, ion2_velocity, Er, Ez, Hphi, delta, dt, Rp, Lp, PHIp,
                           FN, cycle_time_for_electromagneticfield, *, flags=FAITHFUL | POS_IN_CYL,
                           device=0):
    """[e_pos, e_vel, i1_pos, i1_vel, i2_pos, i2_vel, Er, Ez, Hphi, electron_kinetic] =
    electricmagneticfield6(...).  Positions in: (r, phi, z) when POS_IN_CYL (the
    reference's convention), out: (x, y, z); deleted particles removed."""
    ctx = default_context(device)
    sp = [(_col(p, device), _col(v, device)) for p, v in
          ((electron_position0, electron_velocity), (ion1_position0, ion1_velocity),
           (ion2_position0, ion2_velocity))]
    ns = [p.shape[1] for p, _ in sp]
    n_r = int(round(Rp / delta))
    n_z = int(round(Lp / delta))
    Er = _dev(Er, device).t().contiguous()       # (n_z+1, n_r) storage == MATLAB n_r x (n_z+1)
    Ez = _dev(Ez, device).t().contiguous()
    Hphi = _dev(Hphi, device).t().contiguous()
    kin = torch.zeros(max(ns[0], 1), dtype=torch.float64, device=Er.device)
    outs = [ctypes.c_int64() for _ in range(3)]
    check(ctx.handle, lib.gasatt_electricmagneticfield6(
        ctx.handle, _p(sp[0][0]), _p(sp[0][1]), ns[0], _p(sp[1][0]), _p(sp[1][1]), ns[1],
        _p(sp[2][0]), _p(sp[2][1]), ns[2], _p(Er), _p(Ez), _p(Hphi), n_r, n_z, float(delta),
        float(dt), float(Rp), float(Lp), float(PHIp), float(FN),
        int(cycle_time_for_electromagneticfield), _p(kin), *[ctypes.byref(o) for o in outs], flags))
    res = []
    for (p, v), o in zip(sp, outs):
        k = o.value
        res += [p[:, :k].t(), v[:, :k].t()]
    return (*res, Er.t(), Ez.t(), Hphi.t(), kin[:outs[0].value])


def electron_collision(electron_position, electron_velocity, ion1_position, ion1_velocity, t_el,
                       t_sel_1, t_del, t_sdel, t_exc, electron_kinetic, sum_cell, cellnumxy,
                       particle_num_density_in_every_cell, temperature_in_every_cell, PHIp,
                       phimax, dr, dz, sig_elastic, sig_ionization, sig_excitation, dt_transport,
                       *, draws=None, flags=FAITHFUL, device=0):
    """[e_pos, e_vel, ion1_pos, ion1_vel] = electron_collision(...).  Secondaries are
    appended to the electrons and N2+ ions to ion1 (electron_collision.m:63-75).
    draws: optional (n, 8) injected random draws (see GASATT_MCC_NDRAW)."""
    ctx = default_context(device)
    tab = _tables(t_el=t_el, t_sel_1=t_sel_1, t_del=t_del, t_sdel=t_sdel, t_exc=t_exc)
    ep = _dev(electron_position, device)
    n_e = ep.shape[0]
    ip = _dev(ion1_position, device).reshape(-1, 3)
    n_i = ip.shape[0]
    cap_e, cap_i = 2 * n_e + 1, n_i + n_e + 1
    E = torch.zeros(3, cap_e, dtype=torch.float64, device=ep.device)
    EV = torch.zeros_like(E)
    I = torch.zeros(3, cap_i, dtype=torch.float64, device=ep.device)
    IV = torch.zeros_like(I)
    E[:, :n_e] = ep.t()
    EV[:, :n_e] = _dev(electron_velocity, device).t()
    I[:, :n_i] = ip.t()
    IV[:, :n_i] = _dev(ion1_velocity, device).reshape(-1, 3).t()
    kin = _dev(electron_kinetic, device).reshape(-1).contiguous()
    sig = [_dev(s, device).reshape(-1).contiguous() for s in (sig_elastic, sig_ionization, sig_excitation)]
    den = _dev(particle_num_density_in_every_cell, device).t().reshape(-1).contiguous() \
        if torch.as_tensor(particle_num_density_in_every_cell).dim() == 2 else \
        _dev(particle_num_density_in_every_cell, device).reshape(-1).contiguous()
    tem = _dev(temperature_in_every_cell, device).t().reshape(-1).contiguous() \
        if torch.as_tensor(temperature_in_every_cell).dim() == 2 else \
        _dev(temperature_in_every_cell, device).reshape(-1).contiguous()
    sc = np.ascontiguousarray(np.asarray(sum_cell, dtype=np.float64).reshape(-1))
    pm = np.ascontiguousarray(np.asarray(phimax, dtype=np.float64).reshape(-1))
    dr_ = _dev(draws, device).reshape(-1, _lib.MCC_NDRAW).contiguous() if draws is not None else None
    ne_out, ni_out = ctypes.c_int64(), ctypes.c_int64()
    check(ctx.handle, lib.gasatt_electron_collision(
        ctx.handle, _p(E), _p(EV), n_e, cap_e, _p(I), _p(IV), n_i, cap_i, tab.ref, _p(kin),
        sc.ctypes.data_as(ctypes.c_void_p), sc.size, int(cellnumxy), _p(den), _p(tem), den.numel(),
        float(PHIp), pm.ctypes.data_as(ctypes.c_void_p), float(dr), float(dz), _p(sig[0]),
        _p(sig[1]), _p(sig[2]), float(dt_transport), _p(dr_), ctypes.byref(ne_out),
        ctypes.byref(ni_out), flags))
    a, b = ne_out.value, ni_out.value
    return E[:, :a].t(), EV[:, :a].t(), I[:, :b].t(), IV[:, :b].t()

"""The workloads of the resident simulation in plain numpy: physical
constants, gas density from pressure, the preset gas cells, the
photoionization birth sampler and a gasatt_sim_config builder.  Nothing here
loads the CUDA library, so the same inputs feed both the GPU runs and the CPU
oracle timed beside them."""
import math

import numpy as np

from . import abi

TORR = 133.322368           # Pa
KB = 1.380649e-23
ME = 9.1093837015e-31
QE = 1.602176634e-19
C = 299792458.0
K_SHELL_EV = 410.0          # N K-shell binding (EB_14.csv: 409.9 eV)
AUGER_EV = 360.0


def gas_density(torr, T=300.0):
    return torr * TORR / (KB * T)


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


def config(n_r, n_z, delta, dt, torr, *, precision=abi.FP32_SPLIT, capacity=1 << 20, seed=0,
           sort_period=20, secondaries=1, FN=1.0, fdtd_ratio=1, flags=0, ion_capacity=0,
           ion_subcycle=50):
    """A gasatt_sim_config for an n_r x n_z grid of square cells of side
    `delta`, particle step dt and N2 at `torr` (300 K); the rest from
    gasatt_sim_default_config."""
    cfg = abi.default_config()
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

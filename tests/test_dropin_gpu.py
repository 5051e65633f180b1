"""CUDA drop-ins (through the C ABI) against the CPU oracle on the same inputs."""
import math

import numpy as np
import pytest
import torch

import gasatt
import pyoracle as O
from _cases import cell_structure, close, draws, grid_fields, kinetic_kev, wedge_particles
from gasatt import _lib

pytestmark = pytest.mark.gpu

MODES = [("faithful", _lib.FAITHFUL), ("corrected", 0)]


def np_(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("name,flags", MODES)
def test_find_cs0(tables, name, flags):
    E = np.concatenate([np.exp(np.linspace(np.log(1e-4), np.log(30.0), 5000)),
                        tables["t_el"][0], tables["t_ion"][:, 0] / 1000, [0.05, 0.0156, 0.02]])
    got = gasatt.find_CS0(tables["t_el"], tables["t_sel"], tables["t_ion"], tables["t_exc"],
                          torch.tensor(E), flags=flags)
    want = O.find_cs0(tables, E, flags)
    for g, w, k in zip(got, want, ("el", "ion", "exc")):
        g = np_(g)
        np.testing.assert_array_equal(np.isnan(g), np.isnan(w), err_msg=k)
        m = ~np.isnan(w)
        close(g[m], w[m], 1e-13, k)


def test_free_motion():
    rng = np.random.default_rng(4)
    a = [rng.normal(size=10000) * s for s in (1e7, 1e7, 1e7, 1e-3, 1e-3, 1e-2)]
    got = gasatt.free_motion(*[torch.tensor(x) for x in a], 1e-12)
    want = O.free_motion(*a, 1e-12)
    for g, w in zip(got, want):
        close(np_(g), w, 1e-15)


def test_particle_density():
    PHIp, Rp, rmax, delta = 0.1, 1e-2, 25, 4e-4
    phimax, sum_cell, cellnumxy = cell_structure(PHIp, Rp, rmax, delta)
    zmax, dz = 6, 1e-2
    dphi = PHIp / phimax
    VC = np.concatenate([[0.5 * ((i * delta)**2 - ((i - 1) * delta)**2) * dphi[i - 1] * dz]
                         * int(phimax[i - 1]) for i in range(1, rmax + 1)])
    rng = np.random.default_rng(9)
    n = 200000
    r = rng.uniform(0, Rp * 1.02, n); phi = rng.uniform(-0.01, PHIp, n); z = rng.uniform(0, zmax * dz, n)
    got = gasatt.particle_density(delta, dz, dphi, torch.tensor(r), torch.tensor(phi), torch.tensor(z),
                                  cellnumxy, sum_cell, VC, 3.0, ncell=cellnumxy * zmax)
    want = O.particle_density(delta, dz, dphi, r, phi, z, cellnumxy, sum_cell, VC, 3.0, cellnumxy * zmax)
    np.testing.assert_array_equal(np_(got), want)


def emf6_inputs(seed, n_e=3000, n_i1=300, n_i2=300, nr=16, nz=40, d=1e-4, PHIp=0.1):
    rng = np.random.default_rng(seed)
    Er, Ez, H = grid_fields(nr, nz, rng, E0=3e5, H0=300.0)
    e = wedge_particles(n_e, nr * d, nz * d, PHIp, rng, vmag=4e7)
    i1 = wedge_particles(n_i1, nr * d, nz * d, PHIp, rng, vmag=2e3)
    i2 = wedge_particles(n_i2, nr * d, nz * d, PHIp, rng, vmag=2e3)
    e[0][:40, 0] = nr * d * 0.995                          # some electrons leave through the wall
    return dict(e=e, i1=i1, i2=i2, Er=Er, Ez=Ez, H=H, d=d, nr=nr, nz=nz, PHIp=PHIp)


@pytest.mark.parametrize("name,flags", MODES)
def test_electricmagneticfield6(name, flags):
    cs = emf6_inputs(5 if flags else 6)
    d, nr, nz, PHIp = cs["d"], cs["nr"], cs["nz"], cs["PHIp"]
    args = (cs["e"][0], cs["e"][1], cs["i1"][0], cs["i1"][1], cs["i2"][0], cs["i2"][1],
            cs["Er"], cs["Ez"], cs["H"], d, 1e-13, nr * d, nz * d, PHIp, 1e4, 20)
    got = gasatt.electricmagneticfield6(*[torch.tensor(a) if isinstance(a, np.ndarray) else a for a in args],
                                        flags=flags | _lib.POS_IN_CYL)
    want = O.electricmagneticfield6(*args, flags | _lib.POS_IN_CYL)
    names = ["e_pos", "e_vel", "i1_pos", "i1_vel", "i2_pos", "i2_vel", "Er", "Ez", "Hphi", "kin"]
    assert len(np_(got[0])) == len(want[0]) < 3000       # wall losses happened, same survivors
    for g, w, k in zip(got, want, names):
        close(np_(g), w, 1e-12, k)


def collision_inputs(seed, n=5000, PHIp=0.1, Rp=1e-2, rmax=20, zmax=5, Lp=0.05):
    rng = np.random.default_rng(seed)
    delta = Rp / rmax
    phimax, sum_cell, cellnumxy = cell_structure(PHIp, Rp, rmax, delta)
    pos, _ = wedge_particles(n, Rp, Lp, PHIp, rng, cyl=False)
    E_eV = np.exp(rng.uniform(np.log(3.0), np.log(8000.0), n))
    m, e, c = 9.109e-31, 1.6022e-19, 3e8
    g = 1 + E_eV * e / (m * c * c)
    d = rng.normal(size=(n, 3)); d /= np.linalg.norm(d, axis=1)[:, None]
    v = d * (c * np.sqrt(1 - 1 / g**2))[:, None]
    ncell = cellnumxy * zmax
    return dict(pos=pos, vel=v, kin=kinetic_kev(v), sum_cell=sum_cell, cellnumxy=cellnumxy,
                density=np.full(ncell, 3.2e22) * rng.uniform(0.5, 1.5, ncell),
                temperature=300 * rng.uniform(0.8, 1.2, ncell), PHIp=PHIp, phimax=phimax,
                dr=delta, dz=Lp / zmax, ion_pos=rng.uniform(0, 1e-3, (7, 3)),
                ion_vel=rng.normal(size=(7, 3)), draws=draws(n, rng))


@pytest.mark.parametrize("name,flags", MODES)
def test_electron_collision(tables, name, flags):
    cs = collision_inputs(7 if flags else 8)
    se, si, sx = O.find_cs0(tables, cs["kin"], _lib.FAITHFUL)
    se, si, sx = (np.nan_to_num(a, nan=0.0) for a in (se, si, sx))
    common = (tables["t_el"], tables["t_sel_1"], tables["t_del"], tables["t_sdel"], tables["t_exc"])
    got = gasatt.electron_collision(torch.tensor(cs["pos"]), torch.tensor(cs["vel"]),
                                    torch.tensor(cs["ion_pos"]), torch.tensor(cs["ion_vel"]), *common,
                                    torch.tensor(cs["kin"]), cs["sum_cell"], cs["cellnumxy"],
                                    torch.tensor(cs["density"]), torch.tensor(cs["temperature"]),
                                    cs["PHIp"], cs["phimax"], cs["dr"], cs["dz"], torch.tensor(se),
                                    torch.tensor(si), torch.tensor(sx), 2e-10,
                                    draws=torch.tensor(cs["draws"]), flags=flags)
    want = O.electron_collision(cs["pos"], cs["vel"], cs["ion_pos"], cs["ion_vel"], tables,
                                cs["kin"], cs["sum_cell"], cs["cellnumxy"], cs["density"],
                                cs["temperature"], cs["PHIp"], cs["phimax"], cs["dr"], cs["dz"],
                                se, si, sx, 2e-10, cs["draws"], flags)
    assert len(np_(got[0])) == len(want[0]) > 5000 + 100     # secondaries appended
    assert len(np_(got[2])) == len(want[2]) == len(want[0]) - 5000 + 7
    rtol = 1e-6 if flags & _lib.Q_EXC_POWF else 1e-12
    for g, w, k in zip(got, want, ("e_pos", "e_vel", "i_pos", "i_vel")):
        close(np_(g), w, rtol, k)


def test_electron_collision_philox_reproducible(tables):
    """Without injected draws the stream is Philox(seed, particle, call): two
    contexts with the same seed give identical results."""
    cs = collision_inputs(10, n=2000)
    se, si, sx = (np.nan_to_num(a, nan=0.0) for a in O.find_cs0(tables, cs["kin"], _lib.FAITHFUL))
    outs = []
    for _ in range(2):
        gasatt.dropin._ctx_cache.clear()
        ctx = gasatt.default_context(0)
        outs.append(gasatt.electron_collision(
            torch.tensor(cs["pos"]), torch.tensor(cs["vel"]), torch.zeros(0, 3), torch.zeros(0, 3),
            tables["t_el"], tables["t_sel_1"], tables["t_del"], tables["t_sdel"], tables["t_exc"],
            torch.tensor(cs["kin"]), cs["sum_cell"], cs["cellnumxy"], torch.tensor(cs["density"]),
            torch.tensor(cs["temperature"]), cs["PHIp"], cs["phimax"], cs["dr"], cs["dz"],
            torch.tensor(se), torch.tensor(si), torch.tensor(sx), 2e-10))
    for a, b in zip(outs[0], outs[1]):
        assert torch.allclose(a, b, rtol=0, atol=0, equal_nan=True)
    assert outs[0][0].shape[0] > 2000


def test_rebond():
    """REBOND.m: azimuths up to three wedges out on either side, z beyond both
    ends; against the oracle, and the wrap limit."""
    rng = np.random.default_rng(13)
    n, PHIp, Lp = 20000, 0.1, 1e-2
    r = rng.uniform(1e-4, 5e-3, n)
    phi = rng.uniform(-3.2 * PHIp, 4.2 * PHIp, n)
    pos = np.stack([r * np.cos(phi), r * np.sin(phi), rng.uniform(-0.2 * Lp, 1.3 * Lp, n)], 1)
    vel = rng.normal(size=(n, 3)) * 1e7
    got = gasatt.REBOND(torch.tensor(pos), torch.tensor(r), torch.tensor(phi), torch.tensor(vel),
                        Lp, PHIp)
    want = O.rebond(pos, r, phi, vel, Lp, PHIp)
    assert got[2] == want[2] > n // 2
    close(np_(got[0]), want[0], 1e-14, "pos")
    close(np_(got[1]), want[1], 1e-14, "vel")
    assert np_(got[1])[:, 2].tolist() != vel[:, 2].tolist()       # some z reflections
    bad = phi.copy(); bad[7] = -1e3                                # 10,000 wedges below
    with pytest.raises(gasatt.GasattError):
        gasatt.REBOND(torch.tensor(pos), torch.tensor(r), torch.tensor(bad), torch.tensor(vel),
                      Lp, PHIp)

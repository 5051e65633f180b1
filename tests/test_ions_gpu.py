"""N2+ ion species of the resident simulation, against the oracle and closed
forms.

One ion per ionization (electron_transport.cu:202-204: at the parent's
position, Maxwellian at the gas temperature), ions of charge +e or +2e and
mass m_ion pushed in the electrons' fields (electricmagneticfield6.m:6-7,
68-69), sub-cycled: one push of ion_subcycle x dt every ion_subcycle steps,
whose current the field update adds to the electrons' until the next push."""
import numpy as np
import pytest

import pyoracle as O
from _cases import close, grid_fields
from gasatt import _lib
from gasatt.sim import Sim, births, config
from test_sim_gpu import by_id

pytestmark = pytest.mark.gpu

NR, NZ, D = 32, 64, 5e-6


def ion_cfg(precision, sub, torr=300.0, ion_cap=40000, cap=40000, nr=NR, nz=NZ):
    return config(nr, nz, D, 1e-14, torr, precision=precision, capacity=cap, seed=7,
                  sort_period=0, ion_capacity=ion_cap, ion_subcycle=sub)


def start(precision, sub, n_photo=2000, torr=300.0):
    cfg = ion_cfg(precision, sub, torr=torr)
    parts = births(n_photo, 8.0, NZ * D, seed=3, sigma_r=30e-6, Rp=NR * D)
    sim = Sim(cfg)
    sim.load(*parts)
    Er, Ez, H = grid_fields(NR, NZ, np.random.default_rng(8), E0=3e6, H0=2e3)
    Er[:, 0] = 0; Er[:, -1] = 0; Ez[-1, :] = 0
    sim.set_fields(Er, Ez, H)
    return cfg, sim, parts, (Er, Ez, H)


def alive_by_id(d, keys=("r", "z", "ur", "ut", "uz")):
    a = d["r"] >= 0
    return by_id(d["id"][a], *[d[k][a] for k in keys]), set(d["id"][a].tolist())


def test_fp64_ions_match_oracle(tables):
    """Electrons, ions, fields and counters after 6 steps with an ion push
    every 2 steps."""
    steps, sub = 6, 2
    cfg, sim, parts, flds = start(_lib.FP64, sub)
    sim.step(steps)
    orc = O.Sim(cfg, tables, cap=cfg.capacity)
    orc.load(*parts)
    orc.Er[:], orc.Ez[:], orc.H[:] = flds
    orc.prologue()
    for _ in range(steps):
        orc.step()

    d = sim.diag()
    ion, ela, exc, nul, lost, ovf = orc.counters
    assert (d["n_ionizations"], d["n_elastic"], d["n_excitation"], d["n_null"]) == (ion, ela, exc, nul)
    assert ion > 10
    assert d["collision_loss_ev"] == pytest.approx(orc.collision_loss_ev, rel=1e-12)
    # one ion per ionization, ids of the secondary electrons
    gi = sim.read_ions()
    r, z, ur, ut, uz, ids, alive, q = orc.ion_state_rz()
    assert orc.ions.n == ion and len(gi["id"]) == ion
    a = alive.astype(bool)
    have, hset = alive_by_id(gi)
    assert hset == set(ids[a].tolist())
    want = by_id(ids[a], r[a], z[a], ur[a], ut[a], uz[a])
    for h, w, k in zip(have, want, ("r", "z", "ur", "ut", "uz")):
        close(h, w, 1e-12, "ion " + k)
    assert np.all(gi["charge"] == 1)
    # electrons and fields (the held ion current enters the field update)
    ge = sim.read()
    r, z, ur, ut, uz, ids, alive = orc.state_rz()
    a = alive.astype(bool)
    have, hset = alive_by_id(ge)
    assert hset == set(ids[a].tolist())
    want = by_id(ids[a], r[a], z[a], ur[a], ut[a], uz[a])
    for h, w, k in zip(have, want, ("r", "z", "ur", "ut", "uz")):
        close(h, w, 1e-12, k)
    Er, Ez, H = sim.fields()
    close(Er, orc.Er, 1e-12, "Er"); close(Ez, orc.Ez, 1e-12, "Ez"); close(H, orc.H, 1e-12, "H")


@pytest.mark.parametrize("precision", [_lib.FP64, _lib.FP32_SPLIT])
def test_ion_current_drives_the_fields_like_the_oracle(tables, precision):
    """Ions alone (no electrons), fields zero: the only source is the held ion
    current of each push, so the fields measure its deposit and its addition
    in the field update."""
    sub, steps = 1, 4
    cfg = ion_cfg(precision, sub)
    rng = np.random.default_rng(11)
    n = 3000
    ions = (rng.uniform(2, NR - 3, n) * D, rng.uniform(2, NZ - 3, n) * D,
            rng.normal(0, 2e5, n), rng.normal(0, 2e5, n), rng.normal(0, 2e5, n),
            np.arange(n, dtype=np.uint64) + np.uint64(1 << 40))
    charge = rng.integers(1, 3, n).astype(np.int8)
    sim = Sim(cfg)
    sim.load(*[np.zeros(0)] * 5, np.zeros(0, np.uint64))
    sim.load_ions(*ions, charge=charge)
    sim.step(steps)
    orc = O.Sim(cfg, tables, cap=cfg.capacity)
    orc.load(*[np.zeros(0)] * 5, np.zeros(0, np.uint64))
    orc.load_ions(*ions, charge=charge)
    orc.prologue()
    for _ in range(steps):
        orc.step()
    # FP64: the held ion current is 64-bit fixed point at 2^-48 of q_e FN c per
    # unit, and ions move at |v|/c ~ 1e-3, so each contribution is quantised at
    # ~5e-12 of itself where the oracle sums doubles (measured: 1.2e-12)
    tol = 1e-11 if precision == _lib.FP64 else 1e-5
    Er, Ez, H = sim.fields()
    assert np.abs(orc.Ez).max() > 0
    close(Er, orc.Er, tol, "Er"); close(Ez, orc.Ez, tol, "Ez"); close(H, orc.H, tol, "H")
    gi = sim.read_ions()
    r, z, ur, ut, uz, ids, alive, q = orc.ion_state_rz()
    assert np.array_equal(np.sort(gi["charge"]), np.sort(q))
    have, hset = alive_by_id(gi)
    a = alive.astype(bool)
    assert hset == set(ids[a].tolist())
    want = by_id(ids[a], r[a], z[a], ur[a], ut[a], uz[a])
    for h, w, k in zip(have, want, ("r", "z", "ur", "ut", "uz")):
        close(h, w, 1e-12 if precision == _lib.FP64 else 1e-6, "ion " + k)


@pytest.mark.parametrize("precision", [_lib.FP64, _lib.FP32_SPLIT])
@pytest.mark.parametrize("Z", [1, 2])
def test_ion_kick_in_a_uniform_field(precision, Z):
    """One push of 4 dt in a uniform Ez: delta u_z = Z e E (4 dt) / m_ion and
    delta z = u_z (4 dt) (gamma - 1 < 1e-11), for ions far from the walls."""
    sub = 4
    cfg = ion_cfg(precision, sub, nr=64, nz=64)
    E0 = 1.0e6
    Er = np.zeros((64, 65), order="F")
    Ez = np.full((65, 64), E0, order="F")
    H = np.zeros((64, 64), order="F")
    sim = Sim(cfg)
    sim.load(*[np.zeros(0)] * 5, np.zeros(0, np.uint64))
    sim.set_fields(Er, Ez, H)
    n = 64
    r0 = np.linspace(24, 40, n) * D
    z0 = np.linspace(24, 40, n) * D
    uz0 = np.linspace(-300, 300, n)
    sim.load_ions(r0, z0, np.zeros(n), np.zeros(n), uz0, np.arange(n, dtype=np.uint64),
                  charge=np.full(n, Z, np.int8))
    sim.step(sub)
    gi = sim.read_ions()
    o = np.argsort(gi["id"])
    dt_i = sub * cfg.dt
    uz1 = uz0 + Z * cfg.q_e * E0 * dt_i / cfg.m_ion
    np.testing.assert_allclose(gi["uz"][o], uz1, rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(gi["z"][o], z0 + uz1 * dt_i, rtol=1e-14, atol=1e-20)
    np.testing.assert_allclose(gi["r"][o], r0, rtol=1e-14)
    assert np.all(gi["charge"] == Z)


@pytest.mark.parametrize("precision", [_lib.FP64, _lib.FP32_SPLIT])
def test_ion_births_one_per_ionization_maxwellian(precision):
    cfg, sim, parts, _ = start(precision, 1000, n_photo=4000)
    sim.step(20)
    d = sim.diag()
    gi = sim.read_ions()
    n_ion = d["n_ionizations"]
    assert n_ion > 500
    assert len(gi["id"]) == n_ion and d["n_ions"] == n_ion
    # each ion carries the id of the secondary electron born with it
    ge = sim.read()
    born = set(ge["id"].tolist()) - set(parts[5].tolist())
    assert set(gi["id"].tolist()) == born
    sigma = np.sqrt(cfg.kb * cfg.gas_temperature / cfg.m_ion)
    for k in ("ur", "ut", "uz"):
        u = gi[k]
        assert abs(u.mean()) < 5 * sigma / np.sqrt(n_ion), k
        assert abs(u.std() / sigma - 1) < 5 / np.sqrt(2 * n_ion), k
    e_ion = 0.5 * cfg.m_ion * (gi["ur"]**2 + gi["ut"]**2 + gi["uz"]**2).sum() / cfg.q_e
    assert d["ion_kinetic_ev"] == pytest.approx(e_ion, rel=1e-6)


@pytest.mark.parametrize("precision", [_lib.FP64, _lib.FP32_SPLIT])
def test_charge_is_conserved(precision):
    """Ionizations add an electron and an ion; only the walls remove charge:
    ions - electrons = -N0 + electrons lost - ions lost, exactly."""
    cfg, sim, parts, _ = start(precision, 5, n_photo=3000)
    n0 = len(parts[0])
    sim.step(30)
    d = sim.diag()
    assert d["n_ionizations"] > 100 and d["status_flags"] == 0
    assert d["n_ions"] - d["n_alive"] == -n0 + d["n_lost_wall"] - d["n_ion_lost_wall"]
    assert d["net_charge_c"] == pytest.approx(cfg.q_e * cfg.FN * (d["n_ions"] - d["n_alive"]),
                                              rel=1e-15)


def test_fp32_with_ions_tracks_fp64():
    res = {}
    for prec in (_lib.FP64, _lib.FP32_SPLIT):
        cfg, sim, _, _ = start(prec, 10, n_photo=4000, torr=100.0)
        sim.step(40)
        res[prec] = (sim.diag(), sim.fields())
        sim.close()
    (d64, f64), (d32, f32) = res[_lib.FP64], res[_lib.FP32_SPLIT]
    assert d64["n_ions"] > 200
    assert abs(d32["n_ions"] - d64["n_ions"]) <= 0.005 * d64["n_ions"] + 2
    for a, b in zip(f32, f64):
        close(a, b, 1e-4, "field FP32 vs FP64")


def test_ion_capacity_overflow_is_flagged():
    cfg = ion_cfg(_lib.FP32_SPLIT, 50, ion_cap=20)
    sim = Sim(cfg)
    sim.load(*births(2000, 8.0, NZ * D, seed=3, sigma_r=30e-6, Rp=NR * D))
    sim.step(10)
    d = sim.diag()
    assert d["n_ionizations"] > 20
    assert d["n_ions"] == 20 and d["status_flags"] & 4


def test_ion_arguments_are_checked():
    with pytest.raises(RuntimeError):
        Sim(ion_cfg(_lib.FP64, 0))                       # sub-cycle 0
    sim = Sim(config(NR, NZ, D, 1e-14, 300.0, precision=_lib.FP64, capacity=1000))
    with pytest.raises(RuntimeError):                    # no ion species
        sim.load_ions(np.ones(1) * D, np.ones(1) * D, np.zeros(1), np.zeros(1), np.zeros(1),
                      np.zeros(1, np.uint64))
    assert len(sim.read_ions()["id"]) == 0
    sim2 = Sim(ion_cfg(_lib.FP64, 5, ion_cap=4))
    with pytest.raises(RuntimeError):                    # beyond the ion capacity
        sim2.load_ions(*[np.ones(5) * D] * 2, *[np.zeros(5)] * 3, np.zeros(5, np.uint64))


@pytest.mark.parametrize("precision,tol", [(_lib.FP64, 1e-6), (_lib.FP32_SPLIT, 1e-4)])
def test_energy_budget_closes(precision, tol):
    """No applied field, no wall losses: the electrons' kinetic energy drops by
    what the collisions give to the gas (15.6 eV per ionization plus the
    excitation losses) and what the self-field takes."""
    cfg = ion_cfg(precision, 10)
    sim = Sim(cfg)
    sim.load(*births(4000, 8.0, NZ * D, seed=3, sigma_r=30e-6, Rp=NR * D))
    d0 = sim.diag()
    sim.step(20)
    d = sim.diag()
    assert d["n_lost_wall"] == 0 and d["n_ionizations"] > 100 and d["n_excitation"] > 100
    e_c = 6.241509074e18                          # eV per joule
    lhs = d0["kinetic_ev"] + d0["field_energy_j"] * e_c
    rhs = d["kinetic_ev"] + d["field_energy_j"] * e_c + d["collision_loss_ev"]
    assert abs(rhs - lhs) < tol * lhs, (lhs, rhs, d["collision_loss_ev"])


@pytest.mark.parametrize("precision,tol", [(_lib.FP64, 1e-6), (_lib.FP32_SPLIT, 1e-4)])
def test_energy_budget_closes_with_wall_losses(precision, tol):
    """A narrow cell (80 um radius) that many electrons leave: the energy
    carried out through r = Rp is counted too, so the electrons' kinetic +
    field + given to the gas + absorbed at the wall stays what it was.  The
    ions' kinetic energy is left out: they are born with a thermal 0.04 eV
    each (600 eV over this run, more than the FP64 tolerance) that the
    electrons never had."""
    nr = 16
    cfg = ion_cfg(precision, 10, nr=nr)
    sim = Sim(cfg)
    sim.load(*births(3000, 8.0, NZ * D, seed=3, sigma_r=30e-6, Rp=nr * D))
    d0 = sim.diag()
    sim.step(200)
    d = sim.diag()
    assert d["n_lost_wall"] > 500 and d["wall_loss_ev"] > 0.1 * d0["kinetic_ev"]
    e_c = 6.241509074e18                          # eV per joule
    lhs = d0["kinetic_ev"] + d0["field_energy_j"] * e_c
    rhs = d["kinetic_ev"] + d["field_energy_j"] * e_c + d["collision_loss_ev"] + d["wall_loss_ev"]
    assert abs(rhs - lhs) < tol * lhs, (lhs, rhs, d["wall_loss_ev"])


def test_gas_temperature_map_sets_the_newborn_ions_spread(tables):
    """A per-cell gas temperature (300 K in the lower half of z, 3000 K in the
    upper): the FP64 form's ions match the oracle's, and ions born in the hot
    half spread sqrt(10) times wider.  A uniform 300 K map is the scalar run."""
    steps = 20
    cfg, sim, parts, flds = start(_lib.FP64, 1000, n_photo=3000)
    T = np.full((NR, NZ), 300.0)
    T[:, NZ // 2:] = 3000.0
    sim.set_gas_temperature(T)
    sim.step(steps)
    gi = sim.read_ions()
    orc = O.Sim(cfg, tables, cap=cfg.capacity)
    orc.load(*parts)
    orc.Er[:], orc.Ez[:], orc.H[:] = flds
    orc.set_gas_temperature(T)
    orc.prologue()
    for _ in range(steps):
        orc.step()
    r, z, ur, ut, uz, ids, alive, q = orc.ion_state_rz()
    assert len(gi["id"]) == len(ids) > 300
    have, _ = alive_by_id(gi)
    want = by_id(ids, r, z, ur, ut, uz)
    for h, w, k in zip(have, want, ("r", "z", "ur", "ut", "uz")):
        close(h, w, 1e-12, "ion " + k)
    hot = gi["z"] >= NZ // 2 * D
    s_hot, s_cold = gi["uz"][hot].std(), gi["uz"][~hot].std()
    assert hot.sum() > 100 and (~hot).sum() > 100
    assert abs(s_hot / s_cold / np.sqrt(10) - 1) < 0.25
    # a uniform map at the configured temperature is the scalar run
    runs = []
    for use_map in (False, True):
        cfg2, sim2, _, _ = start(_lib.FP32_SPLIT, 1000)
        if use_map:
            sim2.set_gas_temperature(np.full((NR, NZ), cfg2.gas_temperature))
        sim2.step(8)
        st = sim2.read_ions()
        o = np.argsort(st["id"])
        runs.append(np.stack([st[k][o] for k in ("r", "z", "ur", "ut", "uz")]))
        sim2.close()
    assert runs[0].shape[1] > 10 and np.array_equal(runs[0], runs[1])

"""CPU checks of the oracle: known-answer vectors, MATLAB built-in semantics,
table assembly, and physics invariants of the restated kernels."""
import math

import numpy as np
import pytest

import pyoracle as O
from _cases import cell_structure, close, grid_fields, wedge_particles
from gasatt import _lib

A0SQ = 2.8002852e-21


def test_philox_known_answers():
    # Random123 kat_vectors, philox4x32 10 rounds
    assert O.philox([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert O.philox([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert O.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_u01_open_interval():
    assert 0 < O.lib.orc_u01(0, 0) < 1e-15
    assert 1 - 1e-15 < O.lib.orc_u01(0xffffffff, 0xffffffff) < 1


def test_child_ids_distinct():
    ids = {O.child_id(p, s) for p in range(200) for s in range(50)}
    assert len(ids) == 200 * 50


def test_interp1_semantics():
    x = np.array([1.0, 2.0, 4.0]); y = np.array([10.0, 20.0, 0.0])
    f = lambda q: O.lib.orc_interp1(O.P(x), 1, O.P(y), 1, 3, q)
    assert f(1.0) == 10.0 and f(2.0) == 20.0 and f(4.0) == 0.0
    assert f(1.5) == 15.0 and f(3.0) == 10.0
    assert math.isnan(f(0.999)) and math.isnan(f(4.001))


def test_find_cs0_faithful_at_knots(tables):
    t_el, t_sel, t_ion, t_exc = tables["t_el"], tables["t_sel"], tables["t_ion"], tables["t_exc"]
    E = np.concatenate([t_el[0, :], t_sel[:-1, 0] / 1000])
    se, si, sx = O.find_cs0(tables, E, _lib.FAITHFUL)
    n = t_el.shape[1]
    np.testing.assert_allclose(se[:n], t_el[1, :] * A0SQ * 2, rtol=1e-15)
    # below 50 eV the small-energy table in 1e-20 m^2 (find_CS0.m:108-111)
    np.testing.assert_allclose(se[n:], t_sel[:-1, 1] * 1e-20, rtol=1e-15)
    # ionization at its own knots
    _, si2, _ = O.find_cs0(tables, t_ion[:, 0] / 1000, _lib.FAITHFUL)
    np.testing.assert_allclose(si2, t_ion[:, 1] * 1e-20, rtol=1e-15)
    # excitation restated by hand at 1 keV (find_CS0.m:123-142)
    T = 1000.0
    ref = sum(6.542e-14 * A / k**2 * (k / T) ** om * (1 - (k / T) ** ga) ** nu
              for k, A, om, nu, ga in t_exc) * 1e-4
    _, _, sx1 = O.find_cs0(tables, np.array([1.0]), _lib.FAITHFUL)
    assert abs(sx1[0] - ref) <= 1e-15 * abs(ref)


def test_find_cs0_nan_outside_tables(tables):
    se, si, sx = O.find_cs0(tables, np.array([0.0005, 0.010, 25.0]), _lib.FAITHFUL)
    assert math.isnan(se[0]) and math.isnan(si[0])     # 0.5 eV: below both tables
    assert not math.isnan(se[1]) and math.isnan(si[1])  # 10 eV: elastic ok, below 15.6 eV
    assert math.isnan(se[2]) and math.isnan(si[2])     # 25 keV: above both tables


def test_find_cs0_corrected_finite(tables):
    E = np.logspace(np.log10(1e-4), np.log10(30.0), 3000)
    se, si, sx = O.find_cs0(tables, E, 0)
    assert np.all(np.isfinite(se)) and np.all(se > 0)
    assert np.all(np.isfinite(si)) and np.all(si >= 0)
    assert np.all(si[E * 1000 <= 15.6] == 0)
    assert np.all(np.isfinite(sx)) and np.all(sx >= 0)
    assert np.all(sx[E * 1000 <= tables["t_exc"][:, 0].min()] == 0)


def test_elastic_tables_assembly(tables):
    xI, yI, V = O.elastic_tables(tables)
    assert xI.size == 36 and V.shape == (36, 181)
    E = np.concatenate([tables["t_sdel"][0, 1:], tables["t_del"][0, 1:]])
    np.testing.assert_array_equal(xI, np.log(E))
    # electron_collision.m:15-20: low-energy TCS rescaled to a0^2 per atom, last row dropped
    np.testing.assert_allclose(yI[:7], tables["t_sel_1"][:7, 1] * 1e-20 / A0SQ / 2, rtol=1e-15)
    np.testing.assert_array_equal(yI[7:], tables["t_el"][1, :])
    np.testing.assert_array_equal(V[0], np.log(tables["t_sdel"][1:, 1]))
    np.testing.assert_array_equal(V[-1], np.log(tables["t_del"][1:, -1]))


def test_null_collision_bound_holds(tables):
    n_gas = 3.2e22
    xs = O.XS(tables, 2048, 0.1, 30000.0, n_gas, 299792458.0, 9.1093837015e-31, 1.602176634e-19)
    se, si, sx = xs.array(0), xs.array(1), xs.array(2)
    G = 2048
    lnE = np.log(0.1) + np.arange(G) * (np.log(30000.0) - np.log(0.1)) / (G - 1)
    # dense sampling between grid points, linear in the log index
    f = np.linspace(0, 1, 17)[None, :]
    L = (np.arange(G - 1)[:, None] + f).ravel()
    i = np.minimum(L.astype(int), G - 2)
    fr = L - i
    st = se + si + sx
    sig = st[i] + fr * (st[i + 1] - st[i])
    E = np.exp(lnE[0] + L * (lnE[1] - lnE[0]))
    eps = E * 1.602176634e-19 / (9.1093837015e-31 * 299792458.0**2)
    v = 299792458.0 * np.sqrt(eps * (2 + eps)) / (1 + eps)
    assert np.max(n_gas * sig * v) <= xs.nu_max * (1 + 1e-12)
    cdf = xs.array(3).reshape(G, 181)
    assert np.all(cdf[:, 0] == 0) and np.all(cdf[:, -1] == 1) and np.all(np.diff(cdf, axis=1) > 0)


def test_boris_pure_magnetic_conserves_energy():
    """EM4 with the Boris flag: a magnetic-only field does no work."""
    rng = np.random.default_rng(5)
    nr, nz, d = 16, 32, 1e-4
    _, _, H = grid_fields(nr, nz, rng, H0=5e4)
    Er = np.zeros((nr, nz + 1), order="F"); Ez = np.zeros((nr + 1, nz), order="F")
    pos, v = wedge_particles(500, nr * d, nz * d, 0.1, rng, cyl=False, vmag=2e7)
    x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
    vx, vy, vz = (np.ascontiguousarray(v[:, k]) for k in range(3))
    r = np.hypot(x, y); phi = np.arctan2(y, x); vr = vx * np.cos(phi) + vy * np.sin(phi)
    q = np.full(500, -1.6e-19); m = np.full(500, 9.1096e-31); E = np.zeros(500)
    dele = np.zeros(500, np.int32)
    speed0 = np.sqrt(vx**2 + vy**2 + vz**2)
    O.em4(x, y, z, vx, vy, vz, r, phi, vr, Er, Ez, H, q, m, E, dele, nr * d, nz * d, 0.1, nr, nz,
          4e-7 * math.pi, 3e8, d, d, 5e-13, 0)
    speed1 = np.sqrt(vx**2 + vy**2 + vz**2)
    close(speed1, speed0, 1e-14, "|v| under Boris in pure B")


def test_fdtd_vacuum_energy_bounded():
    """Source-free Yee cavity (conducting walls): field energy stays bounded."""
    from gasatt.sim import config
    cfg = config(24, 48, 1e-5, 2e-14, 1.0, precision=_lib.FP64)
    rng = np.random.default_rng(3)
    Er, Ez, H = grid_fields(24, 48, rng)
    Er[:, 0] = 0; Er[:, -1] = 0; Ez[-1, :] = 0
    j = np.zeros((24, 48), order="F")
    Er, Ez, H = (np.asfortranarray(a) for a in (Er, Ez, H))
    W = []
    for _ in range(400):
        O.lib.orc_sim_fdtd(O.ctypes.byref(cfg), O.P(Er), O.P(Ez), O.P(H), O.P(j), O.P(j))
        W.append(O.lib.orc_field_energy(O.ctypes.byref(cfg), O.P(Er), O.P(Ez), O.P(H)))
    W = np.array(W)
    assert np.all(np.isfinite(W))
    assert W.max() / W.min() < 1.5


def test_free_motion_formula():
    rng = np.random.default_rng(1)
    a = [rng.normal(size=100) for _ in range(6)]
    xn, yn, zn, rn, phin = O.free_motion(*a, 1e-3)
    np.testing.assert_array_equal(xn, a[3] + a[0] * 1e-3)
    np.testing.assert_array_equal(rn, np.sqrt(xn * xn + yn * yn))
    np.testing.assert_allclose(phin, np.arctan2(yn, xn), rtol=1e-15, atol=1e-15)  # libm vs numpy atan2


def test_particle_density_counts():
    PHIp, Rp, rmax, delta = 0.1, 1e-2, 10, 1e-3
    phimax, sum_cell, cellnumxy = cell_structure(PHIp, Rp, rmax, delta)
    zmax, dz = 4, 1e-2
    dphi = PHIp / phimax
    VC = np.concatenate([[0.5 * ((i * delta)**2 - ((i - 1) * delta)**2) * dphi[i - 1] * dz]
                         * int(phimax[i - 1]) for i in range(1, rmax + 1)])
    rng = np.random.default_rng(0)
    n = 5000
    r = rng.uniform(0, Rp * 0.999, n); phi = rng.uniform(0, PHIp * 0.999, n); z = rng.uniform(0, zmax * dz * 0.999, n)
    dens = O.particle_density(delta, dz, dphi, r, phi, z, cellnumxy, sum_cell, VC, 2.0, cellnumxy * zmax)
    counts = dens * np.tile(VC, zmax) / 2.0
    assert abs(counts.sum() - n) < 1e-6
    # one particle by hand: ring 3, phi cell 2, layer 2
    i_r, i_p, i_z = 3, 2, 2
    r1 = np.array([(i_r - 0.5) * delta]); z1 = np.array([(i_z - 0.5) * dz])
    p1 = np.array([(i_p - 0.5) * dphi[i_r - 1]])
    d1 = O.particle_density(delta, dz, dphi, r1, p1, z1, cellnumxy, sum_cell, VC, 1.0, cellnumxy * zmax)
    idx = (i_z - 1) * cellnumxy + int(sum_cell[i_r - 2]) + i_p - 1
    assert np.nonzero(d1)[0].tolist() == [idx]


def test_emf6_oracle_wall_deletion_and_counts():
    rng = np.random.default_rng(2)
    nr, nz, d = 12, 20, 1e-4
    Er, Ez, H = grid_fields(nr, nz, rng)
    pos, v = wedge_particles(300, nr * d, nz * d, 0.1, rng, vmag=3e7)
    pos[:5, 0] = nr * d * 0.9999                # at the wall, moving outward in x
    v[:5] = [[3e7, 0, 0]] * 5
    out = O.electricmagneticfield6(pos, v, np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 3)),
                                   np.zeros((0, 3)), Er, Ez, H, d, 1e-13, nr * d, nz * d, 0.1,
                                   1.0, 10, _lib.FAITHFUL | _lib.POS_IN_CYL)
    e_pos, kin = out[0], out[9]
    assert len(e_pos) <= 295 and len(kin) == len(e_pos)
    assert np.all(np.hypot(e_pos[:, 0], e_pos[:, 1]) <= nr * d)
    assert np.all((e_pos[:, 2] >= 0) & (e_pos[:, 2] <= nz * d))


def _oracle_sim(tables, gas=None, steps=3):
    from gasatt.sim import births, config
    nr, nz, d = 16, 32, 5e-6
    cfg = config(nr, nz, d, 1e-14, 300.0, precision=_lib.FP64, capacity=8000, seed=7)
    orc = O.Sim(cfg, tables, cap=cfg.capacity)
    orc.load(*births(600, 8.0, nz * d, seed=3, sigma_r=30e-6, Rp=nr * d))
    if gas is not None:
        orc.set_gas_density(gas(cfg, nr, nz))
    orc.prologue()
    for _ in range(steps):
        orc.step()
    return orc


def test_oracle_uniform_gas_map_equals_scalar_density(tables):
    a = _oracle_sim(tables)
    b = _oracle_sim(tables, lambda cfg, nr, nz: np.full((nr, nz), cfg.gas_density))
    assert a.counters[0] > 0 and np.array_equal(a.counters, b.counters)
    for u, v in zip(a.state_rz(), b.state_rz()):
        assert np.array_equal(u, v)
    assert np.array_equal(a.jr, b.jr) and np.array_equal(a.jz, b.jz)


def test_oracle_vacuum_gas_map_has_no_collisions(tables):
    o = _oracle_sim(tables, lambda cfg, nr, nz: np.zeros((nr, nz)))
    assert list(o.counters[:4]) == [0, 0, 0, 0]


def test_oracle_rebond_small_case():
    """REBOND.m by hand: one particle a wedge and a half below, one above,
    one past z = Lp."""
    PHIp, Lp = 0.5, 1.0
    pos = np.array([[0.0, 0.0, 0.5], [0.0, 0.0, 0.5], [1.0, 0.0, 1.25]])
    r = np.array([2.0, 1.0, 1.0])
    phi = np.array([-0.75, 0.8, 0.0])
    vel = np.array([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 3.0]])
    p, v, nb = O.rebond(pos, r, phi, vel, Lp, PHIp)
    assert nb == 2 + 1 + 1
    np.testing.assert_allclose(p[0, :2], [2 * np.cos(0.25), 2 * np.sin(0.25)], rtol=1e-15)
    np.testing.assert_allclose(v[0, :2], [np.cos(1.0), np.sin(1.0)], rtol=1e-15)   # turned by 2 PHIp
    np.testing.assert_allclose(p[1, :2], [np.cos(0.3), np.sin(0.3)], rtol=1e-14)
    np.testing.assert_allclose(v[1, :2], [np.sin(0.5), np.cos(0.5)], rtol=1e-15)   # turned by -PHIp
    np.testing.assert_allclose([p[2, 2], v[2, 2]], [0.75, -3.0], rtol=1e-15)
    assert O.rebond(pos, r, np.array([-10.0, 0.0, 0.0]), vel, Lp, PHIp, max_wraps=8)[2] == -1


def test_oracle_ion_births_follow_the_gas_temperature_map(tables):
    """Oracle ions born in the 3000 K half spread sqrt(10) wider than those
    born in the 300 K half (one ion per ionization)."""
    from gasatt.sim import births, config
    nr, nz, d = 16, 32, 5e-6
    cfg = config(nr, nz, d, 1e-14, 300.0, precision=_lib.FP64, capacity=20000, seed=7,
                 ion_capacity=20000, ion_subcycle=1000)
    orc = O.Sim(cfg, tables, cap=cfg.capacity)
    orc.load(*births(3000, 8.0, nz * d, seed=3, sigma_r=30e-6, Rp=nr * d))
    T = np.full((nr, nz), 300.0)
    T[:, nz // 2:] = 3000.0
    orc.set_gas_temperature(T)
    orc.prologue()
    for _ in range(15):
        orc.step()
    r, z, ur, ut, uz, ids, alive, q = orc.ion_state_rz()
    assert len(ids) == orc.counters[0] > 300
    hot = z >= nz // 2 * d
    assert abs(uz[hot].std() / uz[~hot].std() / np.sqrt(10) - 1) < 0.25

"""Per-cell neutral gas density in the resident simulation
(gasatt_sim_set_gas_density), against the uniform scalar run and the oracle.

The reference looks the gas density up by cell before every collision
(electron_transport.cu:64-76); the resident simulation takes the density of
the cell an electron ends the step in, with the null-collision bound set by
the densest cell."""
import numpy as np
import pytest

from _cases import close
from gasatt import _lib
from gasatt.sim import Sim
from test_sim_gpu import NR, NZ, by_id, oracle_run, start

pytestmark = pytest.mark.gpu


def graded(cfg):
    """Density rising along z from 0.2 to 1.8 times the uniform value, with a
    radial dip: every cell differs, the densest is 1.8 x."""
    iz = (np.arange(NZ) + 0.5) / NZ
    ir = (np.arange(NR) + 0.5) / NR
    return cfg.gas_density * np.outer(1.0 - 0.3 * ir**2, 0.2 + 1.6 * iz)


def snapshot(sim):
    d = sim.diag()
    jr, jz = sim.current()
    return (sim.read(), sim.fields(), (jr, jz),
            (d["n_ionizations"], d["n_elastic"], d["n_excitation"], d["n_null"], d["n_alive"]))


@pytest.mark.parametrize("precision", [_lib.FP64, _lib.FP32_SPLIT])
def test_uniform_map_reproduces_scalar_run_bit_for_bit(precision):
    outs = []
    for use_map in (False, True):
        cfg, sim, _, _ = start(precision)
        if use_map:
            sim.set_gas_density(np.full((NR, NZ), cfg.gas_density))
        sim.step(6)
        outs.append(snapshot(sim))
        sim.close()
    (p0, f0, j0, c0), (p1, f1, j1, c1) = outs
    assert c0 == c1 and c0[0] > 0
    # births take slots in the order the collision threads reach them, so the
    # particles are compared by id
    o0, o1 = np.argsort(p0["id"]), np.argsort(p1["id"])
    for k in ("r", "z", "ur", "ut", "uz", "id"):
        assert np.array_equal(p0[k][o0], p1[k][o1]), k
    for a, b in zip(f0 + j0, f1 + j1):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("switch_at", [0, 2])
def test_fp64_graded_density_matches_oracle(tables, switch_at):
    """Graded density from the start, or switched on after two uniform steps
    (the collisions queued at the switch still see the old density)."""
    steps = 5
    cfg, sim, parts, flds = start(_lib.FP64)
    rho = graded(cfg)
    sim.step(switch_at)
    sim.set_gas_density(rho)
    sim.step(steps - switch_at)
    got = sim.read()

    import pyoracle as O
    orc = O.Sim(cfg, tables, cap=cfg.capacity)
    orc.load(*parts)
    orc.Er[:], orc.Ez[:], orc.H[:] = flds
    orc.prologue()
    for s in range(steps):
        if s == switch_at:
            orc.set_gas_density(rho)
        orc.step()
    r, z, ur, ut, uz, ids, alive = orc.state_rz()
    a = alive.astype(bool)
    g_alive = got["r"] >= 0
    assert set(got["id"][g_alive].tolist()) == set(ids[a].tolist())
    want = by_id(ids[a], r[a], z[a], ur[a], ut[a], uz[a])
    have = by_id(got["id"][g_alive], got["r"][g_alive], got["z"][g_alive], got["ur"][g_alive],
                 got["ut"][g_alive], got["uz"][g_alive])
    for h, w, k in zip(have, want, ("r", "z", "ur", "ut", "uz")):
        close(h, w, 1e-12, k)
    d = sim.diag()
    ion, ela, exc, nul, lost, ovf = orc.counters
    assert (d["n_ionizations"], d["n_elastic"], d["n_excitation"], d["n_null"]) == (ion, ela, exc, nul)
    assert ion > 10 and ela > 10
    jr, jz = sim.current()
    close(jr, orc.jr, 1e-12, "jr"); close(jz, orc.jz, 1e-12, "jz")
    # the graded run differs from the uniform one (the map is really used)
    uni = oracle_run(cfg, tables, parts, flds, steps)
    assert tuple(uni.counters[:4]) != (ion, ela, exc, nul)


@pytest.mark.parametrize("precision", [_lib.FP64, _lib.FP32_SPLIT])
def test_vacuum_map_stops_all_collisions_and_reverts(precision):
    cfg, sim, _, _ = start(precision)
    sim.set_gas_density(np.zeros((NR, NZ)))
    sim.step(4)
    d = sim.diag()
    assert (d["n_ionizations"], d["n_elastic"], d["n_excitation"], d["n_null"]) == (0, 0, 0, 0)
    sim.set_gas_density(None)                    # back to the uniform density
    sim.step(3)
    d = sim.diag()
    assert d["n_ionizations"] > 0 and d["n_elastic"] > 0


def test_fp32_graded_density_tracks_fp64():
    """Collision counts of the two forms under the same graded map agree to
    the FP32 yield tolerance (0.5 %)."""
    res = {}
    for prec in (_lib.FP64, _lib.FP32_SPLIT):
        cfg, sim, _, _ = start(prec, n_photo=4000, torr=100.0)
        sim.set_gas_density(graded(cfg))
        sim.step(30)
        res[prec] = sim.diag()
        sim.close()
    i64, i32 = res[_lib.FP64]["n_ionizations"], res[_lib.FP32_SPLIT]["n_ionizations"]
    assert i64 > 100
    assert abs(i32 - i64) <= 0.005 * i64 + 2


def test_bad_density_is_rejected():
    cfg, sim, _, _ = start(_lib.FP32_SPLIT)
    for bad in (-1.0, np.nan, np.inf):
        rho = np.full((NR, NZ), cfg.gas_density)
        rho[3, 5] = bad
        with pytest.raises(RuntimeError):
            sim.set_gas_density(rho)
    with pytest.raises(ValueError):
        sim.set_gas_density(np.full((NZ, NR), cfg.gas_density))
    sim.step(2)                                  # the simulation is still usable
    assert sim.diag()["n_ionizations"] >= 0

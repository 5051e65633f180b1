"""Resident simulation (the hot path) against the CPU oracle, plus the
FP32-split-vs-FP64 accuracy gates and run-to-run bit-exactness."""
import numpy as np
import pytest

import pyoracle as O
from _cases import close, grid_fields
from gasatt import _lib
from gasatt.sim import Sim, births, config

pytestmark = pytest.mark.gpu

NR, NZ, D = 32, 64, 5e-6


def small_cfg(precision, torr=300.0, sort_period=0, seed=7, cap=40000):
    return config(NR, NZ, D, 1e-14, torr, precision=precision, capacity=cap, seed=seed,
                  sort_period=sort_period)


def start(precision, n_photo=2000, sort_period=0, fields=True, torr=300.0):
    cfg = small_cfg(precision, torr=torr, sort_period=sort_period)
    r, z, ur, ut, uz, ids = births(n_photo, 8.0, NZ * D, seed=3, sigma_r=30e-6, Rp=NR * D)
    sim = Sim(cfg)
    sim.load(r, z, ur, ut, uz, ids)
    Er = Ez = H = None
    if fields:
        Er, Ez, H = grid_fields(NR, NZ, np.random.default_rng(8), E0=3e6, H0=2e3)
        Er[:, 0] = 0; Er[:, -1] = 0; Ez[-1, :] = 0
        sim.set_fields(Er, Ez, H)
    return cfg, sim, (r, z, ur, ut, uz, ids), (Er, Ez, H)


def oracle_run(cfg, tables, parts, flds, steps):
    orc = O.Sim(cfg, tables, cap=cfg.capacity)
    orc.load(*parts)
    if flds[0] is not None:
        orc.Er[:], orc.Ez[:], orc.H[:] = flds
    orc.prologue()
    for _ in range(steps):
        orc.step()
    return orc


def by_id(state_ids, *arrays):
    order = np.argsort(state_ids)
    return [a[order] for a in arrays]


@pytest.mark.parametrize("steps", [1, 4])
def test_fp64_matches_oracle(tables, steps):
    cfg, sim, parts, flds = start(_lib.FP64)
    sim.step(steps)
    got = sim.read()
    orc = oracle_run(cfg, tables, parts, flds, steps)
    r, z, ur, ut, uz, ids, alive = orc.state_rz()
    # same population: alive ids (births included) identical
    g_alive = got["r"] >= 0
    assert set(got["id"][g_alive].tolist()) == set(ids[alive.astype(bool)].tolist())
    assert len(got["id"]) == len(ids)
    a = alive.astype(bool)
    want = by_id(ids[a], r[a], z[a], ur[a], ut[a], uz[a])
    have = by_id(got["id"][g_alive], got["r"][g_alive], got["z"][g_alive], got["ur"][g_alive],
                 got["ut"][g_alive], got["uz"][g_alive])
    for h, w, k in zip(have, want, ("r", "z", "ur", "ut", "uz")):
        close(h, w, 1e-12, k)
    d = sim.diag()
    ion, ela, exc, nul, lost, ovf = orc.counters
    assert (d["n_ionizations"], d["n_elastic"], d["n_excitation"], d["n_null"]) == (ion, ela, exc, nul)
    assert d["n_lost_wall"] == lost
    if steps > 1:
        assert ion > 10 and ela > 10 and exc > 10
    Er, Ez, H = sim.fields()
    close(Er, orc.Er, 1e-12, "Er"); close(Ez, orc.Ez, 1e-12, "Ez"); close(H, orc.H, 1e-12, "H")
    jr, jz = sim.current()
    close(jr, orc.jr, 1e-12, "jr"); close(jz, orc.jz, 1e-12, "jz")


def test_fp64_field_energy_diag_matches_oracle(tables):
    cfg, sim, parts, flds = start(_lib.FP64)
    sim.step(2)
    orc = oracle_run(cfg, tables, parts, flds, 2)
    close(sim.diag()["field_energy_j"], orc.field_energy(), 1e-12, "field energy")


@pytest.mark.parametrize("precision", [_lib.FP64, _lib.FP32_SPLIT])
def test_bit_exact_run_to_run_and_sort_invariant(precision):
    outs = []
    for sp in (0, 0, 1):
        cfg, sim, _, _ = start(precision, sort_period=sp)
        sim.step(6)
        jr, jz = sim.current()
        Er, Ez, H = sim.fields()
        d = sim.diag()
        outs.append((jr, jz, Er, Ez, H, d["n_ionizations"], d["n_alive"]))
        sim.close()
    for o in outs[1:]:
        for a, b in zip(outs[0], o):
            assert np.array_equal(a, b)


def test_fp32_split_tracks_fp64():
    res = {}
    for prec in (_lib.FP64, _lib.FP32_SPLIT):
        cfg, sim, parts, _ = start(prec, n_photo=4000, sort_period=5, torr=100.0)
        sim.step(40)
        res[prec] = (sim.diag(), sim.fields(), sim.read())
    d64, f64, p64 = res[_lib.FP64]
    d32, f32, p32 = res[_lib.FP32_SPLIT]
    assert d64["n_ionizations"] > 200
    assert abs(d32["n_ionizations"] - d64["n_ionizations"]) <= 0.005 * d64["n_ionizations"] + 2
    assert abs(d32["kinetic_ev"] / d64["kinetic_ev"] - 1) < 1e-4
    for a, b in zip(f32, f64):
        close(a, b, 1e-4, "field FP32 vs FP64")


def test_capacity_overflow_is_reported():
    cfg = small_cfg(_lib.FP32_SPLIT, cap=4100)
    r, z, ur, ut, uz, ids = births(2000, 8.0, NZ * D, seed=3, sigma_r=30e-6, Rp=NR * D)
    sim = Sim(cfg)
    sim.load(r, z, ur, ut, uz, ids)
    sim.step(20)
    d = sim.diag()
    assert d["n_total"] <= 4100
    assert d["status_flags"] & 2


def test_fp64_matches_oracle_multi_window(tables):
    """A grid large enough for several deposit windows and field tiles per
    direction (64 x 256 cells), 20,000 electrons, three steps."""
    cfg = config(64, 256, 5e-6, 1e-14, 300.0, precision=_lib.FP64, capacity=60000, seed=11,
                 sort_period=2)
    r, z, ur, ut, uz, ids = births(10000, 8.0, 256 * 5e-6, seed=5, sigma_r=60e-6, Rp=64 * 5e-6)
    Er, Ez, H = grid_fields(64, 256, np.random.default_rng(2), E0=3e6, H0=2e3)
    Er[:, 0] = 0; Er[:, -1] = 0; Ez[-1, :] = 0
    sim = Sim(cfg)
    sim.load(r, z, ur, ut, uz, ids)
    sim.set_fields(Er, Ez, H)
    sim.step(3)
    orc = oracle_run(cfg, tables, (r, z, ur, ut, uz, ids), (Er, Ez, H), 3)
    got = sim.read()
    rr, zz, urr, utt, uzz, oid, alive = orc.state_rz()
    a = alive.astype(bool)
    ga = got["r"] >= 0
    assert set(got["id"][ga].tolist()) == set(oid[a].tolist())
    want = by_id(oid[a], rr[a], zz[a], urr[a], utt[a], uzz[a])
    have = by_id(got["id"][ga], got["r"][ga], got["z"][ga], got["ur"][ga], got["ut"][ga], got["uz"][ga])
    for h, w, k in zip(have, want, ("r", "z", "ur", "ut", "uz")):
        close(h, w, 1e-12, k)
    jr, jz = sim.current()
    close(jr, orc.jr, 1e-12, "jr"); close(jz, orc.jz, 1e-12, "jz")
    f = sim.fields()
    for g, w, k in zip(f, (orc.Er, orc.Ez, orc.H), ("Er", "Ez", "H")):
        close(g, w, 1e-12, k)
    d = sim.diag()
    assert (d["n_ionizations"], d["n_elastic"], d["n_excitation"]) == tuple(orc.counters[:3])


@pytest.mark.parametrize("precision", [_lib.FP64, _lib.FP32_SPLIT])
@pytest.mark.parametrize("sort_period", [0, 3])
def test_births_conserved(precision, sort_period):
    """Every ionization appends exactly one secondary (secondaries=1): over many
    steps, one at a time and in bursts, the alive count equals the loaded count
    plus the ionizations minus the wall losses, the state agrees with it, and
    no id repeats; without sorting no slot is ever reused."""
    cfg, sim, parts, _ = start(precision, n_photo=4000, sort_period=sort_period, torr=600.0)
    n0 = len(parts[0])
    for burst in (1, 1, 1, 2, 5, 1, 10, 1, 20):
        sim.step(burst)
        d = sim.diag()
        got = sim.read()
        alive = got["r"] >= 0
        assert d["n_alive"] == n0 + d["n_ionizations"] - d["n_lost_wall"]
        assert int(alive.sum()) == d["n_alive"]
        if sort_period == 0:
            assert d["n_total"] == n0 + d["n_ionizations"]
        assert len(np.unique(got["id"][alive])) == int(alive.sum())
    assert d["n_ionizations"] > 50


def test_fp32_gather_matches_fp64_in_strong_fields():
    """One step in strong random fields: the FP32 form's packed-quad gather
    gives the kicks of the FP64 form's scalar gather to float precision (a
    wrong corner or edge clamp would show as an O(1) error in the kick)."""
    got = {}
    for prec in (_lib.FP64, _lib.FP32_SPLIT):
        cfg, sim, parts, _ = start(prec, n_photo=4000)
        sim.set_gas_density(np.zeros((NR, NZ)))          # no collisions: pure push
        sim.step(1)
        d = sim.read()
        got[prec] = by_id(d["id"], d["r"], d["z"], d["ur"], d["ut"], d["uz"])
        u0 = np.sqrt(parts[2]**2 + parts[3]**2 + parts[4]**2)
        sim.close()
    r64, z64, ur64, ut64, uz64 = got[_lib.FP64]
    r32, z32, ur32, ut32, uz32 = got[_lib.FP32_SPLIT]
    umax = u0.max()
    for a, b, k in ((ur32, ur64, "ur"), (ut32, ut64, "ut"), (uz32, uz64, "uz")):
        assert np.abs(a - b).max() < 5e-7 * umax, k     # kicks here are ~1e-4 of |u|
    assert np.abs(r32 - r64).max() < 1e-6 * NR * D
    assert np.abs(z32 - z64).max() < 1e-6 * NZ * D


@pytest.mark.parametrize("precision,tol", [(_lib.FP64, 1e-8), (_lib.FP32_SPLIT, 1e-6)])
def test_free_drift_keeps_kinetic_energy(precision, tol):
    """2000 steps without fields or collisions (gas map all zero, FN 1e-6 so
    the self-field does no measurable work): the drift only turns (u_r,
    u_theta), so the kinetic energy must stay put; the FP32 form's turns are
    far below one ulp of u each step, and stochastic rounding keeps them from
    adding up to a drift."""
    nr, nz = 64, 64
    cfg = config(nr, nz, D, 1e-14, 1.0, precision=precision, capacity=8000, seed=5,
                 sort_period=50, FN=1e-6)
    rng = np.random.default_rng(9)
    n = 8000
    speed = 5.93e6                                     # about 100 eV
    ct = rng.uniform(-1, 1, n); ph = rng.uniform(0, 2 * np.pi, n); st = np.sqrt(1 - ct**2)
    sim = Sim(cfg)
    # radii 20-150 um against a wall at 320 um: 2000 steps move them 119 um at most
    sim.load(rng.uniform(20e-6, 150e-6, n), rng.uniform(5, nz - 5, n) * D,
             speed * st * np.cos(ph), speed * st * np.sin(ph), speed * ct,
             np.arange(n, dtype=np.uint64))
    sim.set_gas_density(np.zeros((nr, nz)))
    e0 = sim.diag()["kinetic_ev"]
    sim.step(2000)
    d = sim.diag()
    assert d["n_lost_wall"] == 0 and d["n_alive"] == n
    assert abs(d["kinetic_ev"] / e0 - 1) < tol, d["kinetic_ev"] / e0 - 1


C1 = dict(nr=64, nz=256, d=10e-6, dt=2e-14, torr=1.0, photo=10_000, steps=500, seed=0)


def c1_cfg(precision):
    return config(C1["nr"], C1["nz"], C1["d"], C1["dt"], C1["torr"], precision=precision,
                  capacity=200_000, seed=C1["seed"], sort_period=30)


@pytest.fixture(scope="module")
def c1_oracle(tables):
    """The oracle's run of the reference's CPU-runnable case at full size:
    20,000 electrons (10,000 photoionizations at 8 keV), 64 x 256 cells at
    10 um, 1 Torr, dt 2e-14 s, 500 steps."""
    cfg = c1_cfg(_lib.FP64)
    parts = births(C1["photo"], 8.0, C1["nz"] * C1["d"], seed=C1["seed"], Rp=C1["nr"] * C1["d"])
    orc = O.Sim(cfg, tables, cap=cfg.capacity)
    orc.load(*parts)
    orc.prologue()
    for _ in range(C1["steps"]):
        orc.step()
    return parts, orc


def c1_gpu(precision, parts):
    sim = Sim(c1_cfg(precision))
    sim.load(*parts)
    sim.step(C1["steps"])
    out = (sim.read(), sim.fields(), sim.diag())
    sim.close()
    return out


def test_c1_full_size_fp64_matches_oracle(c1_oracle):
    """C1 at full size for 500 steps: the FP64 form and the oracle keep the
    same population and event counts, and agree to 1e-12 (particles: max
    |a - b| / max |b| per component; fields likewise)."""
    parts, orc = c1_oracle
    got, flds, dg = c1_gpu(_lib.FP64, parts)
    ion, ela, exc, nul, lost, ovf = orc.counters
    assert (dg["n_ionizations"], dg["n_elastic"], dg["n_excitation"], dg["n_null"],
            dg["n_lost_wall"]) == (ion, ela, exc, nul, lost)
    assert ion > 500
    r, z, ur, ut, uz, ids, alive = orc.state_rz()
    a = alive.astype(bool)
    ga = got["r"] >= 0
    assert set(got["id"][ga].tolist()) == set(ids[a].tolist())
    want = by_id(ids[a], r[a], z[a], ur[a], ut[a], uz[a])
    have = by_id(got["id"][ga], got["r"][ga], got["z"][ga], got["ur"][ga], got["ut"][ga],
                 got["uz"][ga])
    for h, w, k in zip(have, want, ("r", "z", "ur", "ut", "uz")):
        close(h, w, 1e-12, k)
    for g, w, k in zip(flds, (orc.Er, orc.Ez, orc.H), ("Er", "Ez", "H")):
        close(g, w, 1e-12, k)


def test_c1_full_size_fp32_product_against_oracle(c1_oracle):
    """The FP32 split form (the product) against the FP64 oracle directly, C1
    at full size for 500 steps: ionization yield within 0.5%, fields within
    1e-4 (||F32 - F64||_2 / ||F64||_2, worst of Er, Ez, H; the max-abs form
    within 1e-3), and the electron energy distribution (40 log bins from 0.1
    eV to 10 keV) and the mean energy within 3 sigma of their Monte Carlo
    error."""
    parts, orc = c1_oracle
    got, flds, dg = c1_gpu(_lib.FP32_SPLIT, parts)
    ion = int(orc.counters[0])
    assert ion > 500
    assert abs(dg["n_ionizations"] - ion) <= 0.005 * ion, (dg["n_ionizations"], ion)
    for g, w, k in zip(flds, (orc.Er, orc.Ez, orc.H), ("Er", "Ez", "H")):
        assert np.linalg.norm(g - w) <= 1e-4 * np.linalg.norm(w), k
        close(g, w, 1e-3, k)
    me, c, qe = 9.1093837015e-31, 299792458.0, 1.602176634e-19

    def energies(ur, ut, uz):
        u2 = (ur ** 2 + ut ** 2 + uz ** 2) / c ** 2
        return me * c * c * (u2 / (np.sqrt(1 + u2) + 1)) / qe

    r, z, ur, ut, uz, ids, alive = orc.state_rz()
    a = alive.astype(bool)
    ga = got["r"] >= 0
    E64 = energies(ur[a], ut[a], uz[a])
    E32 = energies(got["ur"][ga], got["ut"][ga], got["uz"][ga])
    assert abs(len(E32) - len(E64)) <= 0.005 * len(E64)
    bins = np.logspace(-1, 4, 41)
    h64, _ = np.histogram(E64, bins)
    h32, _ = np.histogram(E32, bins)
    assert np.all(np.abs(h32 - h64) <= 3 * np.sqrt(h64 + 1) + 1)
    assert abs(E32.mean() - E64.mean()) <= 3 * E64.std() / np.sqrt(len(E64))


def test_fp32_energy_distribution_within_3_sigma_of_fp64():
    """Free-running 60 steps at 100 Torr: the electron energy distribution of
    the FP32 split form (40 log-spaced bins from 0.1 eV to 10 keV), its mean
    energy and the ionization yield agree with the FP64 form's within 3 sigma
    of the Monte Carlo error of a bin (sqrt of its count)."""
    me, c, qe = 9.1093837015e-31, 299792458.0, 1.602176634e-19
    res = {}
    for prec in (_lib.FP64, _lib.FP32_SPLIT):
        cfg, sim, _, _ = start(prec, n_photo=4000, sort_period=5, torr=100.0)
        sim.step(60)
        d = sim.read()
        a = d["r"] >= 0
        u2 = (d["ur"][a] ** 2 + d["ut"][a] ** 2 + d["uz"][a] ** 2) / c ** 2
        E = me * c * c * (u2 / (np.sqrt(1 + u2) + 1)) / qe
        res[prec] = (E, sim.diag()["n_ionizations"])
        sim.close()
    (E64, i64), (E32, i32) = res[_lib.FP64], res[_lib.FP32_SPLIT]
    bins = np.logspace(-1, 4, 41)
    h64, _ = np.histogram(E64, bins)
    h32, _ = np.histogram(E32, bins)
    assert h64.sum() > 5000
    assert np.all(np.abs(h32 - h64) <= 3 * np.sqrt(h64 + 1) + 1)
    assert abs(E32.mean() - E64.mean()) <= 3 * E64.std() / np.sqrt(len(E64))
    assert abs(i32 - i64) <= 3 * np.sqrt(i64) + 1


@pytest.mark.parametrize("ratio", [2, 3])
def test_field_subcycle_ratio_matches_oracle(tables, ratio):
    """fdtd_ratio > 1 (ratio field sub-cycles of dt/ratio per particle step,
    the general fused field kernel): the FP64 form against the oracle, and the
    FP32 form (whose gather quads that kernel then writes value by value)
    against the FP64 form."""
    out = {}
    for prec in (_lib.FP64, _lib.FP32_SPLIT):
        cfg = config(NR, NZ, D, 1e-14, 300.0, precision=prec, capacity=40000, seed=7,
                     sort_period=0, fdtd_ratio=ratio)
        parts = births(2000, 8.0, NZ * D, seed=3, sigma_r=30e-6, Rp=NR * D)
        Er, Ez, H = grid_fields(NR, NZ, np.random.default_rng(8), E0=3e6, H0=2e3)
        Er[:, 0] = 0; Er[:, -1] = 0; Ez[-1, :] = 0
        sim = Sim(cfg)
        sim.load(*parts)
        sim.set_fields(Er, Ez, H)
        sim.step(4)
        out[prec] = (sim.fields(), sim.diag(), cfg, parts, (Er, Ez, H))
        sim.close()
    f64, d64, cfg, parts, flds = out[_lib.FP64]
    orc = oracle_run(cfg, tables, parts, flds, 4)
    for g, w, k in zip(f64, (orc.Er, orc.Ez, orc.H), ("Er", "Ez", "H")):
        close(g, w, 1e-12, k)
    assert d64["n_ionizations"] == orc.counters[0]
    f32, d32 = out[_lib.FP32_SPLIT][:2]
    for g, w, k in zip(f32, f64, ("Er", "Ez", "H")):
        assert np.linalg.norm(g - w) <= 1e-4 * np.linalg.norm(w), k
    assert abs(d32["n_ionizations"] - d64["n_ionizations"]) <= 2


@pytest.mark.parametrize("precision", [_lib.FP64, _lib.FP32_SPLIT])
def test_fields_set_between_steps(tables, precision):
    """Fields replaced after two steps (the FP32 form must rebuild its gather
    quads from them): the FP64 form follows the oracle, the FP32 form the
    FP64 form."""
    out = {}
    for prec in (_lib.FP64, precision):
        cfg, sim, parts, flds = start(prec)
        sim.step(2)
        F2 = grid_fields(NR, NZ, np.random.default_rng(21), E0=2e6, H0=3e3)
        F2[0][:, 0] = 0; F2[0][:, -1] = 0; F2[1][-1, :] = 0
        sim.set_fields(*F2)
        sim.step(3)
        out[prec] = (sim.fields(), sim.diag()["n_ionizations"])
        sim.close()
    orc = O.Sim(cfg, tables, cap=cfg.capacity)
    orc.load(*parts)
    orc.Er[:], orc.Ez[:], orc.H[:] = flds
    orc.prologue()
    for _ in range(2):
        orc.step()
    orc.Er[:], orc.Ez[:], orc.H[:] = F2
    for _ in range(3):
        orc.step()
    f64, i64 = out[_lib.FP64]
    for g, w, k in zip(f64, (orc.Er, orc.Ez, orc.H), ("Er", "Ez", "H")):
        close(g, w, 1e-12, k)
    assert i64 == orc.counters[0]
    f, i = out[precision]
    for g, w, k in zip(f, f64, ("Er", "Ez", "H")):
        assert np.linalg.norm(g - w) <= 1e-4 * np.linalg.norm(w), k
    assert abs(i - i64) <= 2


@pytest.mark.parametrize("precision", [_lib.FP64, _lib.FP32_SPLIT])
def test_sort_orders_by_deposit_quad_and_drops_the_dead(precision):
    """The counting sort (runs of equal keys found with a shuffle and ballots,
    per-run slot claims, the single-pass scan): after it the slots hold only
    live electrons, in non-decreasing deposit-quad key (the cell shifted by
    half a cell), each electron exactly once.  A dense population (most
    electrons in a few cells: long runs of equal keys) with wall losses
    (dead slots between them), loaded in random order."""
    cfg = config(NR, NZ, D, 1e-14, 300.0, precision=precision, capacity=60000, seed=9,
                 sort_period=0)
    # a dense core on the axis, and a spread population whose outer part
    # crosses the wall within the 40 steps
    dense = births(8000, 8.0, NZ * D, seed=4, sigma_r=D, Rp=NR * D)
    wide = births(4000, 8.0, NZ * D, seed=5, sigma_r=NR * D, Rp=NR * D, id_base=1 << 40)
    r, z, ur, ut, uz, ids = (np.concatenate([a, b]) for a, b in zip(dense, wide))
    perm = np.random.default_rng(2).permutation(len(r))
    sim = Sim(cfg)
    sim.load(*(a[perm] for a in (r, z, ur, ut, uz, ids)))
    sim.step(40)                          # wall losses leave dead slots
    before = sim.read()
    live_ids = np.sort(before["id"][before["r"] >= 0])
    d0 = sim.diag()
    sim.sort()
    got = sim.read()
    d1 = sim.diag()
    sim.close()
    assert d0["n_lost_wall"] > 0 and d0["n_total"] > d0["n_alive"]
    assert len(got["r"]) == d1["n_alive"] == d0["n_alive"] and np.all(got["r"] >= 0)
    assert np.array_equal(np.sort(got["id"]), live_ids)
    ar = np.clip(np.floor(got["r"] / D - 0.5).astype(np.int64) + 1, 0, NR)
    az = np.clip(np.floor(got["z"] / D - 0.5).astype(np.int64) + 1, 0, NZ)
    key = ar + az * (NR + 1)
    assert np.all(np.diff(key) >= 0)
    assert np.max(np.bincount(key)) > 64        # runs longer than a warp

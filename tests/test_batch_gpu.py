"""Batched instances: several gas cells of uneven size, pressure and precision
advanced together give bit-for-bit what each gives alone."""
import numpy as np
import pytest

from gasatt import _lib
from gasatt.dropin import Context
from gasatt.sim import Batch, Sim, births, config

pytestmark = pytest.mark.gpu

CELLS = [  # n_r, n_z, delta, torr, photoionizations, photon keV, precision, seed
    (32, 64, 5e-6, 300.0, 2000, 8.0, _lib.FP32_SPLIT, 1),
    (48, 128, 10e-6, 30.0, 5000, 12.0, _lib.FP32_SPLIT, 2),
    (16, 96, 5e-6, 100.0, 800, 5.0, _lib.FP64, 3),
    (64, 64, 5e-6, 3.0, 3000, 20.0, _lib.FP32_SPLIT, 4),
]
SORT_PERIOD = 3


def make(ctx, cell):
    nr, nz, d, torr, photo, kev, prec, seed = cell
    cfg = config(nr, nz, d, 1e-14, torr, precision=prec, capacity=8 * photo, seed=seed,
                 sort_period=SORT_PERIOD)
    sim = Sim(cfg, ctx=ctx)
    sim.load(*births(photo, kev, nz * d, seed=seed, sigma_r=nr * d / 4, Rp=nr * d))
    return sim


def snapshot(sim):
    st = sim.read()
    o = np.argsort(st["id"], kind="stable")
    d = sim.diag()
    return ({k: v[o] for k, v in st.items()}, sim.fields(), sim.current(),
            (d["n_ionizations"], d["n_elastic"], d["n_excitation"], d["n_alive"]))


def test_batch_equals_instances_alone():
    ctx = Context(0)
    alone = []
    for cell in CELLS:
        sim = make(ctx, cell)
        sim.step(5)
        sim.step(7)
        alone.append(snapshot(sim))
        sim.close()
    sims = [make(ctx, cell) for cell in CELLS]
    batch = Batch(sims, sort_period=SORT_PERIOD)
    batch.step(5)
    batch.step(7)
    for sim, ref in zip(sims, alone):
        got = snapshot(sim)
        for k in ref[0]:
            np.testing.assert_array_equal(got[0][k], ref[0][k], err_msg=k)
        for a, b in zip(got[1] + got[2], ref[1] + ref[2]):
            np.testing.assert_array_equal(a, b)
        assert got[3] == ref[3]
    assert sum(r[3][0] for r in alone) > 50             # collisions did happen
    batch.close()
    for s in sims:
        s.close()
    ctx.close()


def test_batch_with_ions_and_gas_maps_equals_instances_alone():
    """Cells with the ion species (pushes every 4 steps) and per-cell gas maps
    give in a batch what they give alone: fields, counts and the ions."""
    ctx = Context(0)

    def make_ionic(cell):
        nr, nz, d, torr, photo, kev, prec, seed = cell
        cfg = config(nr, nz, d, 1e-14, torr, precision=prec, capacity=8 * photo, seed=seed,
                     sort_period=SORT_PERIOD, ion_capacity=8 * photo, ion_subcycle=4)
        sim = Sim(cfg, ctx=ctx)
        sim.load(*births(photo, kev, nz * d, seed=seed, sigma_r=nr * d / 4, Rp=nr * d))
        sim.set_gas_density(cfg.gas_density * np.outer(np.linspace(1.5, 0.5, nr), np.ones(nz)))
        return sim

    def ions(sim):
        st = sim.read_ions()
        o = np.argsort(st["id"], kind="stable")
        return {k: v[o] for k, v in st.items()}

    cells = CELLS[:3]
    alone = []
    for cell in cells:
        sim = make_ionic(cell)
        sim.step(11)
        alone.append((snapshot(sim), ions(sim)))
        sim.close()
    sims = [make_ionic(cell) for cell in cells]
    batch = Batch(sims, sort_period=SORT_PERIOD)
    batch.step(11)
    for sim, (ref, ref_ions) in zip(sims, alone):
        got = snapshot(sim)
        for a, b in zip(got[1] + got[2], ref[1] + ref[2]):
            np.testing.assert_array_equal(a, b)
        assert got[3] == ref[3]
        gi = ions(sim)
        for k in ref_ions:
            np.testing.assert_array_equal(gi[k], ref_ions[k], err_msg=k)
    assert sum(len(r[1]["id"]) for r in alone) > 20
    batch.close()
    for s in sims:
        s.close()


def test_batch_groups_share_launches_and_keep_cells_exact():
    """Twelve FP32 cells of uneven grids and populations, four FP64 cells and
    one cell with a field sub-cycle of 2 (which fits no group and keeps its own
    step graph): each batch step launches the group kernels once per group
    (FP32: field update + pass; FP64: commit, collisions, field update, pass)
    plus the odd cell's own, and every cell ends bit for bit where it ends
    alone."""
    rng = np.random.default_rng(5)
    cells = []
    for i in range(16):
        nr, nz = [(16, 48), (32, 64), (24, 120), (48, 96)][i % 4]
        cells.append((nr, nz, 5e-6, float(10 ** rng.uniform(0.5, 2.5)), int(rng.integers(300, 3000)),
                      float(rng.uniform(3, 15)), _lib.FP32_SPLIT if i < 12 else _lib.FP64, 100 + i))
    ctx = Context(0)

    def make_any(cell, ratio=1):
        nr, nz, d, torr, photo, kev, prec, seed = cell
        cfg = config(nr, nz, d, 1e-14, torr, precision=prec, capacity=8 * photo, seed=seed,
                     sort_period=50, fdtd_ratio=ratio)
        sim = Sim(cfg, ctx=ctx)
        sim.load(*births(photo, kev, nz * d, seed=seed, sigma_r=nr * d / 4, Rp=nr * d))
        return sim

    odd = (32, 64, 5e-6, 50.0, 1500, 8.0, _lib.FP32_SPLIT, 99)
    alone = []
    for cell in cells:
        sim = make_any(cell)
        sim.step(9)
        alone.append(snapshot(sim))
        sim.close()
    sim = make_any(odd, 2)
    sim.step(9)
    alone.append(snapshot(sim))
    sim.close()
    sims = [make_any(c) for c in cells] + [make_any(odd, 2)]
    batch = Batch(sims, sort_period=50)
    batch.step(1)                                    # primes and sorts every cell
    l0 = ctx.launches
    batch.step(8)
    assert ctx.launches - l0 == 8 * (2 + 4 + 2)      # FP32 group, FP64 group, the odd cell
    for sim, ref in zip(sims, alone):
        got = snapshot(sim)
        for a, b in zip(got[1] + got[2], ref[1] + ref[2]):
            np.testing.assert_array_equal(a, b)
        assert got[3] == ref[3]
        for k in ref[0]:
            np.testing.assert_array_equal(got[0][k], ref[0][k], err_msg=k)
    assert sum(r[3][0] for r in alone) > 100
    batch.close()
    for s in sims:
        s.close()
    ctx.close()


def test_batch_sort_flushes_each_group_in_one_launch():
    """Six FP32 and two FP64 cells sorting every 4 steps: before each sort of
    all cells, each group applies its cells' pending collisions with one
    kernel (FP32: k_batch_collide32; FP64: the commits and k_batch_mcc64) and
    one queue clear, not a launch per cell; every cell still ends bit for bit
    where it ends alone."""
    rng = np.random.default_rng(9)
    cells = []
    for i in range(8):
        nr, nz = [(16, 48), (32, 64), (24, 120), (48, 96)][i % 4]
        cells.append((nr, nz, 5e-6, float(10 ** rng.uniform(1.5, 2.5)), int(rng.integers(500, 3000)),
                      float(rng.uniform(3, 15)), _lib.FP32_SPLIT if i < 6 else _lib.FP64, 200 + i))
    ctx = Context(0)

    def make_any(cell):
        nr, nz, d, torr, photo, kev, prec, seed = cell
        cfg = config(nr, nz, d, 1e-14, torr, precision=prec, capacity=8 * photo, seed=seed,
                     sort_period=4)
        sim = Sim(cfg, ctx=ctx)
        sim.load(*births(photo, kev, nz * d, seed=seed, sigma_r=nr * d / 4, Rp=nr * d))
        return sim

    alone = []
    for cell in cells:
        sim = make_any(cell)
        sim.step(9)
        alone.append(snapshot(sim))
        sim.close()
    sims = [make_any(c) for c in cells]
    batch = Batch(sims, sort_period=4)
    batch.step(1)                                    # primes and sorts every cell
    l0 = ctx.launches
    batch.step(8)                                    # all cells sort before steps 5 and 9
    per_step = 2 + 4                                 # FP32 group, FP64 group
    per_sort = (2 + 3) + 4 * len(cells)              # group flushes, then every cell's sort
    assert ctx.launches - l0 == 8 * per_step + 2 * per_sort
    for sim, ref in zip(sims, alone):
        got = snapshot(sim)
        for a, b in zip(got[1] + got[2], ref[1] + ref[2]):
            np.testing.assert_array_equal(a, b)
        assert got[3] == ref[3]
        for k in ref[0]:
            np.testing.assert_array_equal(got[0][k], ref[0][k], err_msg=k)
    assert sum(r[3][0] for r in alone) > 50
    batch.close()
    for s in sims:
        s.close()
    ctx.close()


def test_batch_of_large_cells_equals_instances_alone():
    """Four 256 x 512 cells (FP32): alone, each field update fits in one wave
    of warps; batched, their 3,440 patches take several rounds per warp, so
    patches are staged after neighbouring tiles (of the same cell) were
    written.  Every cell still ends bit for bit where it ends alone."""
    cells = [(256, 512, 10e-6, float(t), 4000, 8.0, _lib.FP32_SPLIT, 300 + i)
             for i, t in enumerate((3.0, 10.0, 30.0, 100.0))]
    ctx = Context(0)
    alone = []
    for cell in cells:
        sim = make(ctx, cell)
        sim.step(10)
        alone.append(snapshot(sim))
        sim.close()
    sims = [make(ctx, cell) for cell in cells]
    batch = Batch(sims, sort_period=SORT_PERIOD)
    batch.step(10)
    for sim, ref in zip(sims, alone):
        got = snapshot(sim)
        for a, b in zip(got[1] + got[2], ref[1] + ref[2]):
            np.testing.assert_array_equal(a, b)
        assert got[3] == ref[3]
        for k in ref[0]:
            np.testing.assert_array_equal(got[0][k], ref[0][k], err_msg=k)
    batch.close()
    for s in sims:
        s.close()
    ctx.close()

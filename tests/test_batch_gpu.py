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

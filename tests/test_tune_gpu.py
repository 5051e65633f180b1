"""The sort-period autotuner: it times every candidate on a fresh copy of the
population and returns the fastest (results do not depend on the period; see
test_sim_gpu.test_bit_exact_run_to_run_and_sort_invariant)."""
import pytest

from gasatt import _lib
from gasatt.sim import births, config
from gasatt.tune import tune_sort_period

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [_lib.FP64, _lib.FP32_SPLIT])
def test_tune_sort_period_returns_the_fastest_candidate(precision):
    cfg = config(32, 64, 5e-6, 1e-14, 300.0, precision=precision, capacity=40000, seed=7)
    parts = births(2000, 8.0, 64 * 5e-6, seed=3, sigma_r=30e-6, Rp=32 * 5e-6)
    best, table = tune_sort_period(cfg, parts, candidates=(2, 5, 50), steps=30)
    assert set(table) == {2, 5, 50}
    assert all(v > 0 for v in table.values())
    assert best in table and table[best] == min(table.values())
    assert cfg.sort_period == 20            # the caller's config is left alone


@pytest.mark.parametrize("precision", [_lib.FP64, _lib.FP32_SPLIT])
def test_tune_every_knob_by_coordinate_descent(precision):
    """tune() times every candidate of every knob (field patch rows, FP32
    chunk size, sort period) and keeps the fastest of each."""
    from gasatt.tune import knob_candidates, tune
    cfg = config(48, 200, 5e-6, 1e-14, 300.0, precision=precision, capacity=60000, seed=7)
    parts = births(6000, 8.0, 200 * 5e-6, seed=3, sigma_r=40e-6, Rp=48 * 5e-6)
    knobs = knob_candidates(cfg)
    if precision == _lib.FP32_SPLIT:
        assert set(knobs) == {"fdtd_tile_rows", "pass_chunk", "gather", "sort_period"}
    else:
        assert set(knobs) == {"fdtd_tile_rows", "sort_period"}
    assert set(knobs["fdtd_tile_rows"]) == {12, 16, 20}
    best, table = tune(cfg, parts, steps=20)
    for name, cands in knobs.items():
        assert set(table[name]) == set(cands)
        assert getattr(best, name) == min(table[name], key=table[name].get)
    assert cfg.fdtd_tile_rows == 0 and cfg.pass_chunk == 0 and cfg.gather == 0
    assert cfg.sort_period == 20


@pytest.mark.parametrize("precision", [_lib.FP64, _lib.FP32_SPLIT])
def test_launch_knobs_leave_results_bit_identical(precision):
    """The tuned knobs change only launch shapes: fields, currents and event
    counts are the same bits for every patch height, chunk size and gather
    source (quads or the fields themselves)."""
    import numpy as np
    from _cases import grid_fields
    from gasatt.sim import Sim
    outs = []
    shapes = [(12, 256, 1), (16, 1792, 2), (20, 1024, 1), (16, 512, 2)]
    for rows, chunk, gather in shapes:
        cfg = config(40, 150, 5e-6, 1e-14, 300.0, precision=precision, capacity=60000, seed=7,
                     sort_period=7)
        cfg.fdtd_tile_rows, cfg.pass_chunk, cfg.gather = rows, chunk, gather
        sim = Sim(cfg)
        sim.load(*births(5000, 8.0, 150 * 5e-6, seed=3, sigma_r=40e-6, Rp=40 * 5e-6))
        Er, Ez, H = grid_fields(40, 150, np.random.default_rng(4), E0=3e6, H0=2e3)
        Er[:, 0] = 0; Er[:, -1] = 0; Ez[-1, :] = 0
        sim.set_fields(Er, Ez, H)
        sim.step(12)
        d = sim.diag()
        outs.append((*sim.fields(), *sim.current(), d["n_ionizations"], d["n_alive"],
                     d["status_flags"]))
        sim.close()
    for o in outs[1:]:
        for a, b in zip(outs[0], o):
            assert np.array_equal(a, b)
    assert outs[0][-1] == 0


def test_bad_launch_knobs_are_rejected():
    from gasatt._lib import GasattError
    from gasatt.sim import Sim
    for prec, rows, chunk in ((_lib.FP32_SPLIT, 40, 0), (_lib.FP32_SPLIT, 8, 0),
                              (_lib.FP64, 24, 0), (_lib.FP32_SPLIT, 0, 300),
                              (_lib.FP32_SPLIT, 0, 2048), (_lib.FP32_SPLIT, 0, -3)):
        cfg = config(32, 64, 5e-6, 1e-14, 1.0, precision=prec, capacity=1000)
        if chunk == -3:
            cfg.gather, chunk = 3, 0
        cfg.fdtd_tile_rows, cfg.pass_chunk = rows, chunk
        with pytest.raises(GasattError):
            Sim(cfg)

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

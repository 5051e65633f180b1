"""Live pinning on a GPU: the reference's own kernels (oracle/_ref) against the
CPU oracle on fresh seeded inputs."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))

import make_golden as G  # noqa: E402
import pyoracle as O  # noqa: E402
from _refcheck import assert_em_match, assert_mcc_match, oracle_em, oracle_mcc  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    if not O.RefKernels.available():
        pytest.skip("oracle/_ref not built (needs the reference sources at build time)")
    return O.RefKernels()


@pytest.mark.parametrize("seed", [21, 22])
def test_em_kernels_pin_oracle(ref, seed):
    cs = G.em_case(seed=seed, n=3000)
    assert_em_match(oracle_em(cs), G.run_em_reference(ref, cs))


@pytest.mark.parametrize("seed", [31, 32])
def test_electron_transport_pins_oracle(ref, tables, seed):
    cs = G.mcc_case(seed=seed, n=6000)
    nion, nexc = assert_mcc_match(oracle_mcc(cs, tables), G.run_mcc_reference(ref, cs), cs)
    assert nion > 100 and nexc > 100

"""The CPU oracle against outputs of the reference's own CUDA kernels
(golden files written by tests/golden/make_golden.py on a GPU)."""
import os

import numpy as np
import pytest

from _refcheck import assert_em_match, assert_mcc_match, oracle_em, oracle_mcc

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    path = os.path.join(GOLD, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated yet")
    z = np.load(path)
    cs = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    ref = {k: z[k] for k in z.files if not k.startswith("in_")}
    return cs, ref


def test_oracle_matches_reference_em_kernels():
    cs, ref = load("ref_em_kernels.npz")
    assert_em_match(oracle_em(cs), ref)


def test_oracle_matches_reference_electron_transport(tables):
    cs, ref = load("ref_electron_transport.npz")
    nion, nexc = assert_mcc_match(oracle_mcc(cs, tables), ref, cs)
    assert nion > 100 and nexc > 100

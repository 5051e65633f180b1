"""Photoionization births drawn on the GPU follow the workload's laws: exact
photoelectron and Auger speeds, dipole (photoelectron) and isotropic (Auger)
directions, Rayleigh radius, uniform z; pairs share their birth point; ids
and draws are reproducible."""
import numpy as np
import pytest

from gasatt import _lib
from gasatt.sim import AUGER_EV, K_SHELL_EV, Sim, config, u_of_energy_ev

pytestmark = pytest.mark.gpu

N, KEV, SIGMA, NR, NZ, D = 200_000, 8.0, 50e-6, 256, 1024, 5e-6


def born(precision, seed):
    cfg = config(NR, NZ, D, 1e-14, 1.0, precision=precision, capacity=2 * N + 1000, seed=1)
    sim = Sim(cfg)
    sim.birth_photo(N, KEV, seed=seed, sigma_r=SIGMA, id_base=100)
    st = sim.read()
    return sim, st


@pytest.mark.parametrize("precision", [_lib.FP64, _lib.FP32_SPLIT])
def test_gpu_births_follow_the_laws(precision):
    sim, st = born(precision, seed=11)
    o = np.argsort(st["id"])
    st = {k: v[o] for k, v in st.items()}
    np.testing.assert_array_equal(st["id"], np.arange(2 * N, dtype=np.uint64) + 100)
    rtol = 1e-12 if precision == _lib.FP64 else 2e-7
    u = np.sqrt(st["ur"] ** 2 + st["ut"] ** 2 + st["uz"] ** 2)
    pe, au = slice(0, None, 2), slice(1, None, 2)
    np.testing.assert_allclose(u[pe], u_of_energy_ev(KEV * 1000 - K_SHELL_EV), rtol=rtol)
    np.testing.assert_allclose(u[au], u_of_energy_ev(AUGER_EV), rtol=rtol)
    # direction moments in the local frame (azimuth-averaged): photoelectron
    # <dz^2> = (1 - <mu^2>) / 2 = 0.2, <dr^2> = <dt^2> = 0.4; Auger 1/3 each
    for sl, want in ((pe, (0.4, 0.4, 0.2)), (au, (1 / 3, 1 / 3, 1 / 3))):
        for comp, w in zip(("ur", "ut", "uz"), want):
            assert abs(np.mean((st[comp][sl] / u[sl]) ** 2) - w) < 5e-3, comp
    # the pair of a photon shares its birth point
    np.testing.assert_allclose(st["r"][pe], st["r"][au], rtol=rtol, atol=1e-15)
    np.testing.assert_allclose(st["z"][pe], st["z"][au], rtol=rtol, atol=1e-15)
    r, z = st["r"][pe], st["z"][pe]
    assert np.all(r >= 0) and np.all(r < NR * D)
    assert abs(np.mean(r ** 2) / (2 * SIGMA ** 2) - 1) < 0.01           # Rayleigh <r^2> = 2 sigma^2
    assert np.all(z >= 0) and np.all(z < NZ * D)
    assert abs(np.mean(z) / (NZ * D) - 0.5) < 0.005
    sim.step(3)                                                          # and they move
    assert sim.diag()["n_alive"] > 0
    sim.close()


def test_gpu_births_reproducible():
    a = born(_lib.FP32_SPLIT, seed=5)
    b = born(_lib.FP32_SPLIT, seed=5)
    c = born(_lib.FP32_SPLIT, seed=6)
    for k in ("r", "z", "ur", "ut", "uz", "id"):
        np.testing.assert_array_equal(a[1][k], b[1][k])
    assert not np.array_equal(a[1]["z"], c[1]["z"])
    for x in (a, b, c):
        x[0].close()

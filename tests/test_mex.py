"""The MATLAB MEX gateway (gas-atenuator_b200/mex/gasatt_mex.c), run without
MATLAB on a stand-in MX/mxGPUArray runtime (tests/mexshim).

CPU: the gateway builds, links libgasatt and turns bad calls into MATLAB
errors.  GPU: every command gives what the same call through the Python
mirror of the C ABI gives, bit for bit."""
import ctypes
import os
import subprocess

import numpy as np
import pytest
import torch

from conftest import ROOT, has_gpu

SHIM = os.path.join(ROOT, "tests", "mexshim")
c_p, c_sz, c_i = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int


class MexError(RuntimeError):
    pass


class Mex:
    """mexFunction driven through the stand-in runtime; MATLAB values are
    numpy arrays (column-major m x n), gpuArrays are wrapped with .gpu()."""

    def __init__(self):
        subprocess.run(["make", "-s", "-C", SHIM], check=True)
        lib = ctypes.CDLL(os.path.join(SHIM, "_build", "libgasatt_mex_shim.so"))
        for name, res, args in (
                ("fx_double", c_p, [c_sz, c_sz, c_p]), ("fx_uint64", c_p, [c_sz, c_sz, c_p]),
                ("fx_string", c_p, [ctypes.c_char_p]), ("fx_gpu", c_p, [c_sz, c_sz, c_p]),
                ("fx_struct", c_p, [c_i, c_p, c_p]), ("fx_call", c_i, [c_i, c_p, c_i, c_p]),
                ("fx_error", ctypes.c_char_p, []), ("fx_rows", c_sz, [c_p]),
                ("fx_cols", c_sz, [c_p]), ("fx_is_gpu", c_i, [c_p]), ("fx_class", c_i, [c_p]),
                ("fx_read", c_i, [c_p, c_p]), ("fx_field", c_p, [c_p, ctypes.c_char_p]),
                ("fx_exit", None, [])):
            f = getattr(lib, name)
            f.restype, f.argtypes = res, args
        self.lib = lib

    @staticmethod
    def _mat(a, dtype):
        a = np.asarray(a, dtype=dtype)
        a = a.reshape(-1, 1) if a.ndim < 2 else a
        return a.shape[0], a.shape[1], np.asfortranarray(a)

    def arg(self, v):
        if isinstance(v, Mx):
            return v.p
        if isinstance(v, Gpu):
            m, n, a = self._mat(v.a, np.float64)
            return self.lib.fx_gpu(m, n, a.ctypes.data_as(c_p))
        if isinstance(v, str):
            return self.lib.fx_string(v.encode())
        if isinstance(v, dict):
            names = (ctypes.c_char_p * len(v))(*[k.encode() for k in v])
            vals = (c_p * len(v))(*[self.arg(x) for x in v.values()])
            return self.lib.fx_struct(len(v), ctypes.cast(names, c_p), ctypes.cast(vals, c_p))
        a = np.asarray(v)
        if a.dtype == np.uint64:
            m, n, a = self._mat(a, np.uint64)
            return self.lib.fx_uint64(m, n, a.ctypes.data_as(c_p))
        m, n, a = self._mat(a, np.float64)
        return self.lib.fx_double(m, n, a.ctypes.data_as(c_p))

    def value(self, p):
        p = p.p if isinstance(p, Mx) else p
        m, n = self.lib.fx_rows(p), self.lib.fx_cols(p)
        dt = np.uint64 if self.lib.fx_class(p) == 15 else np.float64
        out = np.zeros(m * n, dtype=dt)
        assert self.lib.fx_read(p, out.ctypes.data_as(c_p)) == 0
        return out.reshape((m, n), order="F")

    def field(self, p, name):
        p = p.p if isinstance(p, Mx) else p
        return self.value(self.lib.fx_field(p, name.encode()))[0, 0]

    def call(self, nout, *args):
        prhs = (c_p * len(args))(*[self.arg(a) for a in args])
        plhs = (c_p * max(nout, 1))()
        if self.lib.fx_call(nout, ctypes.cast(plhs, c_p), len(args), ctypes.cast(prhs, c_p)):
            raise MexError(self.lib.fx_error().decode())
        return [Mx(plhs[k]) for k in range(nout)]


class Gpu:
    def __init__(self, a):
        self.a = np.asarray(a, dtype=np.float64)


class Mx:
    """An mxArray the gateway returned; passed back as it is."""

    def __init__(self, p):
        self.p = p


@pytest.fixture(scope="module")
def mex():
    m = Mex()
    yield m
    m.lib.fx_exit()


def register_tables(mex, tables):
    mex.call(0, "tables", *[tables[k] for k in ("t_el", "t_sel", "t_sel_1", "t_del", "t_sdel",
                                                "t_ion", "t_exc")])


def test_gateway_turns_bad_calls_into_matlab_errors(mex, tables):
    with pytest.raises(MexError, match="command name"):
        mex.call(0)
    with pytest.raises(MexError, match="unknown command"):
        mex.call(0, "electricmagneticfield7")
    with pytest.raises(MexError, match="tables"):
        mex.call(0, "tables", tables["t_el"])
    register_tables(mex, tables)                          # host-only: works without a GPU


@pytest.mark.gpu
@pytest.mark.parametrize("ncell", [0.0, -3.0, 2.5])
def test_gateway_rejects_a_bad_cell_count_before_allocating(mex, ncell):
    """particle_density's ncell is checked before the gateway asks MATLAB for
    the output gpuArray."""
    g = Gpu([1.0])
    with pytest.raises(MexError, match="ncell must be a positive integer"):
        mex.call(1, "particle_density", 1.0, 1.0, g, g, g, g, 1.0, g, g, 1.0, ncell)


@pytest.mark.skipif(has_gpu(), reason="checks the error path of a machine without a GPU")
def test_gateway_reports_a_missing_gpu(mex, tables):
    register_tables(mex, tables)
    with pytest.raises(MexError, match=r"status 7"):
        mex.call(3, "find_CS0", tables["t_el"], tables["t_sel"], tables["t_ion"], tables["t_exc"],
                 Gpu([1.0, 2.0]))


# --------------------------------------------------------------------- GPU
def np_(t):
    return t.detach().cpu().numpy()


@pytest.mark.gpu
def test_mex_dropins_match_the_c_abi(mex, tables):
    import gasatt
    from test_dropin_gpu import emf6_inputs
    from _cases import cell_structure
    mex.call(0, "init", 0.0, 0.0)
    register_tables(mex, tables)
    # find_CS0
    E = np.exp(np.linspace(np.log(1e-3), np.log(20.0), 3000))
    got = mex.call(3, "find_CS0", tables["t_el"], tables["t_sel"], tables["t_ion"],
                   tables["t_exc"], Gpu(E))
    want = gasatt.find_CS0(tables["t_el"], tables["t_sel"], tables["t_ion"], tables["t_exc"],
                           torch.tensor(E))
    for g, w in zip(got, want):
        np.testing.assert_array_equal(mex.value(g).ravel(), np_(w))
    # free_motion
    rng = np.random.default_rng(4)
    a = [rng.normal(size=5000) * s for s in (1e7, 1e7, 1e7, 1e-3, 1e-3, 1e-2)]
    got = mex.call(5, "free_motion", *[Gpu(x) for x in a], 1e-12)
    want = gasatt.free_motion(*[torch.tensor(x) for x in a], 1e-12)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(mex.value(g).ravel(), np_(w))
    # REBOND
    n, PHIp, Lp = 4000, 0.1, 1e-2
    r = rng.uniform(1e-4, 5e-3, n); phi = rng.uniform(-2.2 * PHIp, 3.2 * PHIp, n)
    pos = np.stack([r * np.cos(phi), r * np.sin(phi), rng.uniform(-0.2 * Lp, 1.3 * Lp, n)], 1)
    vel = rng.normal(size=(n, 3)) * 1e7
    got = mex.call(3, "REBOND", Gpu(pos), Gpu(r), Gpu(phi), Gpu(vel), Lp, PHIp)
    want = gasatt.REBOND(torch.tensor(pos), torch.tensor(r), torch.tensor(phi), torch.tensor(vel),
                         Lp, PHIp)
    np.testing.assert_array_equal(mex.value(got[0]), np_(want[0]))
    np.testing.assert_array_equal(mex.value(got[1]), np_(want[1]))
    assert mex.value(got[2])[0, 0] == want[2]
    # particle_density (the gateway takes the no-allocation variant)
    PHIp, Rp, rmax, delta, zmax, dz = 0.1, 1e-2, 25, 4e-4, 6, 1e-2
    phimax, sum_cell, cellnumxy = cell_structure(PHIp, Rp, rmax, delta)
    dphi = PHIp / phimax
    VC = np.concatenate([[0.5 * ((i * delta)**2 - ((i - 1) * delta)**2) * dphi[i - 1] * dz]
                         * int(phimax[i - 1]) for i in range(1, rmax + 1)])
    r = rng.uniform(0, Rp, 50000); phi = rng.uniform(0, PHIp, 50000); z = rng.uniform(0, zmax * dz, 50000)
    got = mex.call(1, "particle_density", delta, dz, Gpu(dphi), Gpu(r), Gpu(phi), Gpu(z),
                   float(cellnumxy), Gpu(sum_cell), Gpu(VC), 3.0, float(cellnumxy * zmax))
    want = gasatt.particle_density(delta, dz, dphi, torch.tensor(r), torch.tensor(phi),
                                   torch.tensor(z), cellnumxy, sum_cell, VC, 3.0,
                                   ncell=cellnumxy * zmax)
    np.testing.assert_array_equal(mex.value(got[0]).ravel(), np_(want))
    got0 = mex.call(1, "particle_density0", delta, dz, Gpu(dphi), Gpu(np.stack([r, z, phi], 1)),
                    float(cellnumxy), Gpu(sum_cell), Gpu(VC), 3.0, float(cellnumxy * zmax))
    np.testing.assert_array_equal(mex.value(got0[0]).ravel(), np_(want))
    # electricmagneticfield6 (positions (r, phi, z) in, like the reference)
    cs = emf6_inputs(5)
    d, nr, nz, PHIp = cs["d"], cs["nr"], cs["nz"], cs["PHIp"]
    args = (cs["e"][0], cs["e"][1], cs["i1"][0], cs["i1"][1], cs["i2"][0], cs["i2"][1],
            cs["Er"], cs["Ez"], cs["H"])
    scal = (d, 1e-13, nr * d, nz * d, PHIp, 1e4, 20.0)
    got = mex.call(10, "electricmagneticfield6", *[Gpu(x) for x in args], *scal)
    want = gasatt.electricmagneticfield6(*[torch.tensor(x) for x in args], *scal[:-1], 20)
    assert mex.value(got[0]).shape[0] < len(cs["e"][0])        # wall losses removed rows
    for g, w in zip(got, want):
        np.testing.assert_array_equal(mex.value(g).reshape(np_(w).shape), np_(w))


@pytest.mark.gpu
def test_mex_electron_collision_matches_the_c_abi(mex, tables):
    """Philox draws keyed on (context seed, particle, call): a fresh gateway
    context and a fresh library context with the same seed agree."""
    import gasatt
    import pyoracle as O
    from gasatt import _lib
    from test_dropin_gpu import collision_inputs
    cs = collision_inputs(12, n=3000)
    se, si, sx = (np.nan_to_num(a, nan=0.0) for a in O.find_cs0(tables, cs["kin"], _lib.FAITHFUL))
    common = (tables["t_el"], tables["t_sel_1"], tables["t_del"], tables["t_sdel"], tables["t_exc"])
    mex.call(0, "init", 0.0, 0.0)
    register_tables(mex, tables)
    got = mex.call(4, "electron_collision", Gpu(cs["pos"]), Gpu(cs["vel"]), Gpu(cs["ion_pos"]),
                   Gpu(cs["ion_vel"]), *common, Gpu(cs["kin"]), cs["sum_cell"],
                   float(cs["cellnumxy"]), Gpu(cs["density"]), Gpu(cs["temperature"]), cs["PHIp"],
                   cs["phimax"], cs["dr"], cs["dz"], Gpu(se), Gpu(si), Gpu(sx), 2e-10)
    gasatt.dropin._ctx_cache.clear()                      # a fresh context, seed 0
    want = gasatt.electron_collision(
        torch.tensor(cs["pos"]), torch.tensor(cs["vel"]), torch.tensor(cs["ion_pos"]),
        torch.tensor(cs["ion_vel"]), *common, torch.tensor(cs["kin"]), cs["sum_cell"],
        cs["cellnumxy"], torch.tensor(cs["density"]), torch.tensor(cs["temperature"]), cs["PHIp"],
        cs["phimax"], cs["dr"], cs["dz"], torch.tensor(se), torch.tensor(si), torch.tensor(sx),
        2e-10)
    assert mex.value(got[0]).shape[0] > 3000               # secondaries appended
    for g, w in zip(got, want):
        np.testing.assert_array_equal(mex.value(g), np_(w))


@pytest.mark.gpu
def test_mex_resident_simulation_matches_the_python_api(mex, tables):
    from gasatt import _lib
    from gasatt.sim import Sim, births, config
    cfg = config(32, 64, 5e-6, 1e-14, 300.0, precision=_lib.FP32_SPLIT, capacity=40000, seed=7,
                 sort_period=5)
    parts = births(2000, 8.0, 64 * 5e-6, seed=3, sigma_r=30e-6, Rp=32 * 5e-6)
    register_tables(mex, tables)
    fields = {k: float(getattr(cfg, k)) for k, _ in type(cfg)._fields_}
    (h,) = mex.call(1, "sim_create", fields)
    mex.call(0, "sim_load", h, *parts[:5], np.asarray(parts[5], dtype=np.uint64))
    mex.call(0, "sim_step", h, 12.0)
    out = [mex.value(p).ravel() for p in mex.call(6, "sim_read", h)]
    (dg,) = mex.call(1, "sim_diag", h)
    mex.call(0, "sim_destroy", h)
    sim = Sim(cfg)
    sim.load(*parts)
    sim.step(12)
    want = sim.read()
    d = sim.diag()
    o_g, o_w = np.argsort(out[5]), np.argsort(want["id"])
    for k, g in zip(("r", "z", "ur", "ut", "uz", "id"), out):
        np.testing.assert_array_equal(g[o_g], want[k][o_w], err_msg=k)
    for k in ("n_alive", "n_ionizations", "n_elastic", "kinetic_ev", "field_energy_j"):
        assert mex.field(dg, k) == d[k], k


@pytest.mark.gpu
def test_mex_resident_fields_gas_ions_and_births(mex, tables):
    """The sim_* commands for GPU births, fields, a gas map and ions give what
    the Python API gives on the same sequence of calls."""
    from _cases import grid_fields
    from gasatt import _lib
    from gasatt.sim import Sim, config
    nr, nz, d = 32, 64, 5e-6
    cfg = config(nr, nz, d, 1e-14, 300.0, precision=_lib.FP64, capacity=40000, seed=9,
                 sort_period=5, ion_capacity=40000, ion_subcycle=5)
    Er, Ez, H = grid_fields(nr, nz, np.random.default_rng(2), E0=2e6, H0=1e3)
    Er[:, 0] = 0; Er[:, -1] = 0; Ez[-1, :] = 0
    rho = cfg.gas_density * np.outer(np.ones(nr), np.linspace(0.5, 1.5, nz))
    rng = np.random.default_rng(5)
    ions = (rng.uniform(10e-6, 100e-6, 50), rng.uniform(0, nz * d, 50), rng.normal(0, 300, 50),
            rng.normal(0, 300, 50), rng.normal(0, 300, 50), np.arange(50, dtype=np.uint64) + 7,
            rng.integers(1, 3, 50).astype(np.int8))
    register_tables(mex, tables)
    (h,) = mex.call(1, "sim_create", {k: float(getattr(cfg, k)) for k, _ in type(cfg)._fields_})
    mex.call(0, "sim_birth_photo", h, 1500.0, 8.0, 4.0, 30e-6)
    mex.call(0, "sim_set_fields", h, Er, Ez, H)
    mex.call(0, "sim_set_gas_density", h, rho)
    mex.call(0, "sim_load_ions", h, *ions[:5], ions[5], ions[6].astype(np.float64))
    mex.call(0, "sim_step", h, 12.0)
    f_mex = [mex.value(p) for p in mex.call(3, "sim_get_fields", h)]
    i_mex = [mex.value(p).ravel() for p in mex.call(7, "sim_read_ions", h)]
    (dg,) = mex.call(1, "sim_diag", h)
    mex.call(0, "sim_destroy", h)
    sim = Sim(cfg)
    sim.birth_photo(1500, 8.0, seed=4, sigma_r=30e-6)
    sim.set_fields(Er, Ez, H)
    sim.set_gas_density(rho)
    sim.load_ions(*ions[:6], charge=ions[6])
    sim.step(12)
    for g, w in zip(f_mex, sim.fields()):
        np.testing.assert_array_equal(g, w)
    iw = sim.read_ions()
    og, ow = np.argsort(i_mex[5]), np.argsort(iw["id"])
    for g, k in zip(i_mex, ("r", "z", "ur", "ut", "uz", "id", "charge")):
        np.testing.assert_array_equal(g[og], np.asarray(iw[k][ow], dtype=g.dtype), err_msg=k)
    d = sim.diag()
    for k in ("n_alive", "n_ionizations", "n_ions", "kinetic_ev", "wall_loss_ev"):
        assert mex.field(dg, k) == d[k], k
    assert d["n_ionizations"] > 0 and d["n_ions"] > 50

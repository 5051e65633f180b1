"""The resident field update (one warp per patch, TMA-staged, boundary rules
as per-column coefficients) at the edges of its tiling: grids smaller than
one patch, grids cut exactly at a tile edge and one past it, every patch
height, and each field quirk flag.  The FP64 form against the oracle, every
patch height bit-identical, the FP32 form (gather quads or direct field
loads, also bit-identical to each other) against the FP64 form."""
import numpy as np
import pytest

import pyoracle as O
from _cases import close, grid_fields
from gasatt import abi
from gasatt.sim import Sim, births, config

pytestmark = pytest.mark.gpu

D, DT, STEPS = 5e-6, 1e-14, 3
# (n_r, n_z): below one patch; 26 columns = one tile exactly and 27 one past
# it; rows cut at the 10-row tiles of 16-row patches and one past them
GRIDS = [(5, 7), (25, 9), (26, 10), (27, 11), (33, 41)]
FLAGS = [0, abi.Q_ER_END_COPY, abi.Q_EZ_AXIS_JSIGN, abi.Q_EZ_RSHIFT,
         abi.Q_ER_END_COPY | abi.Q_EZ_AXIS_JSIGN | abi.Q_EZ_RSHIFT]


def run(nr, nz, flags, precision, rows, gather=0):
    cfg = config(nr, nz, D, DT, 300.0, precision=precision, capacity=20000, seed=5,
                 sort_period=0, flags=flags)
    cfg.fdtd_tile_rows, cfg.gather = rows, gather
    # electrons near the axis, so that the axis column carries current
    parts = births(1500, 8.0, nz * D, seed=11, sigma_r=2 * D, Rp=nr * D)
    flds = grid_fields(nr, nz, np.random.default_rng(nr * 100 + nz), E0=3e6, H0=2e3)
    sim = Sim(cfg)
    sim.load(*parts)
    sim.set_fields(*flds)
    sim.step(STEPS)
    out = sim.fields(), sim.diag()["status_flags"]
    sim.close()
    return out, cfg, parts, flds


@pytest.mark.parametrize("nr,nz", GRIDS)
@pytest.mark.parametrize("flags", FLAGS)
def test_field_update_at_tile_edges_matches_oracle(tables, nr, nz, flags):
    ref = None
    for rows in (12, 16, 20):
        (f64, st), cfg, parts, flds = run(nr, nz, flags, abi.FP64, rows)
        assert st == 0
        if ref is None:
            ref = f64
            orc = O.Sim(cfg, tables, cap=cfg.capacity)
            orc.load(*parts)
            orc.Er[:], orc.Ez[:], orc.H[:] = flds
            orc.prologue()
            for _ in range(STEPS):
                orc.step()
            for g, w, k in zip(f64, (orc.Er, orc.Ez, orc.H), ("Er", "Ez", "H")):
                close(g, w, 1e-12, k)
        else:
            for a, b in zip(ref, f64):
                assert np.array_equal(a, b)
    f32 = []
    for gather in (abi.GATHER_QUADS, abi.GATHER_FIELDS):
        (f, st), _, _, _ = run(nr, nz, flags, abi.FP32_SPLIT, 16, gather)
        assert st == 0
        f32.append(f)
    for a, b in zip(*f32):
        assert np.array_equal(a, b)
    for g, w, k in zip(f32[0], ref, ("Er", "Ez", "H")):
        assert np.linalg.norm(g - w) <= 1e-4 * np.linalg.norm(w), k


@pytest.mark.parametrize("ratio", [1, 2])
def test_field_update_with_several_patches_per_warp_matches_oracle(tables, ratio):
    """512 x 1024 cells: more patches (or, with a field sub-cycle of 2, more
    blocks) than the field update keeps resident, so most warps take several
    patches and later ones are staged after neighbouring tiles were written;
    the FP64 form still matches the oracle (the tiles go to a second field
    buffer, so every halo holds the fields of the previous step)."""
    nr, nz = 512, 1024
    cfg = config(nr, nz, D, DT, 300.0, precision=abi.FP64, capacity=20000, seed=5,
                 sort_period=0, fdtd_ratio=ratio)
    cfg.fdtd_tile_rows = 12
    parts = births(1500, 8.0, nz * D, seed=11, sigma_r=2 * D, Rp=nr * D)
    flds = grid_fields(nr, nz, np.random.default_rng(3), E0=3e6, H0=2e3)
    flds[0][:, 0] = 0; flds[0][:, -1] = 0; flds[1][-1, :] = 0     # the PEC ends and the outer wall
    sim = Sim(cfg)
    sim.load(*parts)
    sim.set_fields(*flds)
    sim.step(STEPS)
    got, st = sim.fields(), sim.diag()["status_flags"]
    sim.close()
    assert st == 0
    orc = O.Sim(cfg, tables, cap=cfg.capacity)
    orc.load(*parts)
    orc.Er[:], orc.Ez[:], orc.H[:] = flds
    orc.prologue()
    for _ in range(STEPS):
        orc.step()
    for g, w, k in zip(got, (orc.Er, orc.Ez, orc.H), ("Er", "Ez", "H")):
        close(g, w, 1e-12, k)


def test_fp32_run_with_several_patches_per_warp_is_reproducible():
    """Two FP32 runs of the same 512 x 1024 cell (several field patches per
    warp) end with the same fields, current and counts, bit for bit."""
    nr, nz = 512, 1024
    out = []
    for _ in range(2):
        cfg = config(nr, nz, D, DT, 300.0, precision=abi.FP32_SPLIT, capacity=40000, seed=5,
                     sort_period=4)
        parts = births(4000, 8.0, nz * D, seed=11, sigma_r=20 * D, Rp=nr * D)
        flds = grid_fields(nr, nz, np.random.default_rng(3), E0=3e6, H0=2e3)
        sim = Sim(cfg)
        sim.load(*parts)
        sim.set_fields(*flds)
        sim.step(10)
        d = sim.diag()
        out.append((sim.fields(), sim.current(), d["n_ionizations"], d["n_alive"], d["status_flags"]))
        sim.close()
    (fa, ja, *ca), (fb, jb, *cb) = out
    assert ca == cb and ca[-1] == 0
    for a, b in zip(fa + ja, fb + jb):
        np.testing.assert_array_equal(a, b)

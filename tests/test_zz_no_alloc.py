"""gasatt_particle_density_noalloc against gasatt_particle_density.

The no-allocation variant serves callers that must not allocate device memory
-- above all a MEX gateway inside MATLAB, whose gpuArray pool owns the device
memory -- by counting into a fixed array compiled into the library instead of
the context's growable scratch.  Both entry points are called through the
C ABI on the same device inputs; the densities must agree exactly (the same
integer counts times FN / VC), on two calls in a row with different particles
and grid sizes, which also shows that the second call starts from zeroed
counters.  This file is named to be collected last."""
import ctypes

import numpy as np
import pytest
import torch

from _cases import cell_structure
from gasatt import _lib
from gasatt._lib import lib
from gasatt.dropin import Context

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _case(seed, n, zmax, rmax=25, delta=4e-4, PHIp=0.1, dz=1e-2):
    """A sector-cell grid of rmax rings x zmax layers and n particles, about 2%
    of them outside it (not counted)."""
    phimax, sum_cell, cellnumxy = cell_structure(PHIp, rmax * delta, rmax, delta)
    dphi = PHIp / phimax
    VC = np.concatenate([[0.5 * ((i * delta)**2 - ((i - 1) * delta)**2) * dphi[i - 1] * dz]
                         * int(phimax[i - 1]) for i in range(1, rmax + 1)])
    rng = np.random.default_rng(seed)
    r = rng.uniform(0, rmax * delta * 1.02, n)
    phi = rng.uniform(-0.01, PHIp, n)
    z = rng.uniform(0, zmax * dz, n)
    dev = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64)).cuda().contiguous()
    return dict(dr=delta, dz=dz, dphi=dev(dphi), rmax=rmax, r=dev(r), phi=dev(phi), z=dev(z),
                n=n, cellnumxy=int(cellnumxy), sum_cell=dev(sum_cell), VC=dev(VC),
                ncell=int(cellnumxy) * zmax)


def _call(fn, ctx, c, FN, out, ncell=None):
    return fn(ctx.handle, c["dr"], c["dz"], _p(c["dphi"]), c["rmax"], _p(c["r"]), _p(c["phi"]),
              _p(c["z"]), c["n"], c["cellnumxy"], _p(c["sum_cell"]), _p(c["VC"]),
              c["ncell"] if ncell is None else ncell, FN, _p(out))


def test_noalloc_density_matches_allocating_entry_point_twice():
    ctx = Context(0)
    try:
        # the second case has fewer particles and fewer cells than the first, so
        # counts left over from the first call would show up in it
        for seed, n, zmax, FN in ((21, 300000, 9, 3.0), (22, 120000, 6, 1.5)):
            c = _case(seed, n, zmax)
            want = torch.full((c["ncell"],), np.nan, dtype=torch.float64, device="cuda")
            got = torch.full((c["ncell"],), np.nan, dtype=torch.float64, device="cuda")
            assert _call(lib.gasatt_particle_density, ctx, c, FN, want) == _lib.OK
            assert _call(lib.gasatt_particle_density_noalloc, ctx, c, FN, got) == _lib.OK, \
                lib.gasatt_last_error(ctx.handle)
            assert lib.gasatt_synchronize(ctx.handle) == _lib.OK
            w, g = want.cpu().numpy(), got.cpu().numpy()
            assert np.all(np.isfinite(g)) and np.any(g > 0)
            np.testing.assert_array_equal(g, w)
    finally:
        ctx.close()


def test_noalloc_density_rejects_grids_beyond_its_fixed_scratch():
    ctx = Context(0)
    try:
        c = _case(23, 1000, 2)
        too_many = (1 << 20) + 1
        out = torch.zeros(too_many, dtype=torch.float64, device="cuda")
        rc = _call(lib.gasatt_particle_density_noalloc, ctx, c, 1.0, out, ncell=too_many)
        assert rc == _lib.E_CAPACITY
        msg = lib.gasatt_last_error(ctx.handle).decode()
        assert "1048576" in msg and "particle_density_noalloc" in msg
        assert lib.gasatt_synchronize(ctx.handle) == _lib.OK
        assert torch.count_nonzero(out).item() == 0           # nothing was written
    finally:
        ctx.close()


def test_noalloc_density_allocates_nothing():
    """On a fresh context, after one call that loads the library's device code
    (and with it the fixed array), further no-allocation calls leave the
    device's free memory unchanged: they take nothing from the context's
    scratch (which a fresh context would have to cudaMalloc) nor from
    anywhere else."""
    warm = Context(0)
    fresh = Context(0)
    try:
        c = _case(24, 200000, 8)
        out = torch.zeros(c["ncell"], dtype=torch.float64, device="cuda")
        assert _call(lib.gasatt_particle_density_noalloc, warm, c, 1.0, out) == _lib.OK
        assert lib.gasatt_synchronize(warm.handle) == _lib.OK
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        for FN in (1.0, 2.0, 4.0):
            assert _call(lib.gasatt_particle_density_noalloc, fresh, c, FN, out) == _lib.OK, \
                lib.gasatt_last_error(fresh.handle)
            assert lib.gasatt_synchronize(fresh.handle) == _lib.OK
            assert torch.cuda.mem_get_info()[0] == free0
        assert torch.count_nonzero(out).item() > 0
    finally:
        fresh.close()
        warm.close()

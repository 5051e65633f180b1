"""Seeded synthetic inputs shared by the parity tests."""
import math

import numpy as np


def close(a, b, rtol, what=""):
    """Norm-wise relative error: max|a-b| / max|b| <= rtol.  NaNs (which the
    reference produces in some quirk cases) must sit at the same places."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb), f"{what}: NaN positions differ ({na.sum()} vs {nb.sum()})"
    a, b = a[~na], b[~nb]
    if a.size == 0:
        return 0.0
    scale = np.max(np.abs(b))
    err = np.max(np.abs(a - b)) / (scale if scale > 0 else 1.0)
    assert err <= rtol, f"{what}: relative error {err:.3e} > {rtol:.1e}"
    return err


def grid_fields(nr, nz, rng, E0=1e5, H0=50.0):
    """Smooth random fields in the MATLAB shapes Er (nr, nz+1), Ez (nr+1, nz), H (nr, nz)."""
    def smooth(shape):
        i = np.arange(shape[0])[:, None] / shape[0]
        j = np.arange(shape[1])[None, :] / shape[1]
        f = np.zeros(shape)
        for _ in range(4):
            a, b, c = rng.normal(), rng.uniform(0.5, 3), rng.uniform(0.5, 3)
            f += a * np.sin(math.pi * (b * i + rng.uniform())) * np.cos(math.pi * (c * j + rng.uniform()))
        return f
    Er = E0 * smooth((nr, nz + 1))
    Ez = E0 * smooth((nr + 1, nz))
    H = H0 * smooth((nr, nz))
    return np.asfortranarray(Er), np.asfortranarray(Ez), np.asfortranarray(H)


def wedge_particles(n, Rp, Lp, PHIp, rng, vmag=1e7, rmin=0.02, rmax=0.95, cyl=True):
    """n particles inside the wedge; positions (r, phi, z) if cyl else (x, y, z)."""
    r = Rp * rng.uniform(rmin, rmax, n)
    phi = PHIp * rng.uniform(0.02, 0.98, n)
    z = Lp * rng.uniform(0.02, 0.98, n)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    v = d * (vmag * rng.uniform(0.3, 1.0, n))[:, None]
    pos = np.stack([r, phi, z], 1) if cyl else np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    return pos, v


def cell_structure(PHIp, Rp, rmax, delta):
    """cell_structure.m:1-28: cells per ring phi_divide(k) = ceil(k/rmax Rp PHIp/delta)."""
    k = np.arange(1, rmax + 1)
    phimax = np.ceil(k / rmax * Rp * PHIp / delta)
    sum_cell = np.cumsum(phimax)
    return phimax, sum_cell, int(sum_cell[-1])


def draws(n, rng, p_collide=None):
    """Injected draws (n x 8): uniforms in (0,1) in slots 0..3, float-exact normals in 4..6."""
    d = np.empty((n, 8))
    d[:, :4] = (rng.integers(1, 2**53, size=(n, 4)) / 2.0**53)
    d[:, 4:7] = rng.normal(size=(n, 3)).astype(np.float32).astype(np.float64)
    d[:, 7] = 0
    if p_collide is not None:
        d[:, 0] = rng.uniform(0, p_collide, n)
    return np.ascontiguousarray(d)


def kinetic_kev(v, m=9.109e-31, e=1.6022e-19, c=3e8):
    v2 = np.sum(v * v, axis=1)
    g = 1 / np.sqrt(1 - v2 / (c * c))
    return (g - 1) * m * c * c / e / 1000

"""The oracle's restatement of the reference's MATLAB CPU path
(electricmagneticfield3.m:111-319), used as a second CPU baseline: its field
update against the oracle's resident field update with the reference's
field quirks, the nearest-cell current, the explicit kick in a uniform field
and the deletion at the wall."""
import numpy as np

import pyoracle as O
from _cases import grid_fields
from gasatt import abi
from gasatt.workload import config

NR, NZ, D, DT = 24, 40, 10e-6, 2e-14
E_MC, ME_MC, C_MC = 1.6e-19, 9.1096e-31, 3e8      # electricmagneticfield3.m:4-11


def test_field_update_matches_the_resident_one_with_the_reference_quirks():
    """No particles: H(-dt/4), [H(dt/2), E(dt/2)] x 2, H(dt/4) equals the
    resident oracle's fused sub-cycle run with the quirks the MATLAB path has
    (Er end rows copied, +jz on the axis) and its constants."""
    m = O.MatlabCpuPath(NR, NZ, D, DT)
    Er, Ez, H = grid_fields(NR, NZ, np.random.default_rng(3), E0=2e6, H0=4e3)
    m.Er[:], m.Ez[:], m.H[:] = Er, Ez, H
    m.load(*[np.zeros(0)] * 6)
    cfg = config(NR, NZ, D, DT, 1.0, precision=abi.FP64)
    cfg.eps0, cfg.mu0 = 8.854187817e-12, 4 * np.pi * 1e-7
    cfg.flags = abi.Q_ER_END_COPY | abi.Q_EZ_AXIS_JSIGN
    Er2, Ez2, H2 = (np.array(a, order="F") for a in (Er, Ez, H))
    zero = np.zeros((NR, NZ), order="F")
    for _ in range(3):
        m.step()
        O.lib.orc_sim_fdtd(O.ctypes.byref(cfg), O.P(Er2), O.P(Ez2), O.P(H2), O.P(zero), O.P(zero))
    for a, b in ((m.Er, Er2), (m.Ez, Ez2), (m.H, H2)):
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))


def test_explicit_kick_in_a_uniform_field_and_the_two_half_drifts():
    """A uniform Ez and no self-field (W = 0): u = gamma v + q E / m dt, then
    v = u / gamma(u), and the position moves by dt/2 with each velocity."""
    m = O.MatlabCpuPath(NR, NZ, D, DT, W=0.0)
    E0 = 3e6
    m.Ez[:] = E0
    x0, y0, z0 = 60e-6, 70e-6, 200e-6
    v0 = np.array([2e6, 3e6, -1e6])
    m.load([x0], [y0], [z0], [v0[0]], [v0[1]], [v0[2]])
    m.step()
    g0 = 1 / np.sqrt(1 - v0 @ v0 / C_MC ** 2)
    u = g0 * v0 + np.array([0, 0, -E_MC * E0 / ME_MC * DT])
    v1 = u / np.sqrt(1 + u @ u / C_MC ** 2)
    assert np.allclose([m.vx[0], m.vy[0], m.vz[0]], v1, rtol=1e-12, atol=0)
    p1 = np.array([x0, y0, z0]) + DT / 2 * v0 + DT / 2 * v1
    assert np.allclose([m.x[0], m.y[0], m.z[0]], p1, rtol=1e-12, atol=0)


def test_nearest_cell_current_and_deletion_at_the_wall():
    """One electron deposits q v_r and q v_z on the cell round(r/d + 1/2),
    round(z/d + 1/2) (ind2vec), divided by phi ((R + d/2)^2 - (R - d/2)^2) dz
    and times W; an electron crossing r = R is deleted."""
    W = 7.0
    m = O.MatlabCpuPath(NR, NZ, D, DT, W=W)
    x, z = 53e-6, 125e-6
    v = np.array([4e6, 0.0, 2e6])
    Rw = NR * D
    m.load([x, Rw - 1e-9], [0.0, 0.0], [z, z], [v[0], 5e7], [0.0, 0.0], [v[2], 0.0])
    alive = m.step()
    assert alive == 1 and m.alive.tolist() == [1, 0]
    xh, zh = x + DT / 2 * v[0], z + DT / 2 * v[2]
    ar, az = int(np.floor(xh / D + 0.5 + 0.5)), int(np.floor(zh / D + 0.5 + 0.5))
    Rc = (ar - 0.5) * D
    V = 2 * np.pi * ((Rc + D / 2) ** 2 - (Rc - D / 2) ** 2) * D
    jr = np.zeros((NR, NZ)); jz = np.zeros((NR, NZ))
    jr[ar - 1, az - 1] = W * -E_MC * v[0] / V
    jz[ar - 1, az - 1] = W * -E_MC * v[2] / V
    assert np.allclose(m.jr, jr, rtol=1e-13, atol=0) and np.allclose(m.jz, jz, rtol=1e-13, atol=0)

"""Golden vectors from the reference's own CUDA kernels.

The reference ships no tests or fixtures, so its kernels (EM2.cu, EM7.cu,
EM3_1.cu, EM3.cu, EM4.cu, electron_transport.cu - compiled from the
reference sources into oracle/_ref by `make -C oracle ref`, with random
draws injected through oracle/refdrv/rng_shim.h) are run on seeded inputs and
their outputs saved next to the inputs.  tests/test_golden.py then checks the
CPU oracle against these files without a GPU.

Inputs stay where the reference kernels read in bounds: particles strictly
inside the grid and the wedge, electron energies below 2.5 keV in the
collision case (the reference's elastic bin search compares keV with ln E and
would run past its 36-entry table above ln 20 keV = 3.0).

    python tests/golden/make_golden.py [out_dir]     (needs a GPU)
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "gas-atenuator_b200"), os.path.join(ROOT, "oracle"),
                os.path.join(ROOT, "tests")]

from _cases import cell_structure, draws, grid_fields, kinetic_kev, wedge_particles  # noqa: E402

MU = 4e-7 * math.pi
EPS = 8.854187817e-12


def em_case(seed=11, n=2000, nr=12, nz=20, d=1e-4, PHIp=0.1):
    """Inputs for EM2 -> EM7 -> EM3_1 -> EM3 -> EM4 (one particle step, feval order)."""
    rng = np.random.default_rng(seed)
    Er, Ez, H = grid_fields(nr, nz, rng, E0=2e5, H0=200.0)
    pos, v = wedge_particles(n, nr * d, nz * d, PHIp, rng, cyl=False, vmag=3e7)
    jr0, jz0 = grid_fields(nr, nz, rng, E0=1e6, H0=1e6)[2], grid_fields(nr, nz, rng, H0=1e6)[2]
    return dict(nr=nr, nz=nz, d=d, PHIp=PHIp, Rp=nr * d, Lp=nz * d, dt=1e-13,
                x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(),
                vx=v[:, 0].copy(), vy=v[:, 1].copy(), vz=v[:, 2].copy(),
                q=np.where(rng.random(n) < 0.8, -1.6e-19, 1.6e-19),
                m=np.where(rng.random(n) < 0.8, 9.1096e-31, 4.65e-26),
                Er=Er, Ez=Ez, H=H, jr=np.asfortranarray(jr0), jz=np.asfortranarray(jz0))


def mcc_case(seed=12, n=4000, PHIp=0.1, Rp=1e-2, rmax=20, zmax=5, Lp=0.05):
    rng = np.random.default_rng(seed)
    delta = Rp / rmax
    phimax, sum_cell, cellnumxy = cell_structure(PHIp, Rp, rmax, delta)
    pos, _ = wedge_particles(n, Rp, Lp, PHIp, rng, cyl=False)
    E_eV = np.exp(rng.uniform(np.log(16.0), np.log(2500.0), n))
    E_eV[: n // 8] = rng.uniform(1.0, 15.0, n // 8)          # below the ionization threshold
    m, e, c = 9.109e-31, 1.6022e-19, 3e8
    g = 1 + E_eV * e / (m * c * c)
    speed = c * np.sqrt(1 - 1 / g**2)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    v = d * speed[:, None]
    v[:20, :2] = 0.0                                          # along z: rotate() fallback branch
    v[:20, 2] = speed[:20]
    ncell = cellnumxy * zmax
    density = np.full(ncell, 3.2e22) * rng.uniform(0.5, 1.5, ncell)
    temperature = 300.0 * rng.uniform(0.8, 1.2, ncell)
    # cross-sections of the reference's own table lookups, scaled so most electrons collide
    return dict(n=n, PHIp=PHIp, Rp=Rp, Lp=Lp, rmax=rmax, zmax=zmax, phimax=phimax,
                sum_cell=sum_cell, cellnumxy=cellnumxy, dr=delta, dz=Lp / zmax,
                x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(),
                vx=v[:, 0].copy(), vy=v[:, 1].copy(), vz=v[:, 2].copy(),
                energy=kinetic_kev(v), density=density, temperature=temperature,
                se=rng.uniform(1e-21, 2e-19, n), si=rng.uniform(0, 5e-20, n),
                sx=rng.uniform(0, 5e-20, n), dt=2e-10, draws=draws(n, rng))


def run_em_reference(ref, cs):
    out = {}
    n = cs["x"].size
    x, y, z, vx, vy, vz = (cs[k].copy() for k in ("x", "y", "z", "vx", "vy", "vz"))
    r = np.zeros(n); phi = np.zeros(n); vr = np.zeros(n); dele = np.zeros(n, np.int32)
    ddt = 5 * cs["dt"]
    assert ref.EM2(x, y, z, vx, vy, vz, r, phi, vr, dele, cs["Rp"], cs["Lp"], cs["PHIp"], cs["d"],
                   cs["d"], ddt) == 0
    out.update(em2_x=x.copy(), em2_y=y.copy(), em2_z=z.copy(), em2_vx=vx.copy(), em2_vy=vy.copy(),
               em2_vz=vz.copy(), em2_r=r.copy(), em2_phi=phi.copy(), em2_vr=vr.copy(),
               em2_del=dele.copy())
    nr, nz = cs["nr"], cs["nz"]
    jr = np.zeros((nr, nz), order="F"); jz = np.zeros((nr, nz), order="F")
    assert ref.EM7(r, z, cs["q"], vr, vz, jr, jz, dele, nr, nz, cs["d"], cs["d"], 1e3, cs["PHIp"]) == 0
    out.update(em7_jr=jr.copy(), em7_jz=jz.copy())
    H = cs["H"].copy(order="F")
    assert ref.EM3_1(cs["Er"], cs["Ez"], H, nr, nz, MU, cs["d"], cs["d"], cs["dt"] / 2) == 0
    out.update(em3_1_H=H.copy())
    Er = cs["Er"].copy(order="F"); Ez = cs["Ez"].copy(order="F")
    assert ref.EM3(cs["Er"], cs["Ez"], H, Er, Ez, cs["jr"], cs["jz"], nr, nz, MU, EPS, cs["d"],
                   cs["d"], cs["dt"] / 2) == 0
    out.update(em3_Er=Er.copy(), em3_Ez=Ez.copy())
    E = np.zeros(n)
    assert ref.EM4(x, y, z, vx, vy, vz, r, phi, vr, Er, Ez, H, cs["q"], cs["m"], E, dele,
                   cs["Rp"], cs["Lp"], cs["PHIp"], nr, nz, MU, 3e8, cs["d"], cs["d"], ddt) == 0
    out.update(em4_x=x, em4_y=y, em4_z=z, em4_vx=vx, em4_vy=vy, em4_vz=vz, em4_E=E, em4_del=dele)
    return out


def mcc_tables():
    from gasatt.tables import N2Tables
    import pyoracle as O
    tab = N2Tables()
    xI, yI, V = O.elastic_tables(tab)
    return tab, xI, yI, V


def run_mcc_reference(ref, cs):
    tab, xI, yI, V = mcc_tables()
    vx, vy, vz = cs["vx"].copy(), cs["vy"].copy(), cs["vz"].copy()
    sc0 = np.concatenate([[0], cs["sum_cell"]]).astype(np.int32)
    dphi = cs["PHIp"] / cs["phimax"]
    rc, sec, outs = ref.electron_transport(cs["x"], cs["y"], cs["z"], vx, vy, vz, cs["se"],
                                           cs["si"], cs["sx"], cs["energy"], xI, yI, V,
                                           cs["density"], cs["temperature"], dphi,
                                           np.asarray(tab["t_exc"]), sc0, cs["cellnumxy"],
                                           cs["dr"], cs["dz"], cs["dt"], cs["draws"])
    assert rc == 0, rc
    return dict(mcc_vx=vx, mcc_vy=vy, mcc_vz=vz, mcc_sec=sec, mcc_svx=outs[0], mcc_svy=outs[1],
                mcc_svz=outs[2], mcc_sample=outs[3], mcc_ivx=outs[4], mcc_ivy=outs[5],
                mcc_ivz=outs[6])


def main(out_dir):
    import pyoracle as O
    ref = O.RefKernels()
    em = em_case()
    mc = mcc_case()
    res_em = run_em_reference(ref, em)
    res_mc = run_mcc_reference(ref, mc)
    os.makedirs(out_dir, exist_ok=True)
    np.savez_compressed(os.path.join(out_dir, "ref_em_kernels.npz"),
                        **{f"in_{k}": np.asarray(v) for k, v in em.items()}, **res_em)
    np.savez_compressed(os.path.join(out_dir, "ref_electron_transport.npz"),
                        **{f"in_{k}": np.asarray(v) for k, v in mc.items()}, **res_mc)
    print("wrote", out_dir, "collisions:", int(res_mc["mcc_sec"].sum()), "ionizations")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)

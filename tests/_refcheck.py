"""Oracle side of the reference-kernel pinning (shared by the golden-file test
on CPU and the live test on a GPU)."""
import math

import numpy as np

import pyoracle as O
from _cases import close
from gasatt import _lib

MU = 4e-7 * math.pi
EPS = 8.854187817e-12


def oracle_em(cs):
    """EM2 -> EM7 -> EM3_1 -> EM3 -> EM4 on the oracle, same call order as the golden run."""
    F = _lib.FAITHFUL
    out = {}
    n = cs["x"].size
    x, y, z, vx, vy, vz = (np.array(cs[k], dtype=np.float64) for k in ("x", "y", "z", "vx", "vy", "vz"))
    r = np.zeros(n); phi = np.zeros(n); vr = np.zeros(n); dele = np.zeros(n, np.int32)
    ddt = 5 * float(cs["dt"])
    Rp, Lp, PHIp, d = float(cs["Rp"]), float(cs["Lp"]), float(cs["PHIp"]), float(cs["d"])
    nr, nz = int(cs["nr"]), int(cs["nz"])
    O.em2(x, y, z, vx, vy, vz, r, phi, vr, dele, Rp, Lp, PHIp, ddt, F)
    out.update(em2_x=x.copy(), em2_y=y.copy(), em2_z=z.copy(), em2_vx=vx.copy(), em2_vy=vy.copy(),
               em2_vz=vz.copy(), em2_r=r.copy(), em2_phi=phi.copy(), em2_vr=vr.copy(),
               em2_del=dele.copy())
    jr = np.zeros((nr, nz), order="F"); jz = np.zeros((nr, nz), order="F")
    O.em7(r, z, np.ascontiguousarray(cs["q"]), vr, vz, jr, jz, dele, nr, nz, d, d, 1e3, PHIp)
    out.update(em7_jr=jr, em7_jz=jz)
    H = np.array(cs["H"], order="F")
    Er0 = np.array(cs["Er"], order="F"); Ez0 = np.array(cs["Ez"], order="F")
    O.em3_1(Er0, Ez0, H, nr, nz, MU, d, d, float(cs["dt"]) / 2)
    out.update(em3_1_H=H.copy())
    Er = Er0.copy(order="F"); Ez = Ez0.copy(order="F")
    O.em3(Er0, Ez0, H, Er, Ez, np.array(cs["jr"], order="F"), np.array(cs["jz"], order="F"), nr, nz,
          EPS, d, d, float(cs["dt"]) / 2, F)
    out.update(em3_Er=Er.copy(), em3_Ez=Ez.copy())
    E = np.zeros(n)
    O.em4(x, y, z, vx, vy, vz, r, phi, vr, Er, Ez, H, np.ascontiguousarray(cs["q"]),
          np.ascontiguousarray(cs["m"]), E, dele, Rp, Lp, PHIp, nr, nz, MU, 3e8, d, d, ddt, F)
    out.update(em4_x=x, em4_y=y, em4_z=z, em4_vx=vx, em4_vy=vy, em4_vz=vz, em4_E=E, em4_del=dele)
    return out


def assert_em_match(got, ref, rtol=1e-12):
    for k in ref:
        if k.endswith("_del"):
            np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
        else:
            close(got[k], ref[k], rtol, k)


def oracle_mcc(cs, tables, flags=_lib.FAITHFUL):
    xI, yI, V = O.elastic_tables(tables)
    vx, vy, vz = (np.array(cs[k], dtype=np.float64) for k in ("vx", "vy", "vz"))
    sc0 = np.concatenate([[0], cs["sum_cell"]]).astype(np.int32)
    dphi = float(cs["PHIp"]) / np.asarray(cs["phimax"], dtype=np.float64)
    sec, outs = O.electron_transport(np.ascontiguousarray(cs["x"]), np.ascontiguousarray(cs["y"]),
                                     np.ascontiguousarray(cs["z"]), vx, vy, vz,
                                     np.ascontiguousarray(cs["se"]), np.ascontiguousarray(cs["si"]),
                                     np.ascontiguousarray(cs["sx"]), np.ascontiguousarray(cs["energy"]),
                                     xI, yI, V, np.ascontiguousarray(cs["density"]),
                                     np.ascontiguousarray(cs["temperature"]), dphi,
                                     np.asarray(tables["t_exc"]), sc0, int(cs["rmax"]),
                                     int(cs["cellnumxy"]), float(cs["dr"]), float(cs["dz"]),
                                     float(cs["dt"]), np.ascontiguousarray(cs["draws"]), flags)
    return dict(mcc_vx=vx, mcc_vy=vy, mcc_vz=vz, mcc_sec=sec, mcc_svx=outs[0], mcc_svy=outs[1],
                mcc_svz=outs[2], mcc_sample=outs[3], mcc_ivx=outs[4], mcc_ivy=outs[5],
                mcc_ivz=outs[6])


def excitation_rows(cs, got):
    """Electrons whose speed changed but direction did not (excitation energy loss)."""
    v0 = np.stack([cs["vx"], cs["vy"], cs["vz"]], 1)
    v1 = np.stack([got["mcc_vx"], got["mcc_vy"], got["mcc_vz"]], 1)
    s0, s1 = np.linalg.norm(v0, axis=1), np.linalg.norm(v1, axis=1)
    cos = np.sum(v0 * v1, 1) / (s0 * s1)
    return (cos > 1 - 1e-9) & (np.abs(s1 / s0 - 1) > 1e-12)


def assert_mcc_match(got, ref, cs, rtol=1e-12, rtol_exc=1e-5):
    """Branch outcomes exact; velocities to rtol, except the excitation loss
    which the reference evaluates with single-precision powf (rtol_exc)."""
    np.testing.assert_array_equal(got["mcc_sec"], ref["mcc_sec"])
    exc = excitation_rows(cs, ref)
    for k in ("mcc_vx", "mcc_vy", "mcc_vz"):
        close(got[k][~exc], ref[k][~exc], rtol, k)
        close(got[k][exc], ref[k][exc], rtol_exc, k + " (excitation)")
    s = ref["mcc_sec"].astype(bool)
    for k in ("mcc_svx", "mcc_svy", "mcc_svz", "mcc_ivx", "mcc_ivy", "mcc_ivz"):
        close(got[k][s], ref[k][s], rtol, k)
    np.testing.assert_array_equal(got["mcc_sample"][s], ref["mcc_sample"][s])
    return int(s.sum()), int(exc.sum())

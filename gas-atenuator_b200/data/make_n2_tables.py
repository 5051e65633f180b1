"""Build ``n2_tables.npz`` from the reference's N2 electron cross-section CSVs.

The arrays are the seven tables exactly as the MATLAB driver loads them with
``readtable`` + ``table2array`` (electron_transport_field3.m:8-37), i.e. the
first line of a CSV is data unless it is non-numeric (the excitation table's
``j,A,omega,v,miu`` header, ParameterExcCS_Nitrogen.csv, which also uses bare
CR line endings).  Shapes are the MATLAB (rows, cols) shapes:

    t_el    (2, 29)   row 0: energy [keV] 0.05..20, row 1: sigma_el [a0^2 per N atom]
    t_sel   (26, 2)   energy [eV] 1..50, sigma_el [1e-20 m^2 per N2]
    t_sel_1 (8, 2)    energy [eV] 5..50, sigma_el [1e-20 m^2 per N2]
    t_del   (182, 30) row 0: energies [keV] (col 0 = 0), col 0: angle [deg] 0..180,
                      body: elastic DCS, E >= 50 eV
    t_sdel  (182, 8)  same layout, 5..40 eV
    t_ion   (38, 2)   energy [eV] 15.6..20000, sigma_ion [1e-20 m^2]
    t_exc   (7, 5)    k_j [eV], A_j, omega_j, nu_j, gamma_j (excitation fit)

These are measured/evaluated physics data; the library needs them verbatim.
Run once where the reference tree is available:

    python gas-atenuator_b200/data/make_n2_tables.py /path/to/reference
"""
import os
import sys

import numpy as np

FILES = {
    "t_el": "TotalElasticCS_Nitrogen.csv",
    "t_sel": "TotalElasticCS_smalleV_Nitrogen.csv",
    "t_sel_1": "TotalElasticCS_smalleV_Nitrogen_1.csv",
    "t_del": "ElasticCS_Nitrogen.csv",
    "t_sdel": "ElasticDCS_smalleV_Nitrogen.csv",
    "t_ion": "TotalIonCS_Nitrogen.csv",
    "t_exc": "ParameterExcCS_Nitrogen.csv",
}


def read_matlab_table(path):
    """Numeric CSV -> 2-D float64 array, skipping a non-numeric header line."""
    txt = open(path, "rb").read().decode("ascii")
    txt = txt.replace("\r\n", "\n").replace("\r", "\n")
    rows = [r for r in txt.split("\n") if r.strip()]
    out = []
    for i, row in enumerate(rows):
        cells = row.split(",")
        try:
            out.append([float(c) for c in cells])
        except ValueError:
            if i == 0:      # header line (variable names)
                continue
            raise
    return np.array(out, dtype=np.float64)


def main(ref_dir):
    tabs = {k: read_matlab_table(os.path.join(ref_dir, f)) for k, f in FILES.items()}
    expect = {"t_el": (2, 29), "t_sel": (26, 2), "t_sel_1": (8, 2), "t_del": (182, 30),
              "t_sdel": (182, 8), "t_ion": (38, 2), "t_exc": (7, 5)}
    for k, shp in expect.items():
        assert tabs[k].shape == shp, (k, tabs[k].shape)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "n2_tables.npz")
    np.savez(out, **tabs)
    print("wrote", out)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GASATT_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: make_n2_tables.py REFERENCE_DIR (or set GASATT_REFERENCE_DIR)")
    main(ref)

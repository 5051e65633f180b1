"""N2 cross-section tables (the reference CSVs as MATLAB readtable loads them)."""
import ctypes
import os

import numpy as np

from .abi import Tables

DATA = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "data",
                    "n2_tables.npz")


class N2Tables:
    """Holds the seven raw tables in Fortran order and a gasatt_tables view."""

    NAMES = ("t_el", "t_sel", "t_sel_1", "t_del", "t_sdel", "t_ion", "t_exc")

    def __init__(self, path=DATA, **override):
        z = np.load(path)
        self.arrays = {k: np.asfortranarray(override.get(k, z[k]), dtype=np.float64)
                       for k in self.NAMES}
        a = self.arrays
        p = lambda k: a[k].ctypes.data_as(ctypes.c_void_p)
        self.struct = Tables(p("t_el"), a["t_el"].shape[1], p("t_sel"), a["t_sel"].shape[0],
                             p("t_sel_1"), a["t_sel_1"].shape[0],
                             p("t_del"), a["t_del"].shape[0], a["t_del"].shape[1],
                             p("t_sdel"), a["t_sdel"].shape[0], a["t_sdel"].shape[1],
                             p("t_ion"), a["t_ion"].shape[0], p("t_exc"), a["t_exc"].shape[0])

    def __getitem__(self, k):
        return self.arrays[k]

    @property
    def ref(self):
        return ctypes.byref(self.struct)

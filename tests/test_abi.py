"""The C-ABI library loads and exports every entry point include/gasatt.h declares."""
import ctypes
import os
import re

import pytest

from conftest import ROOT, has_gpu


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "gasatt.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gasatt_[a-zA-Z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for must in ("gasatt_find_CS0", "gasatt_free_motion", "gasatt_particle_density",
                 "gasatt_electricmagneticfield6", "gasatt_electron_collision", "gasatt_sim_step"):
        assert must in syms


def test_library_exports_every_declared_symbol():
    from gasatt import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared_symbols()) == set(_lib.EXPORTS)


def test_version_string():
    from gasatt import _lib
    assert b"sm_100a" in _lib.lib.gasatt_version()


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_create_without_device_fails_cleanly():
    from gasatt import _lib
    h = ctypes.c_void_p()
    assert _lib.lib.gasatt_create(ctypes.byref(h), 0, 0) == _lib.E_NODEVICE


def test_product_path_never_imports_oracle():
    pkg = os.path.join(ROOT, "gas-atenuator_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
                txt = open(os.path.join(dirpath, f), errors="ignore").read()
                assert "pyoracle" not in txt and "liboracle" not in txt and "orc_" not in txt, f

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


def test_python_default_config_matches_the_library():
    """gasatt.abi.default_config restates gasatt_sim_default_config (host
    code, callable without a device) field by field."""
    from gasatt import _lib
    from gasatt.abi import default_config
    want = _lib.SimConfig()
    assert _lib.lib.gasatt_sim_default_config(ctypes.byref(want)) == _lib.OK
    got = default_config()
    for name, _ in _lib.SimConfig._fields_:
        assert getattr(got, name) == getattr(want, name), name


def test_workload_builders_load_no_library():
    """The workload builders (births, configs, tables) and the CPU oracle are
    importable without libgasatt.so being mapped: the CPU reference arm of
    bench.py builds its inputs this way."""
    import subprocess
    import sys
    code = ("import sys; sys.path[:0] = [%r, %r]\n"
            "import gasatt.workload, gasatt.tables, gasatt.abi, pyoracle\n"
            "cfg = gasatt.workload.config(16, 32, 5e-6, 1e-14, 1.0)\n"
            "p = gasatt.workload.births(10, 8.0, 32 * 5e-6, seed=1)\n"
            "o = pyoracle.Sim(cfg, gasatt.tables.N2Tables(), cap=64)\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'libgasatt' not in maps, 'libgasatt.so mapped'\n"
            "assert 'gasatt._lib' not in sys.modules\n"
            % (os.path.join(ROOT, "gas-atenuator_b200"), os.path.join(ROOT, "oracle")))
    subprocess.run([sys.executable, "-c", code], check=True)

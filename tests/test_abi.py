"""The C-ABI surface without a GPU: the library loads, exports every function include/radb200.h
declares, the ctypes structures match the C layout, and argument checks fail with the documented codes
before any device work."""
from __future__ import annotations

import ctypes
import re
import subprocess

import pytest

from conftest import ROOT
from woof_nam_b200 import _lib, build

HEADER = ROOT / "include" / "radb200.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-zA-Z_][\w\s\*]*?\b(rad_\w+)\s*\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def test_every_declared_symbol_is_exported_and_bound(lib):
    names = declared_functions()
    assert "rad_solve" in names and "rad_create" in names
    for n in names:
        assert hasattr(lib, n), f"libradb200.so does not export {n}"
        assert n in _lib.SIGNATURES, f"the ctypes binding does not declare {n}"
    assert set(_lib.SIGNATURES) == set(names)


def test_struct_layout_matches_header(tmp_path):
    probe = tmp_path / "probe.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for st in (_lib.RadConfig, _lib.RadColumns, _lib.RadOutputs, _lib.RadProfile, _lib.RadPostIn, _lib.RadPostOut,
               _lib.RadRdtemp, _lib.RadAerClim, _lib.RadAerColumns, _lib.RadSolarIn, _lib.RadSolarState, _lib.RadModelColumns,
               _lib.RadLayerFields, _lib.RadDayparts, _lib.RadGasSetup, _lib.RadOzoneClim, _lib.RadAlbedoIn,
               _lib.RadEmisIn, _lib.RadCloudIn, _lib.RadCloudCfg, _lib.RadCloudOut, _lib.RadPayneTables):
        lines.append(f'printf("{st.__name__} size %zu\\n", sizeof({st.__name__}));')
        for f, _ in st._fields_:
            lines.append(f'printf("{st.__name__}.{f} %zu\\n", offsetof({st.__name__}, {f}));')
    lines.append("return 0;}")
    probe.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(probe)], check=True)
    got = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                               check=True).stdout.splitlines())
    for st in (_lib.RadConfig, _lib.RadColumns, _lib.RadOutputs, _lib.RadProfile, _lib.RadPostIn, _lib.RadPostOut,
               _lib.RadRdtemp, _lib.RadAerClim, _lib.RadAerColumns, _lib.RadSolarIn, _lib.RadSolarState, _lib.RadModelColumns,
               _lib.RadLayerFields, _lib.RadDayparts, _lib.RadGasSetup, _lib.RadOzoneClim, _lib.RadAlbedoIn,
               _lib.RadEmisIn, _lib.RadCloudIn, _lib.RadCloudCfg, _lib.RadCloudOut, _lib.RadPayneTables):
        assert int(got[f"{st.__name__} size"]) == ctypes.sizeof(st), st.__name__
        for f, _ in st._fields_:
            assert int(got[f"{st.__name__}.{f}"]) == getattr(st, f).offset, f"{st.__name__}.{f}"


def test_version_and_defaults(lib):
    assert lib.rad_version() == 2
    c = _lib.RadConfig()
    lib.rad_config_default(ctypes.byref(c), 61)
    assert (c.nlay, c.precision, c.route, c.iswmode, c.diagnostic) == (61, _lib.PREC["mixed"], 0, 2, 0)
    assert (c.iovrlw, c.iovrsw, c.lw_seed0, c.sw_seed0) == (1, 1, 140, 1)
    assert c.sw_chunk == 32768 and abs(c.cpathfac - 1.5) < 1e-7
    assert c.lw_chunk == 0 and c.sw_sweep_chunk == 0


@pytest.mark.parametrize("field,value", [("nlay", 1), ("nlay", 100000), ("iswmode", 0), ("iswmode", 4),
                                         ("precision", 7), ("route", 9)])
def test_create_rejects_bad_config(lib, field, value):
    c = _lib.RadConfig()
    lib.rad_config_default(ctypes.byref(c), 61)
    setattr(c, field, value)
    h = ctypes.c_void_p()
    assert lib.rad_create(ctypes.byref(c), ctypes.byref(h)) == _lib.RAD_E_INVALID
    assert not h.value
    assert lib.rad_last_error(None)


def test_null_arguments(lib):
    assert lib.rad_create(None, None) == _lib.RAD_E_INVALID
    assert lib.rad_solve(None, None, None, 0, None) == _lib.RAD_E_INVALID
    assert lib.rad_load_tables(None, None, 0) == _lib.RAD_E_INVALID
    assert lib.rad_load_aerosols(None, None) == _lib.RAD_E_INVALID
    assert lib.rad_setaer(None, None, 0, None, None, None) == _lib.RAD_E_INVALID
    assert lib.rad_setaer_volc(None, None, None, 0, 0, None, 1, 1, 1, 1, 0, None, None, None) == _lib.RAD_E_INVALID
    assert lib.rad_grrad_clw(None, None, 1, 61, 0, 1, 1, 1e-12, None, None) == _lib.RAD_E_INVALID
    assert lib.rad_payne_albedo(None, None, None, None, 0, None, None, None) == _lib.RAD_E_INVALID
    lib.rad_destroy(None)

"""The C-ABI library loads and exports every symbol include/efl.h declares (no GPU needed)."""
import ctypes
import os
import re

import pytest

from bevy_eulerian_fluid_b200 import _capi as capi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(REPO, "include", "efl.h")).read()
    return sorted(set(re.findall(r"EFL_API\s+[\w\s\*]+?\b(efl_\w+)\s*\(", text)))


def test_header_declares_the_boundary():
    syms = header_symbols()
    for s in ("efl_create", "efl_destroy", "efl_step", "efl_set_obstacles", "efl_set_local_forces",
              "efl_set_sources", "efl_read_solid_forces", "efl_get_field", "efl_set_field", "efl_last_error"):
        assert s in syms


def test_library_exports_every_symbol():
    assert os.path.exists(capi.LIB_PATH), "libefl_b200.so not built"
    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_every_symbol_is_bound():
    bound = {"efl_" + k for k in capi.SIGNATURES}
    assert set(header_symbols()) <= bound


def test_struct_layouts():
    assert ctypes.sizeof(capi.SolidObstacle) == 176
    assert ctypes.sizeof(capi.Force) == 16
    assert ctypes.sizeof(capi.Source) == 32
    assert ctypes.sizeof(capi.SolidForce) == 16
    assert ctypes.sizeof(capi.StepStats) == 32


def test_abi_version_and_defaults():
    api = capi.load()
    assert api.abi_version() == 1
    c = capi.Config()
    assert api.default_config(256, 256, ctypes.byref(c)) == capi.OK
    d = capi.default_config(256, 256)
    assert bytes(c) == bytes(d)


def test_create_rejects_bad_length_unit_without_gpu():
    api = capi.load()
    c = capi.default_config(64, 64)
    c.length_unit = 0.0
    h = ctypes.c_void_p()
    st = api.create(ctypes.byref(c), ctypes.byref(h))
    assert st == capi.ERR_INVALID_ARGUMENT
    assert b"length_unit must be positive" in api.last_error(None)


def test_create_rejects_bad_sizes():
    api = capi.load()
    for nx, ny in ((60, 64), (8, 64), (64, 12)):
        c = capi.default_config(nx, ny)
        h = ctypes.c_void_p()
        assert api.create(ctypes.byref(c), ctypes.byref(h)) == capi.ERR_INVALID_ARGUMENT


def test_oracle_mirrors_the_boundary(oracle_api):
    for name in capi.SIGNATURES:
        if name in capi.PRODUCT_ONLY:
            continue
        assert hasattr(oracle_api.lib, "eflo_" + name)

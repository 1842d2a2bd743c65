"""TEST INFRASTRUCTURE: ctypes loader of the CPU oracle (liboracle_efl.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It binds the oracle's eflo_* entry points with the same
signatures as the product's efl_* ones, so bevy_eulerian_fluid_b200._capi.Sim
drives either backend.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle_efl.so")

_API = None


def build(force: bool = False):
    subprocess.run(["make", "-C", ORACLE_DIR] + (["-B"] if force else []), check=True,
                   stdout=subprocess.DEVNULL)


def load():
    global _API
    if _API is not None:
        return _API
    from bevy_eulerian_fluid_b200 import _capi
    if not os.path.exists(ORACLE_LIB):
        build()
    lib = ctypes.CDLL(ORACLE_LIB)
    api = _capi.Api(lib, "eflo_")
    lib.eflo_set_threads.argtypes = [ctypes.c_int32]
    lib.eflo_get_threads.restype = ctypes.c_int32
    lib.eflo_set_fim_serial.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    _API = api
    return api


def set_threads(n: int):
    load().lib.eflo_set_threads(int(n))


def get_threads() -> int:
    return int(load().lib.eflo_get_threads())


def set_fim_serial(sim, on: bool):
    load().lib.eflo_set_fim_serial(sim.h, 1 if on else 0)

"""Shared test helpers: scene setup on both backends, state transfer, comparison."""
from __future__ import annotations

import numpy as np

from bevy_eulerian_fluid_b200 import _capi as capi
from bevy_eulerian_fluid_b200 import scenes

FLOAT_FIELDS = [capi.FIELD_U, capi.FIELD_V, capi.FIELD_U1, capi.FIELD_V1, capi.FIELD_U_SOLID, capi.FIELD_V_SOLID,
                capi.FIELD_LEVELSET_AIR, capi.FIELD_LEVELSET_AIR1, capi.FIELD_LEVELSET_SOLID,
                capi.FIELD_DIVERGENCE, capi.FIELD_PRESSURE, capi.FIELD_GRAD_LEVELSET, capi.FIELD_AREA_FRACTION]
INT_FIELDS = [capi.FIELD_SOLID_ID, capi.FIELD_U_VALID, capi.FIELD_V_VALID, capi.FIELD_FIM_LABELS]
STATE_FIELDS = FLOAT_FIELDS + INT_FIELDS
FIELD_NAMES = {v: k for k, v in vars(capi).items() if k.startswith("FIELD_") and isinstance(v, int)}


def copy_state(src: capi.Sim, dst: capi.Sim, fields=STATE_FIELDS):
    for f in fields:
        dst.set(f, src.get(f))


def compare_fields(a: capi.Sim, b: capi.Sim, fields=STATE_FIELDS, rtol=0.0, atol=0.0, skip=()):
    """Returns a list of (field name, n_mismatch, max_abs_diff) for fields that differ."""
    bad = []
    for f in fields:
        if f in skip:
            continue
        x, y = a.get(f), b.get(f)
        if rtol == 0.0 and atol == 0.0:
            eq = np.array_equal(x, y, equal_nan=True)
            if not eq:
                d = np.abs(x.astype(np.float64) - y.astype(np.float64))
                bad.append((FIELD_NAMES[f], int(np.count_nonzero(d > 0)), float(np.nanmax(d))))
        else:
            ok = np.allclose(x, y, rtol=rtol, atol=atol, equal_nan=True)
            if not ok:
                d = np.abs(x.astype(np.float64) - y.astype(np.float64))
                lim = atol + rtol * np.abs(y.astype(np.float64))
                bad.append((FIELD_NAMES[f], int(np.count_nonzero(d > lim)), float(np.nanmax(d))))
    return bad


def rel_max_err(x: np.ndarray, y: np.ndarray) -> float:
    """max |x - y| / max |y| (the relative max-error of the parity contract)."""
    y64 = y.astype(np.float64)
    den = float(np.max(np.abs(y64))) or 1.0
    return float(np.max(np.abs(x.astype(np.float64) - y64))) / den


def small_coupled(n=128, method=capi.PROJECTION_GAUSS_SEIDEL, tolerance=1e-5, n_per_shape=2, seed=0xC2):
    sc = scenes.coupled(n, tolerance=tolerance, method=method, n_per_shape=n_per_shape, seed=seed)
    return sc


def make_pair(scene, oracle_api, gpu_api):
    return scene.make(oracle_api), scene.make(gpu_api)

"""The allocation-free residual-norm entry point (efl_residual_norms_noalloc).

It serves callers that cannot let the library allocate device memory -- an
engine that owns every GPU buffer through its own arena, or a frame loop
that forbids allocation once running.  The GPU test feeds it the pressure,
divergence, level set and face fractions of a running simulation (caller-
owned device planes) and checks, on two calls in a row with the state
changed in between, that it returns the same relative residual and norms as
the existing efl_residual entry point, within the FP64 tolerance the other
residual tests use.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from bevy_eulerian_fluid_b200 import _capi as capi
from bevy_eulerian_fluid_b200 import scenes

TOL = 1e-12  # FP64 norms summed in a different block order


def _call(api, sim, out_ptr, dx, dt, rho, nx=None, ny=None):
    p, pitch = sim.device_ptr(capi.FIELD_PRESSURE)
    d, _ = sim.device_ptr(capi.FIELD_DIVERGENCE)
    phi, _ = sim.device_ptr(capi.FIELD_LEVELSET_AIR)
    fu, _ = sim.device_ptr(capi.FIELD_AREA_FRACTION_U)
    fv, _ = sim.device_ptr(capi.FIELD_AREA_FRACTION_V)
    return api.residual_norms_noalloc(p, d, phi, fu, fv, nx or sim.nx, ny or sim.ny, pitch, dx, dt, rho,
                                      out_ptr, sim.stream())


@pytest.mark.gpu
def test_noalloc_matches_efl_residual_twice():
    import torch

    api = capi.load()
    sc = scenes.coupled(128, tolerance=0.0, n_per_shape=2)
    sim = sc.make(api)
    for _ in range(3):
        sim.step(sc.dt)
    dx = float(np.float32(1.0) / np.float32(sc.cfg.length_unit))
    out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda")
    # The fill runs on torch's stream and the entry point on the simulation's
    # non-blocking stream: finish the fill before the first call writes `out`.
    torch.cuda.synchronize()
    for call in range(2):
        st = _call(api, sim, out.data_ptr(), dx, sc.dt, sc.cfg.rho)
        assert st == capi.OK, (api.last_error(None) or b"").decode()
        sim.synchronize()
        got = out.cpu().numpy()
        rel, nr, nb = sim.residual()
        assert rel > 0.0 and nb > 0.0
        assert abs(got[0] - rel) <= TOL * max(1.0, rel), (call, got, rel)
        assert abs(got[1] - nr) <= TOL * max(1.0, nr), (call, got, nr)
        assert abs(got[2] - nb) <= TOL * max(1.0, nb), (call, got, nb)
        sim.step(sc.dt)  # new state for the second call
    sim.close()


def test_noalloc_rejects_oversize_grid():
    api = capi.load()
    fake = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    st = api.residual_norms_noalloc(fake, fake, fake, fake, fake, 8192, 4096, 8196 * 4, 0.1, 1 / 60, 99.7,
                                    fake, None)
    assert st == capi.ERR_INVALID_ARGUMENT
    assert b"exceeds the fixed scratch limit" in api.last_error(None)

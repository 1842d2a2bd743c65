"""Row-slab split of one domain's pressure solve (bevy_eulerian_fluid_b200/slab.py), run as torch.distributed
ranks, against the unsplit oracle solve of the same system.

The system is the projection of a dam break with a static body at the centre (the cuts run through the
water, next to solid fractions and ghost-fluid faces), taken after a few steps: the oracle's level set, face fractions,
divergence and previous pressure right before EFL_STAGE_PROJECTION, and the oracle's tolerance-driven RBGS
solve of it (EFL_STAGE_PROJECTION) as the answer.

CPU (gloo, world sizes 2 and 3, uneven slabs): the host driver with the numpy slab restatement
(oracle/slab_ref.py) reproduces the unsplit solve exactly: iteration count, initial and final relative
residual, and the pressure bit for bit.  A driver that skips the correction's halo exchange does not.
GPU (gloo, world size 2, both ranks on one device: the slabs' kernels never wait on each other, the exchange
runs on the host): the CUDA slabs (efl_slab_*) give the same iteration count and pressure bit for bit; the
residual agrees to 1e-12 (per-row sums are trees on the GPU, sequential in the oracle).
"""
from __future__ import annotations

import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from bevy_eulerian_fluid_b200 import _capi as capi
from bevy_eulerian_fluid_b200 import scenes
from bevy_eulerian_fluid_b200.slab import slab_rows

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def projection_case(api, n: int = 96, steps: int = 6):
    """Fields right before the projection of step `steps + 1` of the scale scene at n^2 (a dam break over 60 % of
    the height with a static circle at the centre, so the middle cuts run through water and past the body),
    solved by tolerance-driven RBGS, and the unsplit solve's result."""
    sc = scenes.scale(n)
    p = sc.cfg.projection
    p.method, p.tolerance, p.max_iterations, p.check_interval = capi.PROJECTION_GAUSS_SEIDEL, 1e-5, 20000, 16
    sim = sc.make(api)
    sim.step(sc.dt)  # init sequence
    for _ in range(steps):
        sim.step(sc.dt)
    for stage in range(capi.STAGE_UPDATE_SOLID, capi.STAGE_PROJECTION):
        sim.run_stage(stage, sc.dt)
    fields = {"levelset_air": sim.get(capi.FIELD_LEVELSET_AIR), "area_fraction": sim.get(capi.FIELD_AREA_FRACTION),
              "divergence": sim.get(capi.FIELD_DIVERGENCE), "pressure": sim.get(capi.FIELD_PRESSURE)}
    st = sim.run_stage(capi.STAGE_PROJECTION, sc.dt)
    expect = {"iterations": int(st.pressure_iterations), "r0": float(st.residual_initial), "r1": float(st.residual),
              "pressure": sim.get(capi.FIELD_PRESSURE)}
    p = sc.cfg.projection
    params = {"nx": n, "ny": n, "dx": float(np.float32(1.0) / np.float32(sc.cfg.length_unit)), "dt": float(sc.dt),
              "rho": float(sc.cfg.rho), "sor_weight": float(p.sor_weight), "tolerance": float(p.tolerance),
              "max_iterations": int(p.max_iterations), "check_interval": int(p.check_interval)}
    sim.close()
    return fields, expect, params


def _worker(rank, world, port, backend_kind, fields, params, skip_d, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    if REPO not in sys.path:
        sys.path.insert(0, REPO)
    import torch.distributed as dist

    from bevy_eulerian_fluid_b200 import slab as slab_mod
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        nx, ny = params["nx"], params["ny"]
        row0, rows = slab_rows(ny, world, rank)
        args = (nx, ny, row0, rows, params["dx"], params["dt"], params["rho"], params["sor_weight"])
        if backend_kind == "numpy":
            from oracle.slab_ref import SlabRef
            be = SlabRef(*args)
        else:
            be = slab_mod.CudaSlab(capi.load(), *args, device=0)

        class SkipD(slab_mod.RowSlabSolver):
            def exchange(self, field):
                if field != slab_mod.SLAB_D:
                    super().exchange(field)

        solver = (SkipD if skip_d else slab_mod.RowSlabSolver)(be, nx, ny)
        sl = slice(row0, row0 + rows)
        solver.setup(fields["levelset_air"][sl], fields["area_fraction"][sl], fields["divergence"][sl],
                     fields["pressure"][sl])
        st = solver.solve(params["tolerance"], params["max_iterations"], params["check_interval"])
        p = solver.gather_pressure()
        out[rank] = {"iterations": st.iterations, "r0": st.residual_initial, "r1": st.residual,
                     "converged": st.converged, "pressure": p.astype(np.float32), "rows": (row0, rows),
                     "exchanges": solver.exchanges}
        be.close()
    finally:
        dist.destroy_process_group()


def run_ranks(world, backend_kind, fields, params, skip_d=False):
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, backend_kind, fields, params, skip_d, out), nprocs=world, join=True)
        return dict(out)


def test_slab_rows_cover_the_domain():
    for ny in (1, 7, 96, 4096):
        for world in (1, 2, 3, 8):
            if world > ny:
                with pytest.raises(ValueError):
                    slab_rows(ny, world, 0)
                continue
            parts = [slab_rows(ny, world, r) for r in range(world)]
            assert parts[0][0] == 0
            for (a0, an), (b0, _) in zip(parts, parts[1:]):
                assert a0 + an == b0
            assert parts[-1][0] + parts[-1][1] == ny
            assert max(p[1] for p in parts) - min(p[1] for p in parts) <= 1


@pytest.fixture(scope="module")
def case(oracle_api):
    return projection_case(oracle_api)


@pytest.mark.parametrize("world", [2, 3])
def test_numpy_slabs_reproduce_unsplit_oracle_solve(case, world):
    fields, expect, params = case
    ls = fields["levelset_air"]
    cuts = [slab_rows(params["ny"], world, r)[0] for r in range(1, world)]
    assert any(np.any((ls[c - 1] < 0) & (ls[c] < 0)) for c in cuts)  # some cut runs through the water
    assert expect["iterations"] >= 64  # several check blocks, so the exchanges are exercised many times
    res = run_ranks(world, "numpy", fields, params)
    assert sorted(res) == list(range(world))
    for r in range(world):
        got = res[r]
        assert got["iterations"] == expect["iterations"], (r, got["iterations"], expect["iterations"])
        assert got["r0"] == expect["r0"] and got["r1"] == expect["r1"], (got["r0"], got["r1"], expect)
        assert got["converged"]
        assert np.array_equal(got["pressure"], expect["pressure"]), r
    # 1 level-set exchange, one x exchange per residual, one d exchange per half-sweep
    blocks = expect["iterations"] // params["check_interval"]
    assert res[0]["exchanges"] == 1 + (blocks + 1) + 2 * expect["iterations"]


def test_missing_correction_exchange_is_detected(case):
    """The same driver with the correction's halo exchange left out (a mistake planted on the CPU side):
    the slabs no longer reproduce the unsplit solve."""
    fields, expect, params = case
    cut = slab_rows(params["ny"], 3, 2)[0]
    ls = fields["levelset_air"]
    assert np.any((ls[cut - 1] < 0) & (ls[cut] < 0))  # fluid on both sides of the lower cut
    res = run_ranks(3, "numpy", fields, params, skip_d=True)
    got = res[0]
    assert got["iterations"] != expect["iterations"] or not np.array_equal(got["pressure"], expect["pressure"])


def test_slab_create_rejects_bad_rows():
    """Argument checks of efl_slab_create run before any device call."""
    import ctypes as C
    api = capi.load()
    h = C.c_void_p()
    for nx, ny, row0, rows in ((64, 64, 0, 0), (64, 64, 60, 8), (0, 64, 0, 8)):
        d = capi.SlabDesc(0, nx, ny, row0, rows, 1.0, 1.0 / 60, 1.0, 1.9)
        assert api.slab_create(C.byref(d), C.byref(h)) == capi.ERR_INVALID_ARGUMENT
    d = capi.SlabDesc(0, 64, 64, 0, 8, 1.0, 1.0 / 60, 1.0, 2.5)
    assert api.slab_create(C.byref(d), C.byref(h)) == capi.ERR_INVALID_ARGUMENT
    assert b"sor_weight" in api.last_error(None)


@pytest.mark.gpu
def test_cuda_slabs_reproduce_unsplit_oracle_solve(case):
    fields, expect, params = case
    res = run_ranks(2, "cuda", fields, params)
    for r in range(2):
        got = res[r]
        assert got["iterations"] == expect["iterations"], (r, got["iterations"], expect["iterations"])
        assert abs(got["r1"] - expect["r1"]) <= 1e-12 * expect["r1"]
        assert abs(got["r0"] - expect["r0"]) <= 1e-12 * expect["r0"]
        assert np.array_equal(got["pressure"], expect["pressure"]), r

"""Bounded device waits that run out: the error path of every spin-wait.

The cooperative pressure solves wait on a grid barrier and the TMA sweep
waits on mbarriers for its tile copies.  Each wait has a poll limit (about a
second by default) after which the kernel stops waiting, records an error
flag and leaves; the host turns the flag into EFL_ERR_CUDA with a message
naming the wait.  These tests set the limit to one poll, so the wait runs
out on the first poll that finds it incomplete: no kernel faults or hangs,
every wait returns.  A fresh handle (or the same handle with the default
limits restored) then steps bit-exactly like the CPU oracle.
"""
import pytest

from bevy_eulerian_fluid_b200 import _capi as capi
from bevy_eulerian_fluid_b200 import scenes

from .helpers import compare_fields

pytestmark = pytest.mark.gpu


def _expect_cuda_error(fn, words):
    with pytest.raises(capi.EflError) as ei:
        fn()
    assert ei.value.status == capi.ERR_CUDA, str(ei.value)
    assert words in str(ei.value), str(ei.value)


def test_grid_barrier_runs_out(oracle_api, gpu_api):
    """Persistent mixed-precision solve (one cooperative launch, 32 CTAs at 256^2): a one-poll barrier limit."""
    sc = scenes.coupled(256, tolerance=1e-5, n_per_shape=2)
    g = sc.make(gpu_api)
    g.step(sc.dt)  # init sequence: no solve
    g.set_wait_limits(barrier_polls=1)
    _expect_cuda_error(lambda: g.step(sc.dt), "grid barrier timed out")
    g.close()
    # A fresh handle with the default limits: converged, bit-exact with the oracle.
    g, o = sc.make(gpu_api), sc.make(oracle_api)
    for _ in range(3):
        sg, so = g.step(sc.dt), o.step(sc.dt)
        assert sg.pressure_iterations == so.pressure_iterations
    assert sg.converged and sg.residual <= 1e-5
    assert not compare_fields(g, o)
    g.close()
    o.close()


def test_fixed_count_sweep_barrier_runs_out(oracle_api, gpu_api):
    """Fixed-count f32 sweeps as one cooperative launch (grids of at most one tile per SM, here 256^2): a
    one-poll grid-barrier limit; the flag is reported at the next synchronisation."""
    sc = scenes.dam_break(256)
    g = sc.make(gpu_api)
    g.step(sc.dt)  # init sequence
    g.set_wait_limits(barrier_polls=1)
    g.step(sc.dt)
    _expect_cuda_error(g.synchronize, "grid barrier timed out")
    g.set_wait_limits(0, 0)
    g.close()
    g, o = sc.make(gpu_api), sc.make(oracle_api)
    for _ in range(4):
        g.step(sc.dt)
        o.step(sc.dt)
    g.synchronize()
    assert not compare_fields(g, o)
    g.close()
    o.close()


def test_mbarrier_wait_runs_out(oracle_api, gpu_api):
    """Fixed-count f32 sweep through the TMA-streamed kernel (grids of more tiles than SMs, here 1024^2): a
    one-poll mbarrier limit."""
    sc = scenes.dam_break(1024)
    g = sc.make(gpu_api)
    g.step(sc.dt)  # init sequence
    g.set_wait_limits(mbarrier_polls=1)
    g.step(sc.dt)  # the sweep's CTAs give up; the flag is reported at the next synchronisation
    _expect_cuda_error(g.synchronize, "mbarrier wait timed out")
    # The flag is cleared once reported; default limits restored, the same handle steps on.
    g.set_wait_limits(0, 0)
    g.step(sc.dt)
    g.synchronize()
    g.close()
    g, o = sc.make(gpu_api), sc.make(oracle_api)
    for _ in range(4):
        g.step(sc.dt)
        o.step(sc.dt)
    g.synchronize()
    assert not compare_fields(g, o)
    g.close()
    o.close()


def test_batched_grid_barrier_runs_out(gpu_api):
    """The batched cooperative solve (all simulations' tiles in one launch): a one-poll barrier limit."""
    b = scenes.batch(6, steps=2, seed=0xC4, shapes=[(64, 64), (128, 64), (128, 128), (192, 128)])
    batch = capi.Batch(gpu_api, b.configs())
    b.setup(batch.sims)
    batch.step(b.scenes[0].dt)  # init sequences
    batch.set_wait_limits(1)
    _expect_cuda_error(lambda: batch.step(b.scenes[0].dt), "grid barrier timed out")
    batch.set_wait_limits(0)
    batch.close()
    batch = capi.Batch(gpu_api, b.configs())
    b.setup(batch.sims)
    for _ in range(3):
        stats = batch.step(b.scenes[0].dt)
    assert all(s.converged for s in stats)
    assert all(0 <= s.residual <= 1e-5 for s in stats)
    batch.close()


def test_wait_limit_arguments(gpu_api):
    sc = scenes.dam_break(64)
    g = sc.make(gpu_api)
    with pytest.raises(capi.EflError) as ei:
        g.set_wait_limits(1 << 41, 0)
    assert ei.value.status == capi.ERR_INVALID_ARGUMENT
    g.set_wait_limits(0, 0)
    g.close()

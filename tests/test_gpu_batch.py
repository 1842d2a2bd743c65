"""Batched stepping (efl_batch_*): every simulation of a batch equals the
same simulation stepped alone by the CPU oracle.

The batch's tolerance-driven solves share one cooperative launch; each
simulation still runs its own mixed-precision refinement, so iteration counts
are equal and the fields bit-exact.
"""
import numpy as np
import pytest

from bevy_eulerian_fluid_b200 import _capi as capi
from bevy_eulerian_fluid_b200 import scenes

from .helpers import compare_fields

pytestmark = pytest.mark.gpu

SMALL_SHAPES = [(64, 64), (128, 64), (96, 96), (128, 128), (192, 128)]


def _small_batch(n=6, seed=0xC4):
    b = scenes.batch(n, steps=6, seed=seed, shapes=SMALL_SHAPES)
    b.force_every = 2
    return b


def _step_both(b, batch, oracles, frames):
    for k in range(frames):
        for i, o in enumerate(oracles):
            f = b.forces(i, k)
            if f:
                o.set_local_forces(f)
                batch[i].set_local_forces(f)
        stats_g = batch.step(b.scenes[0].dt)
        stats_o = [o.step(b.scenes[0].dt) for o in oracles]
        for i, (sg, so) in enumerate(zip(stats_g, stats_o)):
            assert sg.initialized_only == so.initialized_only, (k, i)
            assert sg.pressure_iterations == so.pressure_iterations, (k, i)
            assert sg.converged == so.converged, (k, i)
            if so.residual >= 0:
                assert abs(sg.residual - so.residual) <= 1e-9 * max(1.0, abs(so.residual)), (k, i)


def test_batch_matches_oracle_alone(oracle_api, gpu_api):
    b = _small_batch()
    # One member takes the per-simulation path (fixed multigrid), one carries bodies.
    b.scenes[1].cfg.projection.method = capi.PROJECTION_MULTIGRID
    b.scenes[1].cfg.projection.tolerance = 0.0
    bodies = scenes.random_bodies(1, min(b.scenes[0].cfg.nx, b.scenes[0].cfg.ny), 0xB0)
    b.scenes[0].bodies = bodies
    oracles = [sc.make(oracle_api) for sc in b.scenes]
    with capi.Batch(gpu_api, b.configs()) as batch:
        b.setup(batch.sims)
        batch[0].set_obstacles([x.to_obstacle(i) for i, x in enumerate(bodies)])
        _step_both(b, batch, oracles, 5)
        for i, (g, o) in enumerate(zip(batch.sims, oracles)):
            bad = compare_fields(g, o)
            assert not bad, (i, bad)
        assert np.array_equal(batch[0].force_bins(), oracles[0].force_bins())


def test_batch_stats_and_handles(gpu_api):
    b = _small_batch(3)
    with capi.Batch(gpu_api, b.configs()) as batch:
        b.setup(batch.sims)
        st = batch.step(b.scenes[0].dt)
        assert all(s.initialized_only == 1 for s in st)
        st = batch.step(b.scenes[0].dt)
        assert all(s.initialized_only == 0 and s.converged and s.pressure_iterations > 0 for s in st)
        assert all(0 <= s.residual <= 1e-5 for s in st)
        assert len(batch) == 3 and batch[2].nx == b.scenes[2].cfg.nx


def test_batch_rejects_bad_index(gpu_api):
    b = _small_batch(2)
    with capi.Batch(gpu_api, b.configs()) as batch:
        import ctypes as C
        h = C.c_void_p()
        assert gpu_api.batch_sim(batch.h, 5, C.byref(h)) == capi.ERR_INVALID_ARGUMENT


def test_batch_fast_path_graphs_match_oracle(oracle_api, gpu_api):
    """All members batched: the stages around the solve run as captured CUDA
    graphs (recaptured when local forces appear, replayed after); every member
    still equals the oracle alone."""
    b = _small_batch(5, seed=0xC5)
    oracles = [sc.make(oracle_api) for sc in b.scenes]
    with capi.Batch(gpu_api, b.configs()) as batch:
        b.setup(batch.sims)
        _step_both(b, batch, oracles, 8)
        for i, (g, o) in enumerate(zip(batch.sims, oracles)):
            bad = compare_fields(g, o)
            assert not bad, (i, bad)


@pytest.mark.parametrize("coarse", [4, 1])
def test_batch_with_network_matches_single_sims(gpu_api, coarse):
    """efl_batch_attach_unet: every simulation's solve is warm-started by the network inside the batch step
    (coarsening 4: one forward over a canvas that packs the simulations' coarse grids, 8-pixel gaps kept zero
    between them; coarsening 1: one forward workspace per simulation, forwards side by side); each simulation
    still equals the same simulation stepped alone by efl_step with the network attached -- bit-exact fields,
    equal iteration counts -- and every solve still reaches the tolerance."""
    b = _small_batch(5, seed=0xB1)
    net = capi.UNet(gpu_api, 192, 192, seed=7)
    rng = np.random.default_rng(1)
    p = net.get_params()
    net.set_params(p + rng.standard_normal(p.size).astype(np.float32) * 0.02)  # a non-zero head: a real warm start
    net.set_coarsening(coarse)
    singles = [sc.make(gpu_api) for sc in b.scenes]
    for s in singles:
        net.attach(s, warm_start=True)
    with capi.Batch(gpu_api, b.configs()) as batch:
        b.setup(batch.sims)
        batch.attach_unet(net)
        cw, ch = batch.unet_canvas()
        assert (cw > 0) == (coarse > 1), (cw, ch)
        dts = [1.0, 1.0, 0.75, 0.75, 1.0]  # x the scene's dt: a new dt re-derives the warm start's descriptors
        for k in range(5):
            for i, s in enumerate(singles):
                f = b.forces(i, k)
                if f:
                    s.set_local_forces(f)
                    batch[i].set_local_forces(f)
            dt = b.scenes[0].dt * dts[k]
            gst = batch.step(dt)
            sst = [s.step(dt) for s in singles]
            for i, (g, s) in enumerate(zip(gst, sst)):
                assert g.pressure_iterations == s.pressure_iterations, (k, i)
                assert g.converged == s.converged == 1, (k, i)
                assert abs(g.residual - s.residual) <= 1e-9 * max(1.0, abs(s.residual)), (k, i)
        for i, (g, s) in enumerate(zip(batch.sims, singles)):
            bad = compare_fields(g, s)
            assert not bad, (i, bad)
        batch.attach_unet(net, warm_start=False)
        assert batch.unet_canvas() == (0, 0)
    for s in singles:
        s.close()
    net.close()

"""Parity at the benchmark configurations' own sizes, GPU next to the CPU oracle.

  C1  256^2 dam break (examples/water_surface.rs), Gauss-Seidel 20 at weight
      1.9, FIM(10), 600 steps through efl_step (graph replay): every field
      bit-exact and the fluid volume equal every 50 steps.
  C2  512^2, 24 bodies from seed 0xC2, jump flooding, RBGS to 1e-5 relative
      residual, the two-way coupling loop (force read-back, host rigid
      integration, obstacle upload) for 20 steps: equal iteration counts and
      force bins every step, fields and jump-flood seeds bit-exact at the end.
  C4  one batch of the real size set (128^2, 256x128, 256^2, 384x256, 512^2,
      768x512) with droplets and local forces, 5 frames, once per tile
      configuration of the batched solve: every simulation equals the oracle
      stepping it alone.

The oracle runs on every host thread; these cases take tens of seconds of
CPU time each.
"""
import copy

import numpy as np
import pytest

from bevy_eulerian_fluid_b200 import _capi as capi
from bevy_eulerian_fluid_b200 import scenes
from bevy_eulerian_fluid_b200.plugin import pack_obstacles
from bevy_eulerian_fluid_b200.rigid import RigidWorld

from .helpers import compare_fields, make_pair

pytestmark = pytest.mark.gpu


def test_c1_dam_break_256_600_steps(oracle_api, gpu_api):
    sc = scenes.dam_break(256)
    o, g = make_pair(sc, oracle_api, gpu_api)
    o.step(sc.dt)
    g.step(sc.dt)  # init sequence
    for k in range(1, 601):
        so, sg = o.step(sc.dt), g.step(sc.dt)
        assert so.pressure_iterations == sg.pressure_iterations == 20
        if k % 50 == 0:
            bad = compare_fields(g, o)
            assert not bad, (k, bad)
            assert g.fluid_volume() == o.fluid_volume(), k
    o.close()
    g.close()


def _coupled_arm(api, sc):
    sim = sc.make(api)
    rigid = RigidWorld(copy.deepcopy(list(sc.bodies)), (sc.cfg.nx, sc.cfg.ny), gravity=9.8 * scenes.LENGTH_UNIT,
                       grid_length=1.0 / scenes.LENGTH_UNIT)
    return sim, rigid


def test_c2_coupled_512_twenty_coupled_steps(oracle_api, gpu_api):
    sc = scenes.coupled(512)
    assert len(sc.bodies) == 24
    arms = [_coupled_arm(oracle_api, sc), _coupled_arm(gpu_api, sc)]
    for sim, _ in arms:
        assert sim.step(sc.dt).initialized_only == 1
    for k in range(20):
        stats, bins = [], []
        for sim, rigid in arms:
            st = sim.step(sc.dt)
            rigid.apply_fluid_forces(sim.solid_forces(), sc.dt)
            rigid.step(sc.dt)
            sim.set_obstacles(pack_obstacles(rigid.bodies))
            stats.append(st)
            bins.append(sim.force_bins())
        so, sg = stats
        assert so.pressure_iterations == sg.pressure_iterations, (k, so.as_dict(), sg.as_dict())
        assert so.converged == sg.converged, k
        assert abs(so.residual - sg.residual) <= 1e-9 * max(1.0, abs(so.residual)), k
        assert np.array_equal(bins[0], bins[1]), k
    o, g = arms[0][0], arms[1][0]
    assert not compare_fields(g, o)
    assert np.array_equal(g.get(capi.FIELD_JFA_SEEDS), o.get(capi.FIELD_JFA_SEEDS))
    for sim, _ in arms:
        sim.close()


def _size_set_batch():
    """One simulation per size of the C4 set, each generated like a C4 member, with forces every 2 frames."""
    members = [scenes.batch(1, seed=0xC4 + i, shapes=[shape]).scenes[0] for i, shape in enumerate(scenes.BATCH_SHAPES)]
    b = scenes.BatchScene("c4_size_set", members, 0xC4, steps=5)
    b.force_every = 2
    return b


FRAMES = 5


@pytest.fixture(scope="module")
def c4_oracle_run(oracle_api):
    """Per frame and simulation: (iterations, converged, residual); final fields of every simulation."""
    b = _size_set_batch()
    sims = [sc.make(oracle_api) for sc in b.scenes]
    stats = []
    for k in range(FRAMES + 1):
        row = []
        for i, sim in enumerate(sims):
            f = b.forces(i, k)
            if f:
                sim.set_local_forces(f)
            st = sim.step(b.scenes[0].dt)
            row.append((st.initialized_only, st.pressure_iterations, st.converged, st.residual))
        stats.append(row)
    return b, sims, stats


@pytest.mark.parametrize("tile_config", [0, 1, 2, 3])
def test_c4_size_set_batch_each_tile_config(gpu_api, c4_oracle_run, tile_config):
    b, oracles, ostats = c4_oracle_run
    assert {(sc.cfg.nx, sc.cfg.ny) for sc in b.scenes} == set(scenes.BATCH_SHAPES)
    batch = capi.Batch(gpu_api, b.configs())
    b.setup(batch.sims)
    batch.set_tiles(tile_config)
    for k in range(FRAMES + 1):
        for i in range(len(b.scenes)):
            f = b.forces(i, k)
            if f:
                batch[i].set_local_forces(f)
        gst = batch.step(b.scenes[0].dt)
        for i, (sg, so) in enumerate(zip(gst, ostats[k])):
            assert sg.initialized_only == so[0], (k, i)
            assert sg.pressure_iterations == so[1], (k, i, sg.pressure_iterations, so[1])
            assert sg.converged == so[2], (k, i)
            if so[3] >= 0:
                assert abs(sg.residual - so[3]) <= 1e-9 * max(1.0, abs(so[3])), (k, i)
    (tx, ty, kk), _ = batch.tiles()
    assert (tx, ty, kk) == [(64, 32, 2), (64, 32, 4), (32, 32, 2), (64, 32, 8)][tile_config]
    for i, o in enumerate(oracles):
        bad = compare_fields(batch[i], o)
        assert not bad, (i, bad)
    batch.close()

"""Host-side logic of the plugin-API mirror (no GPU, no compute calls)."""
import math
import warnings

import numpy as np
import pytest

from bevy_eulerian_fluid_b200 import _capi as capi
from bevy_eulerian_fluid_b200 import scenes
from bevy_eulerian_fluid_b200.plugin import (Collider, FastIterativeMethodConfig, FluidPlugin, FluidSourceShape,
                                             GaussSeidelConfig, MultiGridConfig, ProjectionMethod,
                                             ReinitializeMethod, RigidBody, RigidBodyKind, pack_obstacles)
from bevy_eulerian_fluid_b200.rigid import RigidWorld


def test_fluid_plugin_rejects_non_positive_length_unit():
    with pytest.raises(ValueError, match="length_unit must be positive value."):
        FluidPlugin(0.0)
    assert FluidPlugin(10.0).grid_length == pytest.approx(0.1)


def test_projection_and_reinit_display_and_c_structs():
    assert str(ProjectionMethod.Jacobi()) == "Jacobi"
    assert str(ProjectionMethod.GaussSeidel(GaussSeidelConfig(20))) == "Gauss-Seidel(20)"
    assert str(ProjectionMethod.MultiGrid(MultiGridConfig())) == "Multigrid(2-3-2)"
    assert str(ReinitializeMethod.JumpFlooding()) == "Jump Flooding"
    assert str(ReinitializeMethod.FastIterative(FastIterativeMethodConfig(7))) == "Fast Iterative(7)"
    p = ProjectionMethod.MultiGrid().to_c()
    assert (p.method, p.mg_pre, p.mg_post, p.mg_coarsest) == (capi.PROJECTION_MULTIGRID, 2, 2, 3)
    assert ProjectionMethod.default().to_c().gs_iterations == 20
    assert abs(ProjectionMethod.default().to_c().sor_weight - 1.9) < 1e-6
    r = ReinitializeMethod.default().to_c()
    assert (r.method, r.fim_iterations) == (capi.REINIT_FAST_ITERATIVE, 10)


def test_source_shapes():
    c = FluidSourceShape.Circle(3.0)
    a = FluidSourceShape.Aabb((4.0, 5.0))
    assert (c.to_vec2(), c.shape_type_digit()) == ((3.0, 0.0), 0)
    assert (a.to_vec2(), a.shape_type_digit()) == ((4.0, 5.0), 1)


def test_obstacle_packing_layout_and_inverse():
    b = RigidBody(Collider.rectangle(10.0, 4.0), (12.0, -3.0), 0.7, (1.0, 2.0), 0.3)
    o = pack_obstacles([b])[0]
    assert o.shape == capi.SHAPE_RECTANGLE and tuple(o.values[:2]) == (5.0, 2.0)
    m = np.array(o.transform, np.float64).reshape(4, 4).T  # column-major
    inv = np.array(o.inverse_transform, np.float64).reshape(4, 4).T
    assert np.allclose(m @ inv, np.eye(4), atol=1e-6)
    assert m[0, 3] == pytest.approx(12.0) and m[1, 3] == pytest.approx(-3.0)
    assert (o.linear_velocity[0], o.linear_velocity[1], o.angular_velocity) == pytest.approx((1.0, 2.0, 0.3))


def test_batched_packing_equals_per_body_packing():
    """pack_obstacles (all bodies at once) writes the same bytes as RigidBody.to_obstacle per body, for every
    collider kind, over a run of the coupled scene's rigid integration."""
    import copy
    sc = scenes.coupled(256)
    bodies = copy.deepcopy(list(sc.bodies)) + [RigidBody(Collider.triangle((0, 0), (3, 0), (0, 2)), (5.0, 6.0), 1.1)]
    rigid = RigidWorld(bodies, (256, 256), gravity=9.8 * scenes.LENGTH_UNIT, grid_length=1.0 / scenes.LENGTH_UNIT)
    forces = np.random.default_rng(3).standard_normal((capi.MAX_SOLIDS, 3)).astype(np.float32) * 0.01
    for _ in range(20):
        rigid.apply_fluid_forces(forces, sc.dt)
        rigid.step(sc.dt)
        a = pack_obstacles(rigid.bodies)
        b = [x.to_obstacle(i) for i, x in enumerate(rigid.bodies)]
        assert len(a) == len(b) and bytes(a) == bytes((capi.SolidObstacle * len(b))(*b))
    assert pack_obstacles([]) == []


def test_collider_areas():
    assert Collider.circle(2.0).area() == pytest.approx(math.pi * 4)
    assert Collider.rectangle(2.0, 3.0).area() == pytest.approx(6.0)
    assert Collider.triangle((0, 0), (2, 0), (0, 2)).area() == pytest.approx(2.0)
    assert Collider.capsule(1.0, 4.0).area() == pytest.approx(math.pi + 8.0)


def test_scenes_are_deterministic():
    a, b = scenes.coupled(512), scenes.coupled(512)
    assert len(a.bodies) == 24
    assert [bytes(pack_obstacles(a.bodies)[i]) for i in range(24)] == \
        [bytes(pack_obstacles(b.bodies)[i]) for i in range(24)]
    shapes = [x.collider.shape for x in a.bodies]
    assert shapes == [0] * 6 + [1] * 6 + [2] * 6 + [4] * 6
    for x in a.bodies:
        assert -256 < x.position[0] < 256 and 0 < x.position[1] < 256
        assert 0.5 * scenes.RHO <= x.density <= 2.0 * scenes.RHO
    d = scenes.dam_break(256)
    s = d.oneshot[0]
    assert (s.center[0], s.center[1], s.data[0], s.data[1]) == pytest.approx((0.0, -51.2, 128.0, 76.8))
    phi, b = scenes.microbench_inputs(64)
    assert abs(float(b.astype(np.float64).mean())) < 1e-6 and np.all(phi == -1)


def test_rigid_world_gravity_and_walls():
    body = RigidBody(Collider.circle(5.0), (0.0, 0.0), density=1.0)
    w = RigidWorld([body], (64, 64), gravity=98.0, grid_length=0.1)
    for _ in range(600):
        w.step(1 / 60)
    assert body.position[1] == pytest.approx(-32 + 1 + 5)  # rests on the floor
    assert body.linear_velocity[1] == 0.0
    static = RigidBody(Collider.circle(5.0), (10.0, 10.0), kind=RigidBodyKind.Static)
    w2 = RigidWorld([static], (64, 64), gravity=98.0, grid_length=0.1)
    w2.step(1 / 60)
    assert static.position == (10.0, 10.0)


def test_rigid_world_applies_fluid_force_like_the_reference():
    """forces_to_solid_readback: force * dt / grid_length, y flipped, torque negated."""
    body = RigidBody(Collider.circle(2.0), (0.0, 0.0), density=1.0)
    w = RigidWorld([body], (512, 512), gravity=0.0, grid_length=0.1)
    w.apply_fluid_forces(np.array([[10.0, 20.0, 5.0]]), 0.1)
    w.step(0.1)
    m = math.pi * 4
    assert body.linear_velocity[0] == pytest.approx(10.0 * 0.1 / 0.1 / m * 0.1)
    assert body.linear_velocity[1] == pytest.approx(-20.0 * 0.1 / 0.1 / m * 0.1)
    assert body.angular_velocity < 0


def test_default_config_matches_reference_defaults():
    c = capi.default_config(256, 128)
    assert (c.nx, c.ny, c.length_unit, c.rho) == (256, 128, 1.0, 1.0)
    assert tuple(c.gravity) == pytest.approx((0.0, 9.8))
    assert list(c.transform) == [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1]


def test_batch_scene_matches_c4_spec():
    from bevy_eulerian_fluid_b200 import _capi as capi
    from bevy_eulerian_fluid_b200 import scenes
    b = scenes.batch(96)
    again = scenes.batch(96)
    assert [(s.cfg.nx, s.cfg.ny) for s in b.scenes] == [(s.cfg.nx, s.cfg.ny) for s in again.scenes]
    shapes = {(s.cfg.nx, s.cfg.ny) for s in b.scenes}
    assert shapes <= set(scenes.BATCH_SHAPES) and len(shapes) == 6
    for s in b.scenes:
        nx, ny = s.cfg.nx, s.cfg.ny
        pool, drops = s.oneshot[0], s.oneshot[1:]
        depth = 2 * pool.data[1]
        assert 0.2 * ny <= depth <= 0.5 * ny
        assert pool.shape == capi.SOURCE_AABB and abs(pool.center[1] - (-0.5 * ny + 0.5 * depth)) < 1e-3
        assert 1 <= len(drops) <= 4
        for d in drops:
            r = d.data[0]
            assert d.shape == capi.SOURCE_CIRCLE
            assert 0.05 * min(nx, ny) <= r <= 0.15 * min(nx, ny)
            assert d.center[1] >= r - 1e-3  # upper half
        assert s.cfg.projection.tolerance == pytest.approx(1e-5)
        assert s.cfg.projection.method == capi.PROJECTION_GAUSS_SEIDEL
    assert b.forces(3, 0) == [] and b.forces(3, 29) == []
    f = b.forces(3, 30)
    assert len(f) == 8
    for x in f:
        assert (x.force[0] ** 2 + x.force[1] ** 2) ** 0.5 <= 50.0 + 1e-4
        assert 0 <= x.position[0] < b.scenes[3].cfg.nx and 0 <= x.position[1] < b.scenes[3].cfg.ny
    g = scenes.batch(96).forces(3, 30)
    assert [(x.force[0], x.position[0]) for x in f] == [(x.force[0], x.position[0]) for x in g]


def test_oracle_mgpcg_converges_fast(oracle_api):
    """The multigrid-preconditioned CG reaches 1e-5 in a few tens of iterations
    where plain V-cycles of the same structure need over a hundred."""
    sc = scenes.scale(128)
    sc.cfg.projection.method = capi.PROJECTION_MGPCG
    sim = sc.make(oracle_api)
    sim.step(sc.dt)
    st = sim.step(sc.dt)
    assert st.converged and st.residual <= 1e-5 and 0 < st.pressure_iterations <= 40
    sc.cfg.projection.method = capi.PROJECTION_MULTIGRID
    ref = sc.make(oracle_api)
    ref.step(sc.dt)
    sv = ref.step(sc.dt)
    assert sv.converged and sv.pressure_iterations > 3 * st.pressure_iterations


def test_mgpcg_requires_tolerance(oracle_api):
    cfg = scenes.base_config(64, 64)
    cfg.projection.method = capi.PROJECTION_MGPCG
    cfg.projection.tolerance = 0.0
    with pytest.raises(capi.EflError):
        capi.Sim(oracle_api, cfg)


def test_velocity_magnitude_oracle_semantics(oracle_api):
    """The reference's second reduction pass adds partials per lane from 0.0,
    so a grid of fewer than 512 16x16 workgroups reports a minimum of 0; the
    maximum there is the true maximum of the cell-centred speed."""
    sc = scenes.dam_break(64)
    sim = sc.make(oracle_api)
    for _ in range(5):
        sim.step(sc.dt)
    mn, mx = sim.velocity_magnitude()
    u, v = sim.get(capi.FIELD_U), sim.get(capi.FIELD_V)
    uc = 0.5 * (u[:, :-1] + u[:, 1:])
    vc = 0.5 * (v[:-1, :] + v[1:, :])
    speed = np.sqrt(uc * uc + vc * vc).astype(np.float32)
    assert mn == 0.0
    assert mx == pytest.approx(float(speed.max()), rel=1e-6)


def test_cfl_dt_bounds_the_displacement(oracle_api):
    """plugin.cfl_dt: the step moves no fluid more than `cfl` cells at the monitored maximum speed
    (velocities are in grid cells per second: coordinate.wgsl:83-94 moves x by dt * velocity)."""
    from bevy_eulerian_fluid_b200.plugin import cfl_dt
    assert cfl_dt(0.0) == 1.0 / 60.0
    assert cfl_dt(float("nan")) == 1.0 / 60.0
    assert cfl_dt(30.0) == 1.0 / 60.0  # slower than 60 cells/s: the cap
    assert cfl_dt(120.0) == 1.0 / 120.0
    assert cfl_dt(120.0, cfl=0.5) == 0.5 / 120.0
    assert cfl_dt(10.0, dt_max=0.01) == 0.01
    sc = scenes.dam_break(64)
    o = sc.make(oracle_api)
    for _ in range(30):
        o.step(sc.dt)
    _, mx = o.velocity_magnitude()
    assert mx > 0.0
    dt = cfl_dt(mx, cfl=0.5, dt_max=1.0)
    assert dt * mx <= 0.5 * (1 + 1e-6)
    o.close()


def _separated(a, b, gap=8):
    (ax, ay, aw, ah), (bx, by, bw, bh) = a, b
    return ax + aw + gap <= bx or bx + bw + gap <= ax or ay + ah + gap <= by or by + bh + gap <= ay


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_canvas_pack_layout(seed):
    """efl_canvas_pack (host only): every image on the canvas, origins on multiples of 8, at least 8 pixels
    between any two images, the width the smallest multiple of 512 holding the widest image."""
    api = capi.load()
    rng = np.random.default_rng(seed)
    sizes = [(8 * int(rng.integers(1, 100)), 8 * int(rng.integers(1, 60))) for _ in range(int(rng.integers(1, 120)))]
    org, w, h = capi.canvas_pack(api, sizes)
    assert w % 512 == 0 and w - 512 < max(s[0] for s in sizes) <= w and h % 8 == 0
    rects = [(x, y, sw, sh) for (x, y), (sw, sh) in zip(org, sizes)]
    for x, y, sw, sh in rects:
        assert x % 8 == 0 and y % 8 == 0 and x + sw <= w and y + sh <= h
    for i in range(len(rects)):
        for j in range(i):
            assert _separated(rects[i], rects[j]), (rects[i], rects[j])
    with pytest.raises(capi.EflError):
        capi.canvas_pack(api, [(12, 16)])


def test_canvas_of_the_c4_batch():
    """The 96 simulations of the C4 batch on the grid coarsened 8x: one 512-wide canvas, its rectangles fill
    more than half of it (the gaps and shelf ends are the rest)."""
    api = capi.load()
    bs = scenes.batch(96)
    sizes = [(sc.cfg.nx // 8, sc.cfg.ny // 8) for sc in bs.scenes]
    org, w, h = capi.canvas_pack(api, sizes)
    assert w == 512
    fill = sum(a * b for a, b in sizes) / (w * h)
    assert 0.5 < fill <= 1.0, fill

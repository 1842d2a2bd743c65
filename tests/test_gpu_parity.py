"""CUDA path vs the CPU oracle through the C ABI, stage by stage and step by step.

Bar: bit-exact for every field wherever the reference's arithmetic is not
implementation-defined (everything on this path except exp() in the
Gaussian force splat, compared at 1e-5 relative).  JFA seeds, cell labels,
force bins and valid flags are integer/bit-exact by construction of this
check.
"""
import numpy as np
import pytest

from bevy_eulerian_fluid_b200 import _capi as capi
from bevy_eulerian_fluid_b200 import scenes

from .helpers import STATE_FIELDS, compare_fields, copy_state, make_pair, rel_max_err, small_coupled

pytestmark = pytest.mark.gpu

STEP_STAGES = list(range(capi.STAGE_UPDATE_SOLID, capi.STAGE_SOLID_FORCES + 1))


def _warm_oracle(scene, oracle_api, steps):
    o = scene.make(oracle_api)
    o.step(scene.dt)  # init sequence
    for _ in range(steps):
        o.step(scene.dt)
    return o


@pytest.mark.parametrize("reinit", [capi.REINIT_JUMP_FLOODING, capi.REINIT_FAST_ITERATIVE])
@pytest.mark.parametrize("stage", STEP_STAGES)
def test_stage_parity(oracle_api, gpu_api, stage, reinit):
    sc = small_coupled(128, tolerance=0.0)
    sc.cfg.reinit.method = reinit
    o = _warm_oracle(sc, oracle_api, 3)
    g = sc.make(gpu_api)
    copy_state(o, g)
    if stage == capi.STAGE_APPLY_FORCES:
        forces = []
        for k, (fx, fy, px, py) in enumerate([(30.0, -10.0, 40.0, 90.0), (-5.0, 25.0, 100.0, 60.0)]):
            f = capi.Force()
            f.force[0], f.force[1], f.position[0], f.position[1] = fx, fy, px, py
            forces.append(f)
        o.set_local_forces(forces)
        g.set_local_forces(forces)
    so = o.run_stage(stage, sc.dt)
    sg = g.run_stage(stage, sc.dt)
    assert so.pressure_iterations == sg.pressure_iterations
    bad = compare_fields(g, o)
    assert not bad, f"stage {stage}: {bad}"
    if stage == capi.STAGE_SOLID_FORCES:
        assert np.array_equal(g.force_bins(), o.force_bins())
        assert np.array_equal(g.solid_forces(), o.solid_forces())


def test_init_parity(oracle_api, gpu_api):
    sc = scenes.dam_break(128)
    o, g = make_pair(sc, oracle_api, gpu_api)
    so, sg = o.step(sc.dt), g.step(sc.dt)
    assert so.initialized_only == sg.initialized_only == 1
    assert not compare_fields(g, o)


@pytest.mark.parametrize("n,steps", [(64, 40), (128, 25)])
def test_dam_break_steps_bit_exact(oracle_api, gpu_api, n, steps):
    """Reference configuration (GS 20 at weight 1.9, FIM(10)) over many steps."""
    sc = scenes.dam_break(n)
    o, g = make_pair(sc, oracle_api, gpu_api)
    for _ in range(steps + 1):
        o.step(sc.dt)
        g.step(sc.dt)
    bad = compare_fields(g, o)
    assert not bad, bad
    assert g.fluid_volume() == o.fluid_volume()


@pytest.mark.parametrize("iters", [7, 4])
def test_fixed_count_sweeps_with_bodies(oracle_api, gpu_api, iters):
    """Fixed-count f32 RBGS (the TMA-streamed sweep, two iterations per pass and a one-iteration tail for odd
    counts) on a 192 x 128 scene with bodies: fields bit-exact after several steps."""
    sc = small_coupled(128, tolerance=0.0)
    sc.cfg.nx = 192
    sc.cfg.projection.gs_iterations = iters
    o, g = make_pair(sc, oracle_api, gpu_api)
    for _ in range(6):
        o.step(sc.dt)
        g.step(sc.dt)
    bad = compare_fields(g, o)
    assert not bad, bad


def test_coupled_tolerance_steps(oracle_api, gpu_api):
    """JFA + bodies + FP64 RBGS to 1e-5: same iteration counts, bit-exact fields."""
    sc = small_coupled(128, tolerance=1e-5)
    o, g = make_pair(sc, oracle_api, gpu_api)
    o.step(sc.dt)
    g.step(sc.dt)
    for _ in range(4):
        so, sg = o.step(sc.dt), g.step(sc.dt)
        assert so.converged and sg.converged
        assert so.pressure_iterations == sg.pressure_iterations
        assert abs(so.residual - sg.residual) <= 1e-9 * max(1.0, abs(so.residual))
        assert sg.residual <= 1e-5
    bad = compare_fields(g, o)
    assert not bad, bad
    assert np.array_equal(g.force_bins(), o.force_bins())
    assert np.array_equal(g.get(capi.FIELD_JFA_SEEDS), o.get(capi.FIELD_JFA_SEEDS))


def test_multigrid_reference_mode(oracle_api, gpu_api):
    """One V-cycle per step with the reference's level rule (multi_grid.rs:95-97)."""
    sc = scenes.dam_break(128)
    sc.cfg.projection.method = capi.PROJECTION_MULTIGRID
    o, g = make_pair(sc, oracle_api, gpu_api)
    for _ in range(6):
        o.step(sc.dt)
        g.step(sc.dt)
    assert not compare_fields(g, o)


def test_jacobi_mode(oracle_api, gpu_api):
    sc = scenes.dam_break(64)
    sc.cfg.projection.method = capi.PROJECTION_JACOBI
    o, g = make_pair(sc, oracle_api, gpu_api)
    for _ in range(4):
        o.step(sc.dt)
        g.step(sc.dt)
    assert not compare_fields(g, o)


def test_residual_and_volume(oracle_api, gpu_api):
    sc = small_coupled(128, tolerance=0.0)
    o = _warm_oracle(sc, oracle_api, 2)
    g = sc.make(gpu_api)
    copy_state(o, g)
    for s in (o, g):  # the operator depends on dt: give both handles the same one
        s.run_stage(capi.STAGE_LEVELSET_GRADIENT, sc.dt)
    ro, rg = o.residual(), g.residual()
    assert abs(ro[0] - rg[0]) <= 1e-12 * max(1.0, ro[0])
    assert o.fluid_volume() == g.fluid_volume()


def test_local_forces_consumed_once(oracle_api, gpu_api):
    """ForcesToFluid applies to the next step only (apply_forces.rs:157-168), bit-exact with forces."""
    sc = scenes.dam_break(64)
    o, g = make_pair(sc, oracle_api, gpu_api)
    for s in (o, g):
        s.step(sc.dt)
    f = capi.Force()
    f.force[0], f.force[1], f.position[0], f.position[1] = 50.0, -20.0, 32.0, 40.0
    for s in (o, g):
        s.set_local_forces([f])
        s.step(sc.dt)
    assert not compare_fields(g, o)
    u_before = g.get(capi.FIELD_U1)
    for s in (o, g):
        s.run_stage(capi.STAGE_APPLY_FORCES, sc.dt)  # no forces left: gravity only
    assert not compare_fields(g, o)
    for s in (o, g):
        s.step(sc.dt)
    assert not compare_fields(g, o)
    assert u_before.shape == g.get(capi.FIELD_U1).shape


def test_coupled_tolerance_global_path(oracle_api, gpu_api):
    """1024 x 512 does not fit the persistent scheme: the global-memory form of the
    mixed-precision solve runs, with the same iteration count and bit-exact fields."""
    sc = small_coupled(1024, tolerance=1e-5, n_per_shape=1)
    sc.cfg.ny = 512
    sc.oneshot[0].center[1] = -256.0 + 0.5 * 0.4 * 512
    sc.oneshot[0].data[1] = 0.5 * 0.4 * 512
    sc.cfg.projection.max_iterations = 4000  # the first solve from p = 0 needs ~20k: stop early on both
    o, g = make_pair(sc, oracle_api, gpu_api)
    o.step(sc.dt)
    g.step(sc.dt)
    so, sg = o.step(sc.dt), g.step(sc.dt)
    assert so.converged == sg.converged
    assert so.pressure_iterations == sg.pressure_iterations == 4000
    assert abs(so.residual - sg.residual) <= 1e-9 * max(1.0, abs(so.residual))
    for f in (capi.FIELD_PRESSURE, capi.FIELD_U, capi.FIELD_V, capi.FIELD_LEVELSET_AIR):
        assert np.array_equal(g.get(f), o.get(f)), f


def test_mgpcg_bit_exact(oracle_api, gpu_api):
    """MG-preconditioned CG (row-ordered reductions on both sides): same CG
    iteration counts and bit-exact fields on the C3 scene at 256^2."""
    sc = scenes.scale(256)
    sc.cfg.projection.method = capi.PROJECTION_MGPCG
    o, g = make_pair(sc, oracle_api, gpu_api)
    o.step(sc.dt)
    g.step(sc.dt)
    for _ in range(3):
        so, sg = o.step(sc.dt), g.step(sc.dt)
        assert so.converged and sg.converged
        assert so.pressure_iterations == sg.pressure_iterations
        assert so.residual == sg.residual and so.residual_initial == sg.residual_initial
    bad = compare_fields(g, o)
    assert not bad, bad


def test_mgpcg_tma_levels_bit_exact(oracle_api, gpu_api):
    """MGPCG at 512^2: the preconditioner smooths levels 0 (512^2) and 1 (256^2) with the TMA-streamed sweep
    and the rest in the single-CTA tail; same CG counts and bit-exact fields."""
    sc = scenes.scale(512)
    sc.cfg.projection.method = capi.PROJECTION_MGPCG
    o, g = make_pair(sc, oracle_api, gpu_api)
    o.step(sc.dt)
    g.step(sc.dt)
    for _ in range(3):
        so, sg = o.step(sc.dt), g.step(sc.dt)
        assert so.converged and sg.converged
        assert so.pressure_iterations == sg.pressure_iterations
        assert so.residual == sg.residual and so.residual_initial == sg.residual_initial
    bad = compare_fields(g, o)
    assert not bad, bad


def test_mgpcg_with_bodies_bit_exact(oracle_api, gpu_api):
    """MGPCG on the coupled scene (bodies, fractional faces, JFA)."""
    sc = small_coupled(128, method=capi.PROJECTION_MGPCG)
    o, g = make_pair(sc, oracle_api, gpu_api)
    o.step(sc.dt)
    g.step(sc.dt)
    for _ in range(4):
        so, sg = o.step(sc.dt), g.step(sc.dt)
        assert so.converged and sg.converged
        assert so.pressure_iterations == sg.pressure_iterations
        assert so.residual == sg.residual
    bad = compare_fields(g, o)
    assert not bad, bad
    assert np.array_equal(g.force_bins(), o.force_bins())


@pytest.mark.parametrize("tolerance", [0.0, 1e-5])
def test_graph_replay_matches_eager(gpu_api, tolerance):
    """Steps replayed from captured CUDA graphs equal eager launches bit for bit,
    across a change of the local forces (a new signature) and back."""
    sc = small_coupled(128, tolerance=tolerance, n_per_shape=1)
    a, b = sc.make(gpu_api), sc.make(gpu_api)
    b.set_graph_capture(False)
    for k in range(8):
        if k == 4:
            f = capi.Force()
            f.force[0], f.force[1], f.position[0], f.position[1] = 40.0, -20.0, 60.0, 70.0
            a.set_local_forces([f])
            b.set_local_forces([f])
        sa, sb = a.step(sc.dt), b.step(sc.dt)
        assert sa.pressure_iterations == sb.pressure_iterations
    assert not compare_fields(a, b)
    assert np.array_equal(a.force_bins(), b.force_bins())


def test_device_coupling_matches_host_loop(gpu_api):
    """Rigid bodies integrated on the device at the end of each step follow the
    host integrator (rigid.py) driven through the C ABI: same forces, same
    semi-implicit Euler; positions agree to float rounding of the transforms."""
    from bevy_eulerian_fluid_b200.plugin import pack_obstacles
    from bevy_eulerian_fluid_b200.rigid import RigidWorld, device_bodies
    sc = small_coupled(128, tolerance=1e-5, n_per_shape=2)
    host, dev = sc.make(gpu_api), sc.make(gpu_api)
    rw = RigidWorld(list(sc.bodies), (128, 128), gravity=9.8 * scenes.LENGTH_UNIT,
                    grid_length=1.0 / scenes.LENGTH_UNIT)
    host.step(sc.dt)
    dev.step(sc.dt)
    dev.set_rigid_bodies(device_bodies(sc.bodies), 9.8 * scenes.LENGTH_UNIT, 1.0 / scenes.LENGTH_UNIT)
    for _ in range(5):
        host.step(sc.dt)
        rw.apply_fluid_forces(host.solid_forces(), sc.dt)
        rw.step(sc.dt)
        host.set_obstacles(pack_obstacles(rw.bodies))
        dev.step(sc.dt)
    got = dev.get_rigid_bodies(len(rw.bodies))
    for b, g in zip(rw.bodies, got):
        assert abs(g.position[0] - b.position[0]) < 1e-3 and abs(g.position[1] - b.position[1]) < 1e-3
        assert abs(g.rotation - b.rotation) < 1e-4
    d = rel_max_err(dev.get(capi.FIELD_PRESSURE), host.get(capi.FIELD_PRESSURE))
    assert d < 1e-3, d


def test_velocity_magnitude_diagnostics(oracle_api, gpu_api):
    """diagnostics/{min,max}_velocity.wgsl on both backends, bit for bit."""
    for n in (128, 512):  # 64 and 1024 workgroups: below and above the second pass's 512 lanes
        sc = scenes.dam_break(n)
        o, g = make_pair(sc, oracle_api, gpu_api)
        for _ in range(4):
            o.step(sc.dt)
            g.step(sc.dt)
        copy_state(o, g)
        assert g.velocity_magnitude() == o.velocity_magnitude()


# ---------------------------------------------------------------------------
# Edge cases of the domain: empty fluid, ragged (non-square, not a multiple of
# 64) grids, the maximum number of obstacles and sources.

@pytest.mark.parametrize("tolerance", [0.0, 1e-5])
def test_empty_domain(oracle_api, gpu_api, tolerance):
    """No water at all: the solve has nothing to do (b = 0), every field stays
    bit-exact, the volume is 0."""
    cfg = scenes.base_config(64, 48)
    cfg.projection.tolerance = tolerance
    o, g = capi.Sim(oracle_api, cfg), capi.Sim(gpu_api, cfg)
    for _ in range(4):
        so, sg = o.step(scenes.DT), g.step(scenes.DT)
        assert so.pressure_iterations == sg.pressure_iterations
    assert not compare_fields(g, o)
    assert g.fluid_volume() == o.fluid_volume() == 0


@pytest.mark.parametrize("nx,ny", [(136, 88), (200, 40)])
def test_ragged_grid_steps(oracle_api, gpu_api, nx, ny):
    """Grids whose dispatches do not cover every face (sizes not multiples of
    64): the reference's floor(n/64) coverage is replicated, bit-exact."""
    cfg = scenes.base_config(nx, ny)
    src = scenes.aabb_source((0.0, -0.2 * ny), (0.5 * nx, 0.3 * ny))
    sc = scenes.Scene(f"ragged_{nx}x{ny}", cfg, oneshot=[src])
    o, g = make_pair(sc, oracle_api, gpu_api)
    for _ in range(8):
        o.step(sc.dt)
        g.step(sc.dt)
    assert not compare_fields(g, o)


def test_maximum_obstacles_and_sources(oracle_api, gpu_api):
    """256 obstacles (EFL_MAX_SOLIDS) and 16 continuous sources, bit-exact,
    force bins included."""
    from bevy_eulerian_fluid_b200.plugin import Collider, RigidBody, RigidBodyKind, pack_obstacles
    n = 128
    cfg = scenes.base_config(n, n)
    bodies = []
    for i in range(capi.MAX_SOLIDS):
        x, y = -56.0 + 7.0 * (i % 16), -50.0 + 6.5 * (i // 16)
        bodies.append(RigidBody(Collider.circle(1.5 + 0.5 * (i % 3)), (x, y), 0.0, kind=RigidBodyKind.Static,
                                density=scenes.RHO))
    srcs = [scenes.circle_source((-60.0 + 8.0 * k, 40.0), 3.0, velocity=(0.0, -5.0)) for k in range(16)]
    sc = scenes.Scene("crowded_128", cfg, continuous=srcs)
    o, g = make_pair(sc, oracle_api, gpu_api)
    obs = pack_obstacles(bodies)
    o.set_obstacles(obs)
    g.set_obstacles(obs)
    for _ in range(6):
        o.step(sc.dt)
        g.step(sc.dt)
    assert not compare_fields(g, o)
    assert np.array_equal(g.force_bins(), o.force_bins())


def test_reset_matches_oracle_reset(oracle_api, gpu_api):
    """FluidStatus::Reset (fluid_status.rs:15-38, render_node.rs:177-189): efl_reset makes the next step re-run the
    init sequence only.  The fields it writes equal a fresh handle's init; the rest carry over, and the run that
    follows stays bit-exact with the oracle doing the same reset."""
    sc = small_coupled(128, tolerance=1e-5)
    o, g = make_pair(sc, oracle_api, gpu_api)
    for _ in range(4):
        o.step(sc.dt)
        g.step(sc.dt)
    o.reset()
    g.reset()
    so, sg = o.step(sc.dt), g.step(sc.dt)
    assert so.initialized_only == sg.initialized_only == 1
    fresh = sc.make(gpu_api)
    assert fresh.step(sc.dt).initialized_only == 1
    init_fields = [capi.FIELD_U, capi.FIELD_V, capi.FIELD_U1, capi.FIELD_V1, capi.FIELD_LEVELSET_AIR,
                   capi.FIELD_LEVELSET_AIR1, capi.FIELD_JFA_SEEDS, capi.FIELD_GRAD_LEVELSET]
    assert not compare_fields(g, fresh, fields=init_fields)
    assert not compare_fields(g, o)
    for _ in range(3):
        so, sg = o.step(sc.dt), g.step(sc.dt)
        assert so.pressure_iterations == sg.pressure_iterations
    assert not compare_fields(g, o)
    assert np.array_equal(g.force_bins(), o.force_bins())
    fresh.close()
    o.close()
    g.close()

"""Known-answer tests that pin the CPU oracle (the reference publishes no golden vectors).

Each test builds inputs whose result is known analytically or from an
independent computation, runs one oracle stage through the same C ABI the
CUDA library exposes, and checks the answer.
"""
import ctypes
import math

import numpy as np
import pytest

from bevy_eulerian_fluid_b200 import _capi as capi
from bevy_eulerian_fluid_b200 import scenes
from bevy_eulerian_fluid_b200.plugin import Collider, RigidBody, RigidBodyKind


def _sim(oracle_api, n=64, ny=None, **kw):
    c = scenes.base_config(n, ny or n)
    for k, v in kw.items():
        setattr(c, k, v)
    return capi.Sim(oracle_api, c)


def test_init_fields(oracle_api):
    """initialize_grid_center.wgsl: phi = H - y; initialize_grid_edge.wgsl: u = v = 0."""
    s = _sim(oracle_api, 64)
    s.step(scenes.DT)  # the init sequence (no sources: phi stays H - y before reinit)
    s.run_stage(capi.STAGE_INIT, scenes.DT)
    phi1 = s.get(capi.FIELD_LEVELSET_AIR1)
    y = np.arange(64, dtype=np.float32)[:, None]
    assert np.array_equal(phi1, np.broadcast_to(64 - y, (64, 64)))
    assert not s.get(capi.FIELD_U).any() and not s.get(capi.FIELD_V).any()


def test_area_fraction_planar_interface(oracle_api):
    """A face crossed by a planar solid interface is open over the length where phi_s > 0."""
    s = _sim(oracle_api, 64)
    x = np.arange(64, dtype=np.float32)[None, :]
    phis = np.broadcast_to(x - np.float32(30.3), (64, 64)).astype(np.float32)
    s.set(capi.FIELD_LEVELSET_SOLID, phis)
    s.run_stage(capi.STAGE_AREA_FRACTION, scenes.DT)
    af = s.get(capi.FIELD_AREA_FRACTION)
    # cell 30: horizontal faces span x in [29.5, 30.5], phi = -0.8 .. 0.2 -> open 0.2
    assert np.allclose(af[10:50, 30, 2], 0.2, atol=1e-5)
    assert np.allclose(af[10:50, 30, 3], 0.2, atol=1e-5)
    assert np.all(af[10:50, 20, :] == 0.0)  # fully inside the solid: closed
    assert np.all(af[10:50, 40, :] == 1.0)  # fully outside: open
    # vertical face at x = 30.5: both vertices at phi = 0.2 > 0 -> open
    assert np.all(af[10:50, 30, 1] == 1.0)


def test_area_fraction_zero_is_closed(oracle_api):
    """0/0 at a face whose vertices are both 0 clamps to 0 (closed)."""
    s = _sim(oracle_api, 32)
    s.set(capi.FIELD_LEVELSET_SOLID, np.zeros((32, 32), np.float32))
    s.run_stage(capi.STAGE_AREA_FRACTION, scenes.DT)
    assert not s.get(capi.FIELD_AREA_FRACTION).any()


def test_circle_sdf_and_ids(oracle_api):
    """update_solid.wgsl: border ring 0 / id -1, inside min(wall distance, |x - c| - r)."""
    n = 64
    s = _sim(oracle_api, n)
    body = RigidBody(Collider.circle(10.0), (3.0, -5.0), 0.0, kind=RigidBodyKind.Static)
    s.set_obstacles([body.to_obstacle(0)])
    s.run_stage(capi.STAGE_UPDATE_SOLID, scenes.DT)
    ls = s.get(capi.FIELD_LEVELSET_SOLID).astype(np.float64)
    sid = s.get(capi.FIELD_SOLID_ID)
    assert not ls[0].any() and not ls[-1].any() and not ls[:, 0].any() and not ls[:, -1].any()
    assert np.all(sid[0] == -1)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    wx, wy = xx - n / 2, n / 2 - yy  # to_world with the identity transform
    sdf = np.hypot(wx - 3.0, wy + 5.0) - 10.0
    wall = np.minimum(np.minimum(xx, n - 1 - xx), np.minimum(yy, n - 1 - yy))
    want = np.minimum(wall, sdf)
    inner = (slice(1, -1), slice(1, -1))
    assert np.max(np.abs(ls[inner] - want[inner])) < 1e-4
    assert np.all((sid[inner] == 0) == (sdf[inner] < 0.5))


def test_uniform_velocity_is_advected_unchanged(oracle_api):
    """Interpolating a constant field returns it: interior faces keep u = c under advection."""
    n = 64
    s = _sim(oracle_api, n)
    s.set(capi.FIELD_U, np.full((n, n + 1), 3.0, np.float32))
    s.set(capi.FIELD_V, np.zeros((n + 1, n), np.float32))
    s.run_stage(capi.STAGE_ADVECT_VELOCITY, scenes.DT)
    u1 = s.get(capi.FIELD_U1)
    assert np.all(u1[4:-4, 8:-8] == 3.0)


def _operator(phi, af, dx, dt, rho):
    """numpy restatement of residual.wgsl:33-54's operator over counted cells (float64)."""
    import scipy.sparse as sp
    H, W = phi.shape
    act = (phi < 0) & ~(af == 0).all(-1)
    idx = -np.ones((H, W), int)
    idx[act] = np.arange(act.sum())
    fac = dt / rho / dx / dx
    rows, cols, vals = [], [], []
    for y, x in zip(*np.nonzero(act)):
        i = idx[y, x]
        d = 0.0
        for k, (ox, oy) in enumerate(((-1, 0), (1, 0), (0, -1), (0, 1))):
            jx, jy = x + ox, y + oy
            if 0 <= jx < W and 0 <= jy < H:
                f = float(af[y, x, k])
                if phi[jy, jx] < 0:
                    d += f
                    if idx[jy, jx] >= 0:
                        rows.append(i), cols.append(idx[jy, jx]), vals.append(-f * fac)
                else:
                    d += f * (1.0 - float(phi[jy, jx]) / float(phi[y, x]))
        rows.append(i), cols.append(i), vals.append(d * fac)
    return sp.csr_matrix((vals, (rows, cols)), shape=(act.sum(),) * 2), act


def _projection_inputs(oracle_api, n=64):
    sc = scenes.coupled(n, tolerance=0.0, n_per_shape=1)
    s = sc.make(oracle_api)
    s.step(sc.dt)
    for st in range(capi.STAGE_UPDATE_SOLID, capi.STAGE_DIVERGENCE + 1):
        s.run_stage(st, sc.dt)
    return sc, s


def test_residual_matches_independent_operator(oracle_api):
    sc, s = _projection_inputs(oracle_api)
    rng = np.random.default_rng(1)
    p = rng.standard_normal((64, 64)).astype(np.float32) * 100
    s.set(capi.FIELD_PRESSURE, p)
    phi, af, b = s.get(capi.FIELD_LEVELSET_AIR), s.get(capi.FIELD_AREA_FRACTION), s.get(capi.FIELD_DIVERGENCE)
    dx = float(np.float32(1) / np.float32(10))
    A, act = _operator(phi, af, dx, float(np.float32(sc.dt)), float(np.float32(sc.cfg.rho)))
    r = b[act].astype(np.float64) - A @ p[act].astype(np.float64)
    want = np.linalg.norm(r) / np.linalg.norm(b[act].astype(np.float64))
    rel, nr, nb = s.residual()
    assert abs(rel - want) <= 1e-5 * want  # the oracle evaluates the operator in f32


def test_tolerance_solve_matches_direct_solve(oracle_api):
    """Mixed-precision RBGS to 1e-10 reproduces a sparse direct solve of the same system."""
    import scipy.sparse.linalg as spla
    sc, s = _projection_inputs(oracle_api)
    p = capi.default_config(64, 64).projection
    p.method, p.tolerance, p.max_iterations, p.check_interval, p.sor_weight = 1, 1e-10, 200000, 16, 1.9
    s.set_projection(p)
    s.set(capi.FIELD_PRESSURE, np.zeros((64, 64), np.float32))
    st = s.run_stage(capi.STAGE_PROJECTION, sc.dt)
    assert st.converged and st.residual <= 1e-10
    phi, af, b = s.get(capi.FIELD_LEVELSET_AIR), s.get(capi.FIELD_AREA_FRACTION), s.get(capi.FIELD_DIVERGENCE)
    dx = float(np.float32(1) / np.float32(10))
    A, act = _operator(phi, af, dx, float(np.float32(sc.dt)), float(np.float32(sc.cfg.rho)))
    x = spla.spsolve(A.tocsc(), b[act].astype(np.float64))
    got = s.get(capi.FIELD_PRESSURE)[act].astype(np.float64)
    assert np.max(np.abs(got - x)) <= 1e-5 * np.max(np.abs(x))


def test_jump_flooding_distance(oracle_api):
    """Jump flooding turns a circular level set into its signed distance (within a cell)."""
    n = 64
    c = scenes.base_config(n, n)
    c.reinit.method = capi.REINIT_JUMP_FLOODING
    s = capi.Sim(oracle_api, c)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    sdf = np.hypot(xx - 30.3, yy - 33.7) - 14.2
    s.set(capi.FIELD_LEVELSET_AIR1, (np.tanh(sdf / 3) * 7).astype(np.float32))  # same zero set, not a distance
    s.run_stage(capi.STAGE_REINITIALIZE, scenes.DT)
    phi0 = s.get(capi.FIELD_LEVELSET_AIR).astype(np.float64)
    assert np.all(np.sign(phi0[np.abs(sdf) > 1]) == np.sign(sdf[np.abs(sdf) > 1]))
    assert np.max(np.abs(phi0 - sdf)) < 1.0
    seeds = s.get(capi.FIELD_JFA_SEEDS).astype(np.float64)
    dist_seed = np.hypot(seeds[..., 0] - 30.3, seeds[..., 1] - 33.7)
    assert np.max(np.abs(dist_seed - 14.2)) < 0.5  # every seed lies on the interface


def test_fim_two_phase_vs_serial(oracle_api):
    """The deterministic two-phase FIM stays within tolerance of the literal serial execution."""
    from oracle import py_oracle
    n = 64
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    sdf = (np.hypot(xx - 30.3, yy - 33.7) - 14.2).astype(np.float32)
    out = []
    for serial in (False, True):
        c = scenes.base_config(n, n)
        s = capi.Sim(oracle_api, c)
        py_oracle.set_fim_serial(s, serial)
        s.set(capi.FIELD_LEVELSET_AIR1, np.clip(sdf * 1.7, -40, 40))
        s.run_stage(capi.STAGE_REINITIALIZE, scenes.DT)
        out.append(s.get(capi.FIELD_LEVELSET_AIR))
    band = np.abs(sdf) < 4
    a, b = out
    assert np.all(np.sign(a[band]) == np.sign(b[band]))
    assert np.max(np.abs(a[band] - b[band])) < 0.5
    assert np.max(np.abs(a[band] - sdf[band])) < 1.0  # both approximate the distance near the interface


def test_exp_restatement_accuracy(oracle_api):
    lib = oracle_api.lib
    lib.eflo_exp.restype, lib.eflo_exp.argtypes = ctypes.c_float, [ctypes.c_float]
    xs = np.concatenate([-np.logspace(-6, 1.9, 400), np.linspace(-80, 80, 400)]).astype(np.float32)
    got = np.array([lib.eflo_exp(float(x)) for x in xs], np.float32).astype(np.float64)
    ref = np.exp(xs.astype(np.float64))
    ulp = np.spacing(ref.astype(np.float32)).astype(np.float64)
    assert np.max(np.abs(got - ref) / ulp) <= 1.5


def test_volume_count(oracle_api):
    s = _sim(oracle_api, 32)
    phi = np.random.default_rng(3).standard_normal((32, 32)).astype(np.float32)
    s.set(capi.FIELD_LEVELSET_AIR, phi)
    assert s.fluid_volume() == int((phi < 0).sum())


def test_thread_count_does_not_change_results(oracle_api):
    from oracle import py_oracle
    res = []
    for t in (1, 4):
        py_oracle.set_threads(t)
        sc = scenes.coupled(64, tolerance=1e-5, n_per_shape=1)
        s = sc.make(oracle_api)
        for _ in range(3):
            st = s.step(sc.dt)
        res.append((st.pressure_iterations, s.get(capi.FIELD_PRESSURE), s.get(capi.FIELD_LEVELSET_AIR)))
    py_oracle.set_threads(0)
    assert res[0][0] == res[1][0]
    assert np.array_equal(res[0][1], res[1][1]) and np.array_equal(res[0][2], res[1][2])


def test_error_behaviour(oracle_api):
    with pytest.raises(capi.EflError):
        _sim(oracle_api, 60)  # not a multiple of 8
    s = _sim(oracle_api, 32)
    too_many = [capi.SolidObstacle() for _ in range(capi.MAX_SOLIDS + 1)]
    with pytest.raises(capi.EflError) as e:
        s.set_obstacles(too_many)
    assert e.value.status == capi.ERR_TOO_MANY
    bad = capi.SolidObstacle()
    bad.shape = 3
    with pytest.raises(capi.EflError) as e:
        s.set_obstacles([bad])
    assert e.value.status == capi.ERR_UNSUPPORTED_SHAPE
    with pytest.raises(capi.EflError) as e:
        s.set_sources([capi.Source() for _ in range(capi.MAX_FLUID_SOURCE + 1)], False)
    assert e.value.status == capi.ERR_TOO_MANY


def test_learned_fp64_solve_matches_operator_restatement(oracle_api):
    """learned.fp64_solve (the FP64 CPU solve that judges the network's prediction) builds the same system as
    the loop restatement above and solves it: equal matrices, and A x = b to round-off."""
    from bevy_eulerian_fluid_b200 import learned
    sc, s = _projection_inputs(oracle_api)
    phi, af, b = s.get(capi.FIELD_LEVELSET_AIR), s.get(capi.FIELD_AREA_FRACTION), s.get(capi.FIELD_DIVERGENCE)
    dx, dt, rho = float(np.float32(1) / np.float32(10)), float(np.float32(sc.dt)), float(np.float32(sc.cfg.rho))
    A, act = _operator(phi, af, dx, dt, rho)
    x, act2 = learned.fp64_solve(phi, af, b, dx, dt, rho)
    assert np.array_equal(act, act2)
    r = A @ x[act] - b[act].astype(np.float64)
    assert np.linalg.norm(r) <= 1e-9 * np.linalg.norm(b[act].astype(np.float64))


def test_hydrostatic_force_on_a_circle(oracle_api):
    """sample_forces.wgsl / accumulate_forces.wgsl against the analytic buoyancy: with p = G y (y the cell row,
    growing downwards) the pressure force on a submerged circle of radius R cells is -(integral of grad p over
    the disc) = (0, -G pi R^2) per unit depth, times dx for the face length (grid frame, y down: the force points
    up), with no net torque about the centre.  The reference sums the face terms only over cells whose solid id
    is the body's (within half a cell of the circle, update_solid.wgsl), so the open faces just outside are left
    out and the discrete force comes out a few per cent low; the bound below allows 6 %."""
    dx = float(np.float32(1) / np.float32(10))
    G = 1000.0
    for n, R in ((128, 20.0), (256, 40.0), (256, 80.0)):
        s = _sim(oracle_api, n)
        body = RigidBody(Collider.circle(R), (0.0, 0.0), 0.0, kind=RigidBodyKind.Static)
        s.set_obstacles([body.to_obstacle(0)])
        s.run_stage(capi.STAGE_UPDATE_SOLID, scenes.DT)
        yy = np.mgrid[0:n, 0:n][0].astype(np.float32)
        s.set(capi.FIELD_PRESSURE, (np.float32(G) * yy).astype(np.float32))
        s.run_stage(capi.STAGE_SOLID_FORCES, scenes.DT)
        fx, fy, tq = (float(v) for v in s.solid_forces()[0])
        want = -G * math.pi * R * R * dx
        assert 0.94 * abs(want) <= -fy <= 1.0 * abs(want), (R, fy, want)
        assert abs(fx) <= 1e-4 * abs(want) and abs(tq) <= 1e-4 * abs(want) * R * dx, (R, fx, tq)
        # the fixed-point bins (x10, truncated per cell) are what the forces are read from
        bins = s.force_bins()
        assert abs(bins[1][0] * 0.1 - fy) <= 0.1
        # a uniform pressure exerts no net force: the face terms telescope around the body
        s.set(capi.FIELD_PRESSURE, np.full((n, n), 500.0, np.float32))
        s.run_stage(capi.STAGE_SOLID_FORCES, scenes.DT)
        f0 = s.solid_forces()[0]
        assert abs(float(f0[0])) <= 1e-3 * abs(want) and abs(float(f0[1])) <= 1e-3 * abs(want), (R, f0)
        s.close()

"""Python mirror of the reference plugin's user-facing API.

Names, fields and error behaviour follow the Bevy plugin
(src/euler_fluid.rs, settings.rs, fluid_source.rs, apply_forces.rs,
projection.rs, reinitialize_levelset.rs, obstacle.rs, fluid_to_solid.rs);
each simulation step goes through the C ABI of libefl_b200.so.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from enum import Enum, IntEnum
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _capi as capi

Vec2 = Tuple[float, float]


def _warn(msg: str):
    import warnings
    warnings.warn(msg, stacklevel=3)


class FluidPlugin:
    """FluidPlugin::new(length_unit) (euler_fluid.rs:47-53): dx = 1 / length_unit."""

    def __init__(self, length_unit: float):
        if not length_unit > 0.0:
            raise ValueError("length_unit must be positive value.")  # euler_fluid.rs:49-51
        self.length_unit = float(length_unit)
        self.particle_levelset = False

    def add_plugins(self, *plugins) -> "FluidPlugin":
        """App::add_plugins for the fluid's optional plugins: ParticleLevelsetTwoLayersPlugin (the
        reference adds it inside FluidPlugin::build, commented out at euler_fluid.rs:81)."""
        for p in plugins:
            if isinstance(p, ParticleLevelsetTwoLayersPlugin):
                self.particle_levelset = True
            else:
                raise TypeError(f"unknown plugin {p!r}")
        return self

    @property
    def grid_length(self) -> float:  # FluidGridLength (euler_fluid.rs:89)
        return 1.0 / self.length_unit

    def spawn(self, settings: "FluidSettings", transform: Optional[Sequence[float]] = None,
              projection: Optional["ProjectionMethod"] = None, reinitialize: Optional["ReinitializeMethod"] = None,
              device: int = 0) -> "Fluid":
        """Spawns FluidSettings (+ its required components) and allocates the fluid."""
        return Fluid(self, settings, transform, projection or ProjectionMethod.default(),
                     reinitialize or ReinitializeMethod.default(), device)


class ParticleLevelsetTwoLayersPlugin:
    """particle_levelset_two_layers/plugin.rs:93-118: the two-layer particle level set (Enright et al. 2002) on
    every fluid spawned afterwards -- particles seeded by the init sequence, advected and used to correct the
    level set before and after its reinitialisation, reseeded every step."""


@dataclass
class FluidSettings:  # settings.rs:110-114
    rho: float
    gravity: Vec2
    size: Tuple[int, int]


class FluidSourceMode(IntEnum):  # fluid_source.rs:38-43
    Source = 0
    Sink = 1


@dataclass
class FluidSource:  # fluid_source.rs:31-36
    active: bool = True
    mode: FluidSourceMode = FluidSourceMode.Source


@dataclass
class FluidSourceShape:  # fluid_source.rs:55-59
    kind: int
    value: Vec2

    @staticmethod
    def Circle(radius: float) -> "FluidSourceShape":
        return FluidSourceShape(capi.SOURCE_CIRCLE, (float(radius), 0.0))

    @staticmethod
    def Aabb(half_size: Vec2) -> "FluidSourceShape":
        return FluidSourceShape(capi.SOURCE_AABB, (float(half_size[0]), float(half_size[1])))

    def to_vec2(self) -> Vec2:
        return self.value

    def shape_type_digit(self) -> int:
        return self.kind


@dataclass
class FluidSourceVelocity:  # fluid_source.rs:81-82
    value: Vec2 = (0.0, 0.0)


class FluidSourceOneshot:  # fluid_source.rs:86-87 (marker)
    pass


@dataclass
class ForceToFluid:  # apply_forces.rs:36-40: force (m/s^2) at a grid-pixel position, y down
    force: Vec2
    position: Vec2


@dataclass
class ForcesToFluid:  # apply_forces.rs:42-45
    forces: List[ForceToFluid] = field(default_factory=list)


LocalForces = ForcesToFluid  # the README's name for ForcesToFluid


@dataclass
class GaussSeidelConfig:  # gauss_seidel.rs:33-42
    num_iterations: int = 20


@dataclass
class MultiGridConfig:  # multi_grid.rs:56-71
    pre_smooth_config: GaussSeidelConfig = field(default_factory=lambda: GaussSeidelConfig(2))
    post_smooth_config: GaussSeidelConfig = field(default_factory=lambda: GaussSeidelConfig(2))
    coarsest_config: GaussSeidelConfig = field(default_factory=lambda: GaussSeidelConfig(3))


@dataclass
class ProjectionMethod:  # projection.rs:44-58
    """Jacobi | GaussSeidel(GaussSeidelConfig) | MultiGrid(MultiGridConfig).

    tolerance > 0 turns the fixed-count solve into a solve to
    ||b - A p|| / ||b|| <= tolerance (an extension; 0 is the reference).
    """
    method: int
    gauss_seidel: GaussSeidelConfig = field(default_factory=GaussSeidelConfig)
    multigrid: MultiGridConfig = field(default_factory=MultiGridConfig)
    tolerance: float = 0.0
    max_iterations: int = 20000
    check_interval: int = 16
    sor_weight: float = 1.9  # gauss_seidel.rs:72
    mg_levels: int = 0

    @staticmethod
    def Jacobi() -> "ProjectionMethod":
        return ProjectionMethod(capi.PROJECTION_JACOBI)

    @staticmethod
    def GaussSeidel(config: Optional[GaussSeidelConfig] = None, **kw) -> "ProjectionMethod":
        return ProjectionMethod(capi.PROJECTION_GAUSS_SEIDEL, gauss_seidel=config or GaussSeidelConfig(), **kw)

    @staticmethod
    def MultiGrid(config: Optional[MultiGridConfig] = None, **kw) -> "ProjectionMethod":
        return ProjectionMethod(capi.PROJECTION_MULTIGRID, multigrid=config or MultiGridConfig(), **kw)

    @staticmethod
    def default() -> "ProjectionMethod":
        return ProjectionMethod.GaussSeidel()

    def to_c(self) -> capi.Projection:
        p = capi.Projection()
        p.method = self.method
        p.gs_iterations = self.gauss_seidel.num_iterations
        p.sor_weight = self.sor_weight
        p.mg_pre = self.multigrid.pre_smooth_config.num_iterations
        p.mg_post = self.multigrid.post_smooth_config.num_iterations
        p.mg_coarsest = self.multigrid.coarsest_config.num_iterations
        p.mg_levels = self.mg_levels
        p.tolerance = self.tolerance
        p.max_iterations = self.max_iterations
        p.check_interval = self.check_interval
        return p

    def __str__(self) -> str:  # projection.rs:60-79
        if self.method == capi.PROJECTION_JACOBI:
            return "Jacobi"
        if self.method == capi.PROJECTION_GAUSS_SEIDEL:
            return f"Gauss-Seidel({self.gauss_seidel.num_iterations})"
        m = self.multigrid
        return (f"Multigrid({m.pre_smooth_config.num_iterations}-{m.coarsest_config.num_iterations}-"
                f"{m.post_smooth_config.num_iterations})")


@dataclass
class FastIterativeMethodConfig:  # fast_iterative_method.rs:14-23
    num_iterations: int = 10


@dataclass
class ReinitializeMethod:  # reinitialize_levelset.rs:36-46
    method: int
    fast_iterative: FastIterativeMethodConfig = field(default_factory=FastIterativeMethodConfig)

    @staticmethod
    def JumpFlooding() -> "ReinitializeMethod":
        return ReinitializeMethod(capi.REINIT_JUMP_FLOODING)

    @staticmethod
    def FastIterative(config: Optional[FastIterativeMethodConfig] = None) -> "ReinitializeMethod":
        return ReinitializeMethod(capi.REINIT_FAST_ITERATIVE, config or FastIterativeMethodConfig())

    @staticmethod
    def default() -> "ReinitializeMethod":
        return ReinitializeMethod.FastIterative()

    def to_c(self) -> capi.Reinit:
        r = capi.Reinit()
        r.method = self.method
        r.fim_iterations = self.fast_iterative.num_iterations
        return r

    def __str__(self) -> str:
        if self.method == capi.REINIT_JUMP_FLOODING:
            return "Jump Flooding"
        return f"Fast Iterative({self.fast_iterative.num_iterations})"


class FluidStatus(Enum):  # fluid_status.rs:15-21
    Reset = 0
    Uninitialized = 1
    Initialized = 2


@dataclass
class FluidToSolidForce:  # fluid_to_solid.rs:60-64
    force: Vec2
    torque: float


# ---------------------------------------------------------------------------
# Rigid bodies (the avian2d Collider/RigidBody query of obstacle.rs:89-160)

class RigidBodyKind(IntEnum):
    Dynamic = 0
    Static = 1
    Kinematic = 2


@dataclass
class Collider:
    """ShapeVariant (obstacle.rs:45-87), parameters in world units."""
    shape: int
    values: Tuple[float, ...]

    @staticmethod
    def circle(radius: float) -> "Collider":
        return Collider(capi.SHAPE_CIRCLE, (radius,))

    @staticmethod
    def rectangle(width: float, height: float) -> "Collider":
        return Collider(capi.SHAPE_RECTANGLE, (0.5 * width, 0.5 * height))

    @staticmethod
    def capsule(radius: float, length: float) -> "Collider":  # segment along local y
        h = 0.5 * length
        return Collider(capi.SHAPE_CAPSULE, (0.0, -h, 0.0, h, radius))

    @staticmethod
    def triangle(a: Vec2, b: Vec2, c: Vec2) -> "Collider":
        return Collider(capi.SHAPE_TRIANGLE, (a[0], a[1], b[0], b[1], c[0], c[1]))

    def area(self) -> float:
        v = self.values
        if self.shape == capi.SHAPE_CIRCLE:
            return math.pi * v[0] ** 2
        if self.shape == capi.SHAPE_RECTANGLE:
            return 4.0 * v[0] * v[1]
        if self.shape == capi.SHAPE_CAPSULE:
            L = math.hypot(v[2] - v[0], v[3] - v[1])
            return math.pi * v[4] ** 2 + 2.0 * v[4] * L
        return 0.5 * abs((v[2] - v[0]) * (v[5] - v[1]) - (v[4] - v[0]) * (v[3] - v[1]))

    def inertia_per_mass(self) -> float:
        v = self.values
        if self.shape == capi.SHAPE_CIRCLE:
            return 0.5 * v[0] ** 2
        if self.shape == capi.SHAPE_RECTANGLE:
            return ((2 * v[0]) ** 2 + (2 * v[1]) ** 2) / 12.0
        if self.shape == capi.SHAPE_CAPSULE:
            L = math.hypot(v[2] - v[0], v[3] - v[1])
            return (L * L) / 12.0 + 0.5 * v[4] ** 2
        pts = [(v[0], v[1]), (v[2], v[3]), (v[4], v[5])]
        cx = sum(p[0] for p in pts) / 3.0
        cy = sum(p[1] for p in pts) / 3.0
        return sum((p[0] - cx) ** 2 + (p[1] - cy) ** 2 for p in pts) / 6.0


@dataclass
class RigidBody:
    collider: Collider
    position: Vec2
    rotation: float = 0.0
    linear_velocity: Vec2 = (0.0, 0.0)
    angular_velocity: float = 0.0
    kind: RigidBodyKind = RigidBodyKind.Dynamic
    density: float = 1.0

    def transform(self) -> np.ndarray:
        c, s = math.cos(self.rotation), math.sin(self.rotation)
        m = np.eye(4, dtype=np.float64)
        m[0, 0], m[0, 1], m[1, 0], m[1, 1] = c, -s, s, c
        m[0, 3], m[1, 3] = self.position
        return m

    def to_obstacle(self, entity_id: int) -> capi.SolidObstacle:
        """construct_rigid_body_buffer_for_gpu (obstacle.rs:89-160)."""
        o = capi.SolidObstacle()
        o.entity_id = entity_id
        o.shape = self.collider.shape
        for i, v in enumerate(self.collider.values):
            o.values[i] = v
        m = self.transform()
        inv = np.linalg.inv(m)
        colmajor = m.T.reshape(-1)
        icolmajor = inv.T.reshape(-1)
        for i in range(16):
            o.transform[i] = colmajor[i]
            o.inverse_transform[i] = icolmajor[i]
        o.linear_velocity[0], o.linear_velocity[1] = self.linear_velocity
        o.angular_velocity = self.angular_velocity
        return o


_OBSTACLE_DTYPE = np.dtype([("entity_id", "<u4"), ("shape", "<u4"), ("values", "<f4", (6,)),
                            ("transform", "<f4", (16,)), ("inverse_transform", "<f4", (16,)),
                            ("linear_velocity", "<f4", (2,)), ("angular_velocity", "<f4"), ("_pad", "<f4")])
assert _OBSTACLE_DTYPE.itemsize == C.sizeof(capi.SolidObstacle) == 176


def pack_obstacles(bodies: Sequence[RigidBody]):
    """construct_rigid_body_buffer_for_gpu (obstacle.rs:89-160) for every body at once: the same values as
    RigidBody.to_obstacle (the transforms' inverses from one stacked np.linalg.inv, which inverts each matrix
    as the single call does), written straight into a ctypes array that set_obstacles passes on as is."""
    n = len(bodies)
    if n == 0:
        return []
    arr = (capi.SolidObstacle * n)()
    v = np.frombuffer(arr, dtype=_OBSTACLE_DTYPE)
    rot = [(math.cos(b.rotation), math.sin(b.rotation), b.position[0], b.position[1]) for b in bodies]
    c, sn, px, py = np.array(rot, dtype=np.float64).T  # RigidBody.transform, for every body
    m = np.zeros((n, 4, 4), dtype=np.float64)
    m[:, 0, 0], m[:, 0, 1], m[:, 1, 0], m[:, 1, 1] = c, -sn, sn, c
    m[:, 2, 2] = m[:, 3, 3] = 1.0
    m[:, 0, 3], m[:, 1, 3] = px, py
    inv = np.linalg.inv(m)
    v["entity_id"] = np.arange(n, dtype=np.uint32)
    v["shape"] = [b.collider.shape for b in bodies]
    vals = np.zeros((n, 6), dtype=np.float64)
    for i, b in enumerate(bodies):
        vals[i, :len(b.collider.values)] = b.collider.values
    v["values"] = vals
    v["transform"] = m.transpose(0, 2, 1).reshape(n, 16)
    v["inverse_transform"] = inv.transpose(0, 2, 1).reshape(n, 16)
    v["linear_velocity"] = [b.linear_velocity for b in bodies]
    v["angular_velocity"] = [b.angular_velocity for b in bodies]
    return arr


# ---------------------------------------------------------------------------

class FluidTextures:
    """FluidTextures (settings.rs:139-147): host copies of the output fields."""

    def __init__(self, sim: capi.Sim):
        self._sim = sim

    @property
    def u(self) -> np.ndarray:
        return self._sim.get(capi.FIELD_U)

    @property
    def v(self) -> np.ndarray:
        return self._sim.get(capi.FIELD_V)

    @property
    def u_solid(self) -> np.ndarray:
        return self._sim.get(capi.FIELD_U_SOLID)

    @property
    def v_solid(self) -> np.ndarray:
        return self._sim.get(capi.FIELD_V_SOLID)

    @property
    def levelset_air(self) -> np.ndarray:
        return self._sim.get(capi.FIELD_LEVELSET_AIR)

    @property
    def levelset_solid(self) -> np.ndarray:
        return self._sim.get(capi.FIELD_LEVELSET_SOLID)


@dataclass
class _SourceChild:
    source: FluidSource
    shape: FluidSourceShape
    translation: Vec2
    velocity: FluidSourceVelocity
    oneshot: bool


class Fluid:
    """One fluid entity: FluidSettings plus its required components."""

    def __init__(self, plugin: FluidPlugin, settings: FluidSettings, transform, projection: ProjectionMethod,
                 reinitialize: ReinitializeMethod, device: int = 0, api: Optional[capi.Api] = None):
        nx, ny = settings.size
        if nx % 64 or ny % 64:  # setup_components.rs:56-58
            _warn(f"the size is recommended to be multiple of 64. {settings.size}")
        cfg = capi.default_config(nx, ny)
        cfg.length_unit = plugin.length_unit
        cfg.rho = settings.rho
        cfg.gravity[0], cfg.gravity[1] = settings.gravity
        if transform is not None:
            t = np.asarray(transform, dtype=np.float64)
            t = t.T.reshape(-1) if t.shape == (4, 4) else t.reshape(-1)
            for i in range(16):
                cfg.transform[i] = t[i]
        cfg.projection = projection.to_c()
        cfg.reinit = reinitialize.to_c()
        cfg.device = device
        self.plugin = plugin
        self.settings = settings
        self.projection = projection
        self.reinitialize = reinitialize
        self.sim = capi.Sim(api or capi.load(), cfg)
        if plugin.particle_levelset:
            self.sim.set_particle_levelset(True)
        self.forces_to_fluid = ForcesToFluid()
        self.children: List[_SourceChild] = []
        self.status = FluidStatus.Reset
        self.last_stats: Optional[capi.StepStats] = None
        self._sources_dirty = True

    # children --------------------------------------------------------------
    def add_source(self, source: FluidSource, shape: FluidSourceShape, translation: Vec2 = (0.0, 0.0),
                   velocity: Optional[FluidSourceVelocity] = None, oneshot: bool = False) -> _SourceChild:
        child = _SourceChild(source, shape, (float(translation[0]), float(translation[1])),
                             velocity or FluidSourceVelocity(), oneshot)
        self.children.append(child)
        self._sources_dirty = True
        return child

    def _upload_sources(self):
        """update_fluid_source_{init_,}buffer (fluid_source_uniform.rs:77-158)."""
        for oneshot in (True, False):
            out = []
            for ch in self.children:
                if ch.oneshot != oneshot or not ch.source.active:
                    continue
                if len(out) >= capi.MAX_FLUID_SOURCE:
                    _warn(f"The maximum number of fluid source per fluid component is {capi.MAX_FLUID_SOURCE}.")
                    break
                s = capi.Source()
                s.center[0], s.center[1] = ch.translation
                s.data[0], s.data[1] = ch.shape.to_vec2()
                vel = (0.0, 0.0) if oneshot else ch.velocity.value
                s.velocity[0], s.velocity[1] = vel
                s.shape = ch.shape.shape_type_digit()
                s.mode = int(ch.source.mode)
                out.append(s)
            self.sim.set_sources(out, oneshot)
        self._sources_dirty = False

    # components -------------------------------------------------------------
    def set_projection(self, p: ProjectionMethod):
        self.projection = p
        self.sim.set_projection(p.to_c())

    def set_reinitialize(self, r: ReinitializeMethod):
        self.reinitialize = r
        self.sim.set_reinit(r.to_c())

    def set_rigid_bodies(self, bodies: Sequence[RigidBody]):
        self.sim.set_obstacles(pack_obstacles(bodies))

    def reset(self):
        self.status = FluidStatus.Reset
        self.sim.reset()

    @property
    def textures(self) -> FluidTextures:
        return FluidTextures(self.sim)

    # frame ------------------------------------------------------------------
    def step(self, dt: float) -> capi.StepStats:
        """One physics step: uploads ForcesToFluid (then clears it) and runs the pass."""
        if self._sources_dirty:
            self._upload_sources()
        forces = self.forces_to_fluid.forces
        if forces:
            arr = []
            for f in forces:
                c = capi.Force()
                c.force[0], c.force[1] = f.force
                c.position[0], c.position[1] = f.position
                arr.append(c)
            self.sim.set_local_forces(arr)
        forces.clear()  # apply_forces.rs:166
        st = self.sim.step(dt)
        self.status = FluidStatus.Initialized
        self.last_stats = st
        return st

    def forces_to_solid(self, n: Optional[int] = None) -> List[FluidToSolidForce]:
        arr = self.sim.solid_forces()
        n = capi.MAX_SOLIDS if n is None else n
        return [FluidToSolidForce((float(a[0]), float(a[1])), float(a[2])) for a in arr[:n]]

    def particles(self) -> "LevelsetParticles":
        """PLSResources.positive_particles / negative_particles (plugin.rs:186-211) and their counts:
        capi.PARTICLE_DTYPE arrays (position in grid cells, radius, sign, escaped)."""
        return LevelsetParticles(self.sim.read_particles(capi.PLS_POSITIVE), self.sim.read_particles(capi.PLS_NEGATIVE))

    # diagnostics (diagnostics/component.rs: FluidVolume, FluidMin/MaxVelocityMagnitude)
    def diagnostics(self) -> "FluidDiagnostics":
        mn, mx = self.sim.velocity_magnitude()
        return FluidDiagnostics(volume=self.sim.fluid_volume(), min_velocity_magnitude=mn, max_velocity_magnitude=mx)

    def close(self):
        self.sim.close()


@dataclass
class LevelsetParticles:
    positive: np.ndarray  # sign +1, seeded on the air side (phi > 0)
    negative: np.ndarray  # sign -1, seeded on the fluid side (phi < 0)


@dataclass
class FluidDiagnostics:
    volume: int                    # fluid cells (calculate_volume.wgsl)
    min_velocity_magnitude: float  # min_velocity.wgsl, grid units per second
    max_velocity_magnitude: float  # max_velocity.wgsl


def cfl_dt(max_velocity_magnitude: float, cfl: float = 1.0, dt_max: float = 1.0 / 60.0) -> float:
    """A time step that moves no fluid more than `cfl` cells (adaptive dt from
    the max-velocity monitor): min(dt_max, cfl / max_velocity_magnitude)."""
    if not (max_velocity_magnitude > 0.0):
        return dt_max
    return min(dt_max, cfl / max_velocity_magnitude)

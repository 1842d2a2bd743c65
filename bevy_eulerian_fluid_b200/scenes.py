"""Seeded synthetic scenes of the benchmark configurations.

No public dataset is involved: every scene is generated from a seed.
  dam_break_256   256^2 dam break, length unit 10, rho 99.7, g 9.8 down,
                  dt 1/60, walls on all sides, one one-shot AABB source at
                  (0,-0.2)*size with half-size 0.5*(1,0.6)*size
                  (examples/water_surface.rs:18-19,55-75), Gauss-Seidel 20,
                  FIM(10).
  coupled_512     512^2, water in the lower 40 %, 24 rigid bodies from seed
                  0xC2 (6 circles r U[8,32], 6 rectangles half-extents
                  U[6,30], 6 capsules r U[5,15] half-length U[10,30], 6
                  triangles with vertices at radius U[10,30]), positions in
                  the upper half, rotation U[0,2pi), density U[0.5,2]*rho,
                  jump flooding, RBGS to 1e-5 relative residual.
  scale_4096      4096^2 dam break with a static circle r=256 at the centre,
                  multigrid V-cycles (2/2, coarsest 16^2) to 1e-5.
  pressure_microbench  all-fluid domain, walls only, N(0,1) divergence with
                  its mean removed (seed 0xC3).
  batch_96        96 independent simulations (seed 0xC4), each sized
                  uniformly from {128^2, 256x128, 256^2, 384x256, 512^2,
                  768x512} (examples/multiple.rs steps several fluids side by
                  side); a pool of depth U[0.2,0.5]*H, 1-4 circular droplets
                  (r U[0.05,0.15]*min(W,H)) in the upper half, and every 30
                  steps 8 local forces at random cells with magnitude
                  U[0,50] m/s^2 in random directions; RBGS to 1e-5.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _capi as capi
from .plugin import Collider, RigidBody, RigidBodyKind

DT = 1.0 / 60.0
RHO = 99.7
LENGTH_UNIT = 10.0


@dataclass
class Scene:
    name: str
    cfg: capi.Config
    oneshot: List[capi.Source] = field(default_factory=list)
    continuous: List[capi.Source] = field(default_factory=list)
    bodies: List[RigidBody] = field(default_factory=list)
    dt: float = DT
    steps: int = 600

    @property
    def cells(self) -> int:
        return self.cfg.nx * self.cfg.ny

    def make(self, api: capi.Api) -> capi.Sim:
        """Creates the simulation on `api` with this scene's sources and bodies."""
        sim = capi.Sim(api, _copy_cfg(self.cfg))
        sim.set_sources(self.oneshot, True)
        sim.set_sources(self.continuous, False)
        if self.bodies:
            sim.set_obstacles([b.to_obstacle(i) for i, b in enumerate(self.bodies)])
        return sim


def _copy_cfg(c: capi.Config) -> capi.Config:
    n = capi.Config()
    import ctypes
    ctypes.memmove(ctypes.byref(n), ctypes.byref(c), ctypes.sizeof(c))
    return n


def aabb_source(center, half, velocity=(0.0, 0.0), mode=capi.SOURCE_MODE_SOURCE) -> capi.Source:
    s = capi.Source()
    s.center[0], s.center[1] = center
    s.data[0], s.data[1] = half
    s.velocity[0], s.velocity[1] = velocity
    s.shape = capi.SOURCE_AABB
    s.mode = mode
    return s


def circle_source(center, radius, velocity=(0.0, 0.0), mode=capi.SOURCE_MODE_SOURCE) -> capi.Source:
    s = capi.Source()
    s.center[0], s.center[1] = center
    s.data[0], s.data[1] = radius, 0.0
    s.velocity[0], s.velocity[1] = velocity
    s.shape = capi.SOURCE_CIRCLE
    s.mode = mode
    return s


def base_config(nx: int, ny: int) -> capi.Config:
    c = capi.default_config(nx, ny)
    c.length_unit = LENGTH_UNIT
    c.rho = RHO
    c.gravity[0], c.gravity[1] = 0.0, 9.8
    return c


def dam_break(n: int = 256, steps: int = 600) -> Scene:
    """C1: the examples/water_surface.rs scene at n x n (the CPU-runnable case)."""
    cfg = base_config(n, n)
    src = aabb_source((0.0, -0.2 * n), (0.5 * 1.0 * n, 0.5 * 0.6 * n))
    return Scene(f"dam_break_{n}", cfg, oneshot=[src], steps=steps)


def random_bodies(n_per_shape: int, size: int, seed: int, rho: float = RHO) -> List[RigidBody]:
    rng = np.random.default_rng(seed)
    half = 0.5 * size
    bodies: List[RigidBody] = []
    for shape in range(4):
        for _ in range(n_per_shape):
            if shape == 0:
                col = Collider.circle(float(rng.uniform(8, 32)))
            elif shape == 1:
                col = Collider.rectangle(2 * float(rng.uniform(6, 30)), 2 * float(rng.uniform(6, 30)))
            elif shape == 2:
                r = float(rng.uniform(5, 15))
                hl = float(rng.uniform(10, 30))
                col = Collider.capsule(r, 2 * hl)
            else:
                ang = np.sort(rng.uniform(0, 2 * math.pi, 3))
                rad = rng.uniform(10, 30, 3)
                pts = [(float(rad[k] * math.cos(ang[k])), float(rad[k] * math.sin(ang[k]))) for k in range(3)]
                col = Collider.triangle(*pts)
            margin = min(40.0, 0.15 * size)
            pos = (float(rng.uniform(-half + margin, half - margin)), float(rng.uniform(margin, half - margin)))
            rot = float(rng.uniform(0, 2 * math.pi))
            dens = float(rng.uniform(0.5, 2.0)) * rho
            bodies.append(RigidBody(col, pos, rot, (0.0, 0.0), 0.0, RigidBodyKind.Dynamic, dens))
    return bodies


def coupled(n: int = 512, steps: int = 1000, tolerance: float = 1e-5, seed: int = 0xC2,
            n_per_shape: int = 6, method: int = capi.PROJECTION_GAUSS_SEIDEL) -> Scene:
    """C2 (the benchmark scene): lower 40 % water, 24 random bodies, JFA, solve to tolerance."""
    cfg = base_config(n, n)
    cfg.reinit.method = capi.REINIT_JUMP_FLOODING
    cfg.projection.method = method
    cfg.projection.tolerance = tolerance
    cfg.projection.max_iterations = 20000
    cfg.projection.check_interval = 16
    depth = 0.4 * n
    src = aabb_source((0.0, -0.5 * n + 0.5 * depth), (0.5 * n, 0.5 * depth))
    bodies = random_bodies(n_per_shape, n, seed)
    return Scene(f"coupled_{n}", cfg, oneshot=[src], bodies=bodies, steps=steps)


def scale(n: int = 4096, steps: int = 200, tolerance: float = 1e-5, coarsest: int = 16) -> Scene:
    """C3: dam break with a static circle r = n/16 at the centre, MG to tolerance."""
    cfg = base_config(n, n)
    cfg.projection.method = capi.PROJECTION_MULTIGRID
    cfg.projection.tolerance = tolerance
    cfg.projection.max_iterations = 200
    cfg.projection.mg_levels = int(round(math.log2(n / coarsest))) + 1
    src = aabb_source((0.0, -0.2 * n), (0.5 * 1.0 * n, 0.5 * 0.6 * n))
    body = RigidBody(Collider.circle(n / 16.0), (0.0, 0.0), 0.0, kind=RigidBodyKind.Static, density=RHO)
    return Scene(f"scale_{n}", cfg, oneshot=[src], bodies=[body], steps=steps)


def microbench_inputs(n: int, seed: int = 0xC3):
    """All-fluid pressure microbench: phi = -1, walls only, N(0,1) RHS with its mean removed."""
    rng = np.random.default_rng(seed)
    b = rng.standard_normal((n, n)).astype(np.float32)
    b -= b.mean(dtype=np.float64).astype(np.float32)
    phi = -np.ones((n, n), dtype=np.float32)
    return phi, b


BATCH_SHAPES = [(128, 128), (256, 128), (256, 256), (384, 256), (512, 512), (768, 512)]


@dataclass
class BatchScene:
    name: str
    scenes: List[Scene]
    seed: int
    steps: int = 500
    force_every: int = 30
    forces_per_event: int = 8

    @property
    def cells(self) -> int:
        return sum(sc.cells for sc in self.scenes)

    def configs(self) -> List[capi.Config]:
        return [_copy_cfg(sc.cfg) for sc in self.scenes]

    def forces(self, i: int, step: int) -> List[capi.Force]:
        """Local forces of simulation i before frame `step` (every force_every frames, none at frame 0)."""
        if step == 0 or step % self.force_every:
            return []
        sc = self.scenes[i]
        rng = np.random.default_rng([self.seed, i, step])
        out = []
        for _ in range(self.forces_per_event):
            f = capi.Force()
            mag = float(rng.uniform(0.0, 50.0))
            ang = float(rng.uniform(0.0, 2.0 * math.pi))
            f.force[0], f.force[1] = mag * math.cos(ang), mag * math.sin(ang)
            f.position[0] = float(rng.integers(0, sc.cfg.nx))
            f.position[1] = float(rng.integers(0, sc.cfg.ny))
            out.append(f)
        return out

    def setup(self, sims) -> None:
        """Uploads each scene's sources to the matching simulation handle."""
        for sc, sim in zip(self.scenes, sims):
            sim.set_sources(sc.oneshot, True)
            sim.set_sources(sc.continuous, False)


def batch(n: int = 96, steps: int = 500, tolerance: float = 1e-5, seed: int = 0xC4,
          shapes: Optional[List[tuple]] = None) -> BatchScene:
    """C4: n independent pools with droplets and periodic local forces, RBGS to tolerance."""
    rng = np.random.default_rng(seed)
    shapes = shapes or BATCH_SHAPES
    scenes = []
    for i in range(n):
        nx, ny = shapes[int(rng.integers(0, len(shapes)))]
        cfg = base_config(nx, ny)
        cfg.projection.method = capi.PROJECTION_GAUSS_SEIDEL
        cfg.projection.tolerance = tolerance
        cfg.projection.max_iterations = 20000
        cfg.projection.check_interval = 16
        depth = float(rng.uniform(0.2, 0.5)) * ny
        pool = aabb_source((0.0, -0.5 * ny + 0.5 * depth), (0.5 * nx, 0.5 * depth))
        drops = []
        for _ in range(int(rng.integers(1, 5))):
            r = float(rng.uniform(0.05, 0.15)) * min(nx, ny)
            cx = float(rng.uniform(-0.5 * nx + r, 0.5 * nx - r))
            cy = float(rng.uniform(r, 0.5 * ny - r))
            drops.append(circle_source((cx, cy), r))
        scenes.append(Scene(f"batch_{i}_{nx}x{ny}", cfg, oneshot=[pool] + drops, steps=steps))
    return BatchScene(f"batch_{n}", scenes, seed, steps=steps)

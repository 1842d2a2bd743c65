"""Host rigid-body integrator for the two-way coupled scenes.

The reference hands the fluid forces to avian2d (fluid_to_solid.rs:180-209):
force * dt / grid_length with y flipped, torque negated, applied to Dynamic
bodies only.  avian2d is not available here, so this module integrates the
bodies itself: semi-implicit Euler under gravity plus that applied force,
and a clamp that keeps each body's centre inside the fluid domain.
Collisions between bodies are not resolved.  World units are grid cells,
centred on the domain, y up (the identity fluid transform).
"""
from __future__ import annotations

import math
from typing import List, Sequence

import numpy as np

from .plugin import RigidBody, RigidBodyKind


class RigidWorld:
    def __init__(self, bodies: Sequence[RigidBody], domain: tuple, gravity: float, grid_length: float):
        self.bodies: List[RigidBody] = list(bodies)
        self.half = (0.5 * domain[0], 0.5 * domain[1])
        self.gravity = gravity  # world units / s^2, acting along -y
        self.grid_length = grid_length

    def apply_fluid_forces(self, forces: np.ndarray, dt: float):
        """forces: (n, 3) array of (fx, fy, torque) from the fluid (grid frame, y down)."""
        self._pending = forces[: len(self.bodies)].astype(np.float64)
        self._pending_dt = dt

    def step(self, dt: float):
        pend = getattr(self, "_pending", None)
        for i, b in enumerate(self.bodies):
            if b.kind != RigidBodyKind.Dynamic:
                continue
            m = b.density * b.collider.area()
            inertia = m * b.collider.inertia_per_mass()
            fx = fy = tq = 0.0
            if pend is not None and i < len(pend):
                f = pend[i]
                s = self._pending_dt / self.grid_length
                fx, fy, tq = f[0] * s, -f[1] * s, -f[2] * s
            vx, vy = b.linear_velocity
            vx += (fx / m) * dt
            vy += (fy / m - self.gravity) * dt
            w = b.angular_velocity + (tq / inertia) * dt if inertia > 0 else b.angular_velocity
            px, py = b.position
            px += vx * dt
            py += vy * dt
            r = _extent(b)
            lox, hix = -self.half[0] + 1 + r, self.half[0] - 1 - r
            loy, hiy = -self.half[1] + 1 + r, self.half[1] - 1 - r
            if px < lox:
                px, vx = lox, max(vx, 0.0)
            elif px > hix:
                px, vx = hix, min(vx, 0.0)
            if py < loy:
                py, vy = loy, max(vy, 0.0)
            elif py > hiy:
                py, vy = hiy, min(vy, 0.0)
            b.position = (px, py)
            b.linear_velocity = (vx, vy)
            b.angular_velocity = w
            b.rotation = math.fmod(b.rotation + w * dt, 2.0 * math.pi)
        self._pending = None


def _extent(b: RigidBody) -> float:
    v = b.collider.values
    if b.collider.shape == 0:
        return v[0]
    if b.collider.shape == 1:
        return math.hypot(v[0], v[1])
    if b.collider.shape == 2:
        return max(math.hypot(v[0], v[1]), math.hypot(v[2], v[3])) + v[4]
    return max(math.hypot(v[0], v[1]), math.hypot(v[2], v[3]), math.hypot(v[4], v[5]))


def device_bodies(bodies: Sequence[RigidBody]):
    """The bodies as efl_rigid_body records for the device-side coupling
    (body i drives obstacle i of pack_obstacles)."""
    from . import _capi as capi
    out = []
    for i, b in enumerate(bodies):
        r = capi.RigidBodyC()
        r.position[0], r.position[1] = b.position
        r.rotation = b.rotation
        r.linear_velocity[0], r.linear_velocity[1] = b.linear_velocity
        r.angular_velocity = b.angular_velocity
        m = b.density * b.collider.area()
        r.mass = m
        r.inertia = m * b.collider.inertia_per_mass()
        r.extent = _extent(b)
        r.dynamic = 1 if b.kind == RigidBodyKind.Dynamic else 0
        r.obstacle = i
        out.append(r)
    return out

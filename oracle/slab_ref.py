"""CPU restatement of one row slab of the tolerance-driven pressure solve.

Test infrastructure: the numpy counterpart of the efl_slab_* entry points
(bevy_eulerian_fluid_b200/csrc/efl_slab.cuh), with the same methods as
bevy_eulerian_fluid_b200.slab.CudaSlab, so that the host driver
(RowSlabSolver) can run its halo exchange and residual gathering on CPU
ranks and be checked against the unsplit oracle solve.  Never used by the
product path.

The arithmetic follows the oracle's mixed-precision solve
(oracle/efl_oracle.cpp, mix_coefficients and gs_mixed_solve: the residual of
residual.wgsl:33-54 in FP64, the red-black update of
gauss_seidel.wgsl:44-88 in f32 on the correction) operation for operation,
in the same rounding order: f32 products and sums for the sweep, FP64 for
the residual, the per-row sums sequential in x.
"""
from __future__ import annotations

import numpy as np


class SlabRef:
    def __init__(self, nx: int, ny: int, row0: int, rows: int, dx: float, dt: float, rho: float,
                 sor_weight: float = 1.9):
        self.nx, self.ny, self.row0, self.rows = nx, ny, row0, rows
        self.dx, self.dt, self.rho = np.float32(dx), np.float32(dt), np.float32(rho)
        self.weight = np.float32(sor_weight)
        self.omw = np.float32(1.0) - self.weight
        h = rows + 2  # halo row above (0) and below (rows + 1); zero beyond the domain
        self.x = np.zeros((h, nx), np.float64)
        self.d = np.zeros((h, nx), np.float32)
        self.ls = np.zeros((h, nx), np.float32)

    def _field(self, field: int) -> np.ndarray:
        return (self.x, self.d, self.ls)[field]

    def load(self, levelset_air, area_fraction, divergence, pressure):
        self.ls[1:-1] = levelset_air
        self.af = np.array(area_fraction, np.float32).reshape(self.rows, self.nx, 4)
        self.b = np.asarray(divergence, np.float32).astype(np.float64)
        self.x[1:-1] = np.asarray(pressure, np.float32).astype(np.float64)

    def edge(self, field: int, side: int, buf):
        buf.numpy()[:] = self._field(field)[1 if side == 0 else self.rows]

    def set_halo(self, field: int, side: int, buf):
        if (side == 0 and self.row0 == 0) or (side == 1 and self.row0 + self.rows == self.ny):
            raise ValueError("no halo row beyond the domain's edge")
        self._field(field)[0 if side == 0 else self.rows + 1] = buf.numpy()

    def prepare(self):
        """mix_coefficients: mode, w, den (FP64, neighbours in the order left, right, up, down), inv."""
        nx, rows = self.nx, self.rows
        lij = self.ls[1:-1]
        f = self.af
        gy = self.row0 + np.arange(rows)[:, None]
        gx = np.arange(nx)[None, :]
        counted = (lij < 0) & ~np.all(f == 0, axis=2)
        den = np.zeros((rows, nx), np.float64)
        w = np.zeros((rows, nx, 4), np.float32)
        lsp = np.pad(self.ls, ((0, 0), (1, 1)))  # one zero column each side (out of range is masked below)
        for q, (ox, oy) in enumerate(((-1, 0), (1, 0), (0, -1), (0, 1))):
            inb = (gx + ox >= 0) & (gx + ox < nx) & (gy + oy >= 0) & (gy + oy < self.ny)
            level = lsp[1 + oy:1 + oy + rows, 1 + ox:1 + ox + nx]
            fq = f[:, :, q]
            fluid = inb & (level < 0)
            ghost = inb & ~(level < 0)
            with np.errstate(divide="ignore", invalid="ignore"):
                gterm = fq.astype(np.float64) * (1.0 - level.astype(np.float64) / lij.astype(np.float64))
            term = np.where(fluid, fq.astype(np.float64), np.where(ghost, gterm, 0.0))
            den = np.where(counted, den + term, den)
            w[:, :, q] = np.where(counted & fluid, fq, np.float32(0))
        update = counted & ~(np.abs(den) < np.float64(np.float32(1.0e-6)))
        with np.errstate(divide="ignore"):
            inv = np.where(update, (1.0 / np.where(update, den, 1.0)).astype(np.float32), np.float32(0))
        self.counted, self.update = counted, update
        self.w, self.den, self.inv = w, den, inv.astype(np.float32)

    def residual(self) -> np.ndarray:
        """r in FP64, rc = f32(cdiv * r) on updated cells, d = 0; per row the sequential sums of r^2, b^2."""
        dx = np.float64(self.dx)
        cdiv = dx * dx * np.float64(self.rho) / np.float64(self.dt)
        factor = np.float64(self.dt) / np.float64(self.rho) / dx / dx
        xp = np.pad(self.x, ((0, 0), (1, 1)))
        rows, nx = self.rows, self.nx
        nb = [xp[1:-1, 0:nx], xp[1:-1, 2:nx + 2], xp[0:rows, 1:nx + 1], xp[2:rows + 2, 1:nx + 1]]
        w = self.w.astype(np.float64)
        s = w[:, :, 0] * nb[0]
        s = s + w[:, :, 1] * nb[1]
        s = s + w[:, :, 2] * nb[2]
        s = s + w[:, :, 3] * nb[3]
        rv = self.b - factor * (self.den * self.x[1:-1] - s)
        rv = np.where(self.counted, rv, 0.0)
        self.rc = np.where(self.update, (cdiv * rv).astype(np.float32), np.float32(0))
        self.d[1:-1] = 0
        sr = np.cumsum(np.where(self.counted, rv * rv, 0.0), axis=1)[:, -1]
        sb = np.cumsum(np.where(self.counted, self.b * self.b, 0.0), axis=1)[:, -1]
        return np.stack([sr, sb], axis=1)

    def sweep(self, color: int):
        rows, nx = self.rows, self.nx
        gy = self.row0 + np.arange(rows)[:, None]
        gx = np.arange(nx)[None, :]
        sel = self.update & (((gx + gy) & 1) == color)
        dp = np.pad(self.d, ((0, 0), (1, 1)))
        nb = [dp[1:-1, 0:nx], dp[1:-1, 2:nx + 2], dp[0:rows, 1:nx + 1], dp[2:rows + 2, 1:nx + 1]]
        nume = self.rc + self.w[:, :, 0] * nb[0]
        nume = nume + self.w[:, :, 1] * nb[1]
        nume = nume + self.w[:, :, 2] * nb[2]
        nume = nume + self.w[:, :, 3] * nb[3]
        new = self.weight * (nume * self.inv) + self.omw * self.d[1:-1]
        self.d[1:-1] = np.where(sel, new, self.d[1:-1])

    def apply(self):
        self.x[1:-1] = np.where(self.update, self.x[1:-1] + self.d[1:-1].astype(np.float64), 0.0)

    def read(self) -> np.ndarray:
        return self.x[1:-1].copy()

    def close(self):
        pass

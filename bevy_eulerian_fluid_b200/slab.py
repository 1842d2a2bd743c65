"""Row-slab split of one domain's pressure solve across processes.

A domain too large for one device (the 4096^2 scale scene and beyond) is cut
into horizontal slabs of whole rows, one per process and GPU.  Each slab runs
the tolerance-driven red-black Gauss-Seidel solve (the FP64-iterate form of
ProjectionMethod::GaussSeidel, projection.rs:89-164 and
gauss_seidel.wgsl:44-88) on its own rows through the efl_slab_* entry points
of include/efl.h; this module is the host side that makes the slabs one
solve:

  * halo exchange of depth one across every cut, point to point with the two
    neighbouring ranks: the level set once (for the ghost-fluid coefficient
    of the rows next to the cut), the FP64 iterate before every residual and
    the f32 correction before every half-sweep;
  * the relative residual sqrt(sum r^2) / sqrt(sum b^2): every rank gathers
    the per-row FP64 partials of all slabs and adds them in row order, so all
    ranks take the same convergence decision in the same order of additions
    as a single-device solve that sums row by row.

The collective steps are the same on every rank in the same order, and the
slabs compute the unsplit solve's iterates bit for bit.  The exchange moves
torch tensors: CPU tensors with the gloo backend, device tensors with NCCL.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch
import torch.distributed as dist

from . import _capi as capi

SLAB_X, SLAB_D, SLAB_LEVELSET = capi.SLAB_X, capi.SLAB_D, capi.SLAB_LEVELSET
_DTYPES = {SLAB_X: torch.float64, SLAB_D: torch.float32, SLAB_LEVELSET: torch.float32}


def slab_rows(ny: int, world: int, rank: int) -> tuple[int, int]:
    """(row0, rows) of rank `rank`: contiguous slabs in rank order, sizes differing by at most one row."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    if ny < world:
        raise ValueError(f"{ny} rows cannot be split into {world} slabs")
    base, extra = divmod(ny, world)
    row0 = rank * base + min(rank, extra)
    return row0, base + (1 if rank < extra else 0)


class CudaSlab:
    """One slab on a GPU through the C ABI (efl_slab_*)."""

    def __init__(self, api: capi.Api, nx: int, ny: int, row0: int, rows: int, dx: float, dt: float, rho: float,
                 sor_weight: float = 1.9, device: int = 0):
        self.api = api
        self.nx, self.ny, self.row0, self.rows = nx, ny, row0, rows
        d = capi.SlabDesc(device, nx, ny, row0, rows, dx, dt, rho, sor_weight)
        h = C.c_void_p()
        self._check(api.slab_create(C.byref(d), C.byref(h)))
        self.h = h.value

    def _check(self, st: int):
        if st != capi.OK:
            msg = self.api.last_error(None)
            raise capi.EflError(st, msg.decode() if msg else "")

    def load(self, levelset_air, area_fraction, divergence, pressure):
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (levelset_air, area_fraction, divergence, pressure)]
        want = [(self.rows, self.nx), (self.rows, self.nx, 4), (self.rows, self.nx), (self.rows, self.nx)]
        for a, w in zip(arrs, want):
            if a.shape != w:
                raise ValueError(f"expected rows of shape {w}, got {a.shape}")
        self._check(self.api.slab_load(self.h, *[a.ctypes.data_as(C.c_void_p) for a in arrs]))

    def edge(self, field: int, side: int, buf: torch.Tensor):
        self._check(self.api.slab_halo(self.h, field, side, 0, C.c_void_p(buf.data_ptr())))

    def set_halo(self, field: int, side: int, buf: torch.Tensor):
        self._check(self.api.slab_halo(self.h, field, side, 1, C.c_void_p(buf.data_ptr())))

    def prepare(self):
        self._check(self.api.slab_prepare(self.h))

    def residual(self) -> np.ndarray:
        out = np.empty((self.rows, 2), dtype=np.float64)
        self._check(self.api.slab_residual(self.h, out.ctypes.data_as(C.c_void_p)))
        return out

    def sweep(self, color: int):
        self._check(self.api.slab_sweep(self.h, color))

    def apply(self):
        self._check(self.api.slab_apply(self.h))

    def read(self) -> np.ndarray:
        out = np.empty((self.rows, self.nx), dtype=np.float64)
        self._check(self.api.slab_read(self.h, out.ctypes.data_as(C.c_void_p)))
        return out

    def close(self):
        if self.h:
            self.api.slab_destroy(self.h)
            self.h = None


@dataclass
class SlabSolveStats:
    iterations: int
    residual_initial: float
    residual: float
    converged: bool


def _relative(R: float, B: float) -> float:
    if B > 0.0:
        return float(np.sqrt(R) / np.sqrt(B))
    return float("inf") if R > 0.0 else 0.0


class RowSlabSolver:
    """The host driver of one rank's slab. `backend` computes on the slab's rows (CudaSlab, or any object with
    its methods); ranks hold the slabs in row order (rank r: slab_rows(ny, world, r))."""

    def __init__(self, backend, nx: int, ny: int, comm_device: Optional[torch.device] = None):
        if not dist.is_initialized():
            raise RuntimeError("RowSlabSolver needs an initialised torch.distributed process group")
        self.b = backend
        self.nx, self.ny = nx, ny
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.row0, self.rows = slab_rows(ny, self.world, self.rank)
        if (backend.row0, backend.rows) != (self.row0, self.rows):
            raise ValueError(f"backend holds rows [{backend.row0}, {backend.row0 + backend.rows}), rank {self.rank} "
                             f"owns [{self.row0}, {self.row0 + self.rows})")
        if comm_device is None:
            comm_device = torch.device("cuda", torch.cuda.current_device()) \
                if dist.get_backend() == "nccl" else torch.device("cpu")
        self.dev = torch.device(comm_device)
        self.up = self.rank - 1 if self.row0 > 0 else None
        self.down = self.rank + 1 if self.row0 + self.rows < ny else None
        self._bufs = {f: [torch.zeros(nx, dtype=dt, device=self.dev) for _ in range(4)] for f, dt in _DTYPES.items()}
        self.max_rows = slab_rows(ny, self.world, 0)[1]
        self._part = torch.zeros((self.max_rows, 2), dtype=torch.float64, device=self.dev)
        self._gather = [torch.zeros_like(self._part) for _ in range(self.world)]
        self.exchanges = 0

    def _sync(self):
        if self.dev.type == "cuda":
            torch.cuda.current_stream(self.dev).synchronize()

    def exchange(self, field: int):
        """Depth-one halo exchange of `field` with the neighbouring slabs."""
        send_top, send_bot, recv_top, recv_bot = self._bufs[field]
        reqs = []
        if self.up is not None:
            self.b.edge(field, 0, send_top)
            reqs.append(dist.isend(send_top, self.up, tag=2 * field))
            reqs.append(dist.irecv(recv_top, self.up, tag=2 * field + 1))
        if self.down is not None:
            self.b.edge(field, 1, send_bot)
            reqs.append(dist.isend(send_bot, self.down, tag=2 * field + 1))
            reqs.append(dist.irecv(recv_bot, self.down, tag=2 * field))
        for r in reqs:
            r.wait()
        self._sync()
        if self.up is not None:
            self.b.set_halo(field, 0, recv_top)
        if self.down is not None:
            self.b.set_halo(field, 1, recv_bot)
        self.exchanges += 1

    def setup(self, levelset_air, area_fraction, divergence, pressure):
        """Own rows of the step's fields (the previous pressure is the start iterate)."""
        self.b.load(levelset_air, area_fraction, divergence, pressure)
        self.exchange(SLAB_LEVELSET)
        self.b.prepare()

    def relative_residual(self) -> float:
        self.exchange(SLAB_X)
        part = self.b.residual()
        self._part.zero_()
        self._part[:self.rows].copy_(torch.from_numpy(part))
        dist.all_gather(self._gather, self._part)
        rows = np.concatenate([g[:slab_rows(self.ny, self.world, r)[1]].cpu().numpy()
                               for r, g in enumerate(self._gather)])
        tot = np.cumsum(rows, axis=0)[-1]  # row order, sequential
        return _relative(float(tot[0]), float(tot[1]))

    def solve(self, tolerance: float, max_iterations: int, check_interval: int = 16) -> SlabSolveStats:
        """Red-black SOR on the f32 correction in blocks of check_interval iterations, FP64 residual between
        blocks, until ||b - A p|| / ||b|| <= tolerance or max_iterations (the single-device solve's loop)."""
        rel = self.relative_residual()
        r0, iters = rel, 0
        chk = max(1, int(check_interval))
        while not rel <= tolerance and iters < max_iterations:
            n = min(chk, max_iterations - iters)
            for _ in range(n):
                for color in (1, 0):
                    self.exchange(SLAB_D)
                    self.b.sweep(color)
            self.b.apply()
            iters += n
            rel = self.relative_residual()
        return SlabSolveStats(iters, r0, rel, bool(rel <= tolerance))

    def gather_pressure(self) -> np.ndarray:
        """The whole domain's iterate (ny x nx, FP64) on every rank."""
        x = torch.zeros((self.max_rows, self.nx), dtype=torch.float64, device=self.dev)
        x[:self.rows].copy_(torch.from_numpy(self.b.read()))
        out = [torch.zeros_like(x) for _ in range(self.world)]
        dist.all_gather(out, x)
        return np.concatenate([o[:slab_rows(self.ny, self.world, r)[1]].cpu().numpy() for r, o in enumerate(out)])

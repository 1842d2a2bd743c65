"""Training and evaluation of the learned warm start (an extension).

The network (efl_unet_*, tensor-core kernels) learns the change of the
pressure over a step from the system about to be solved; training samples
are recorded from simulations of C2-style scenes (water in the lower 40 %,
random bodies) with seeds other than the benchmark's, solved to the
tolerance by MGPCG.  Evaluation steps a scene twice from the same state --
once warm-started by the network, once from the previous pressure -- and
compares the solver's iterations and time.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import List

from . import _capi as capi
from . import scenes


# (cin, cout) of the network's 15 convolutions and the level each runs at
# (resolution / 2^level), for FLOP counts.
UNET_CONVS = [(16, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2), (64, 64, 3), (64, 64, 3),
              (128, 64, 2), (64, 64, 2), (96, 32, 1), (32, 32, 1), (48, 16, 0), (16, 16, 0), (16, 16, 0)]


def forward_flops(nx: int, ny: int) -> float:
    """Multiply-adds x 2 of one forward pass (the padded channels included)."""
    return float(sum(2 * 9 * ci * co * (nx >> lv) * (ny >> lv) for ci, co, lv in UNET_CONVS))


@dataclass
class TrainLog:
    losses: List[float] = field(default_factory=list)
    seconds: float = 0.0
    samples: int = 0


def train(api: capi.Api, size: int = 256, seeds=(1, 2, 3, 4), steps: int = 200, lr: float = 1e-3,
          n_per_shape: int = 6, net: capi.UNet | None = None, max_size: int | None = None,
          device: int = 0, extra=()) -> tuple[capi.UNet, TrainLog]:
    """Online training: every simulation step records one sample, one Adam step follows.
    Scenes: C2-style coupled scenes at `size` for `seeds`, plus (size, seed) pairs in `extra`."""
    runs = [(size, s) for s in seeds] + list(extra)
    big = max(sz for sz, _ in runs)
    net = net or capi.UNet(api, max(max_size or 0, big), max(max_size or 0, big), seed=0xC5, device=device)
    sims = []
    for sz, s in runs:
        sc = scenes.coupled(sz, seed=s, n_per_shape=n_per_shape, method=capi.PROJECTION_MGPCG)
        sc.cfg.device = device
        sim = sc.make(api)
        sim.step(sc.dt)  # init sequence
        net.attach(sim, warm_start=False, record=True)
        sims.append((sc, sim))
    log = TrainLog()
    t0 = time.time()
    for _ in range(steps):
        for sc, sim in sims:
            sim.step(sc.dt)
            log.losses.append(net.train_step(lr))
            log.samples += 1
    log.seconds = time.time() - t0
    for _, sim in sims:
        net.attach(sim, warm_start=False, record=False)
        sim.close()
    return net, log


# Fields that carry a simulation's state from one step to the next.
STATE_FIELDS = [capi.FIELD_U, capi.FIELD_V, capi.FIELD_U1, capi.FIELD_V1, capi.FIELD_U_SOLID, capi.FIELD_V_SOLID,
                capi.FIELD_LEVELSET_AIR, capi.FIELD_LEVELSET_AIR1, capi.FIELD_LEVELSET_SOLID, capi.FIELD_DIVERGENCE,
                capi.FIELD_PRESSURE, capi.FIELD_GRAD_LEVELSET, capi.FIELD_AREA_FRACTION, capi.FIELD_SOLID_ID,
                capi.FIELD_U_VALID, capi.FIELD_V_VALID, capi.FIELD_FIM_LABELS]


def copy_state(src: capi.Sim, dst: capi.Sim):
    for f in STATE_FIELDS:
        dst.set(f, src.get(f))


def compare(api: capi.Api, net: capi.UNet, scene: scenes.Scene, warmup: int = 5, steps: int = 10) -> dict:
    """Steps two copies of `scene` in lockstep, one warm-started by the
    network, one from the previous pressure (the same state before every
    step); per step and copy: (iterations, initial relative residual, solve
    ms, converged)."""
    a, b = scene.make(api), scene.make(api)
    for sim in (a, b):
        sim.step(scene.dt)
        for _ in range(warmup):
            sim.step(scene.dt)
    copy_state(b, a)
    net.attach(a, warm_start=True)
    out = {"learned": [], "plain": []}
    for _ in range(steps):
        sa, sb = a.step(scene.dt), b.step(scene.dt)
        out["learned"].append((int(sa.pressure_iterations), float(sa.residual_initial), a.projection_ms(),
                               bool(sa.converged)))
        out["plain"].append((int(sb.pressure_iterations), float(sb.residual_initial), b.projection_ms(),
                             bool(sb.converged)))
        copy_state(b, a)  # the same state again for the next step
    net.attach(a, warm_start=False)
    a.close()
    b.close()
    return out

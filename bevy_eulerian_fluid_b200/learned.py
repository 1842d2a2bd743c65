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

import copy
import math
import os
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _capi as capi
from . import scenes

# Weights of the network trained offline by `pretrain` (python -m bevy_eulerian_fluid_b200.learned):
# the FP32 master parameters, the coarsening factor they were trained for, and how they were made.
WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "unet_warm_start.npz")


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
          device: int = 0, extra=(), coarse: int = 1) -> tuple[capi.UNet, TrainLog]:
    """Online training: every simulation step records one sample, one Adam step follows.
    Scenes: C2-style coupled scenes at `size` for `seeds`, plus (size, seed) pairs in `extra`;
    the network runs on the grid coarsened by `coarse`."""
    runs = [(size, s) for s in seeds] + list(extra)
    big = max(sz for sz, _ in runs)
    net = net or capi.UNet(api, max(max_size or 0, big), max(max_size or 0, big), seed=0xC5, device=device)
    net.set_coarsening(coarse)
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


def fp64_solve(phi: np.ndarray, af: np.ndarray, b: np.ndarray, dx: float, dt: float, rho: float):
    """Sparse direct FP64 solve (CPU) of the pressure system the projection iterates on: the operator of
    residual.wgsl:33-54 (ghost-fluid weights f (1 - phi_j / phi_i) for air neighbours) over the counted
    cells (phi < 0, not fully solid).  Returns (x on a full grid, the counted-cell mask)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    H, W = phi.shape
    phi = phi.astype(np.float64)
    act = (phi < 0) & ~(af == 0).all(-1)
    idx = -np.ones((H, W), np.int64)
    idx[act] = np.arange(int(act.sum()))
    fac = dt / rho / dx / dx
    ys, xs = np.nonzero(act)
    rows, cols, vals = [], [], []
    diag = np.zeros(len(ys))
    for k, (ox, oy) in enumerate(((-1, 0), (1, 0), (0, -1), (0, 1))):
        jx, jy = xs + ox, ys + oy
        inb = (jx >= 0) & (jx < W) & (jy >= 0) & (jy < H)
        f = af[ys, xs, k].astype(np.float64)
        pj = np.where(inb, phi[np.clip(jy, 0, H - 1), np.clip(jx, 0, W - 1)], 0.0)
        fluid = inb & (pj < 0)
        air = inb & ~fluid
        diag += np.where(fluid, f, 0.0) + np.where(air, f * (1.0 - pj / phi[ys, xs]), 0.0)
        nb = np.where(fluid, idx[np.clip(jy, 0, H - 1), np.clip(jx, 0, W - 1)], -1)
        sel = nb >= 0
        rows.append(idx[ys, xs][sel])
        cols.append(nb[sel])
        vals.append(-f[sel] * fac)
    rows.append(idx[ys, xs])
    cols.append(idx[ys, xs])
    vals.append(diag * fac)
    n = int(act.sum())
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    x = np.zeros((H, W))
    x[act] = spla.spsolve(A.tocsc(), b[act].astype(np.float64))
    return x, act


def _block_mean(a: np.ndarray, m: np.ndarray, f: int) -> np.ndarray:
    H, W = a.shape
    s = (a * m).reshape(H // f, f, W // f, f).sum(axis=(1, 3))
    c = m.reshape(H // f, f, W // f, f).sum(axis=(1, 3))
    return np.where(c > 0, s / np.maximum(c, 1), 0.0)


def prediction_error(api: capi.Api, net: capi.UNet, scene: scenes.Scene, warmup: int = 5, block: int = 8) -> dict:
    """The network's warm start judged against an FP64 CPU solve of the same Poisson system: after `warmup`
    steps, the stages before the projection, then the projection with no iterations (the start iterate
    only: previous pressure + the network's correction), against a sparse direct solve x* of that system.
    captured = 1 - |x_start - x*| / |p_prev - x*| (the share of the correction the network supplies, 1 =
    all of it), also for the block means over `block` x `block` cells (the part the sweeps remove slowest),
    and |x_start - x*| / |x*|."""
    sim = scene.make(api)
    sim.step(scene.dt)
    for _ in range(warmup):
        sim.step(scene.dt)
    for st in range(capi.STAGE_UPDATE_SOLID, capi.STAGE_DIVERGENCE + 1):
        sim.run_stage(st, scene.dt)
    p_prev = sim.get(capi.FIELD_PRESSURE).astype(np.float64)
    proj = capi.Projection()
    import ctypes
    ctypes.memmove(ctypes.byref(proj), ctypes.byref(scene.cfg.projection), ctypes.sizeof(proj))
    proj.max_iterations = 0
    sim.set_projection(proj)
    net.attach(sim, warm_start=True)
    sim.run_stage(capi.STAGE_PROJECTION, scene.dt)
    net.attach(sim, warm_start=False)
    start = sim.get(capi.FIELD_PRESSURE).astype(np.float64)
    phi, af, b = sim.get(capi.FIELD_LEVELSET_AIR), sim.get(capi.FIELD_AREA_FRACTION), sim.get(capi.FIELD_DIVERGENCE)
    sim.close()
    dx = float(np.float32(1.0) / np.float32(scene.cfg.length_unit))
    x, act = fp64_solve(phi, af, b, dx, float(np.float32(scene.dt)), float(np.float32(scene.cfg.rho)))
    m = act.astype(np.float64)
    e_prev = np.linalg.norm((p_prev - x)[act])
    e_start = np.linalg.norm((start - x)[act])
    bp, bs, bx = (_block_mean(v, m, block) for v in (p_prev, start, x))
    ce_prev, ce_start = np.linalg.norm(bp - bx), np.linalg.norm(bs - bx)
    return {"captured": float(1.0 - e_start / e_prev) if e_prev > 0 else 0.0,
            "captured_block_means": float(1.0 - ce_start / ce_prev) if ce_prev > 0 else 0.0,
            "relative_error_start": float(e_start / np.linalg.norm(x[act])),
            "relative_error_previous": float(e_prev / np.linalg.norm(x[act])), "block": block,
            "cells": int(act.sum())}


def save_weights(net: capi.UNet, coarse: int, info: dict, path: str = WEIGHTS_PATH) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, params=net.get_params(), coarse=np.int32(coarse),
             info=np.array(repr(sorted(info.items()))))


def load_weights(api: capi.Api, max_nx: int, max_ny: int, path: str = WEIGHTS_PATH,
                 device: int = 0) -> Optional[capi.UNet]:
    """The pretrained network (None if the weights file is absent), coarsening set as trained."""
    if not os.path.exists(path):
        return None
    d = np.load(path)
    net = capi.UNet(api, max_nx, max_ny, seed=0xC5, device=device)
    net.set_params(d["params"])
    net.set_coarsening(int(d["coarse"]))
    return net


def pretrain(api: capi.Api, samples: int = 50000, coarse: int = 8, lr: float = 1e-3, lr_final: float = 5e-5,
             episode: int = 120, live: int = 8, pools: float = 0.0, seed0: int = 1000,
             target_tolerance: float = 1e-5, device: int = 0, log=print) -> tuple[capi.UNet, TrainLog]:
    """Offline training for the committed weights: `samples` (input, converged correction) pairs, MGPCG to
    1e-5 for the targets, from two kinds of scenes with seeds from seed0 (never the benchmark's):
      * C2-style coupled scenes (water in the lower 40 %, 24 random bodies, the two-way coupling loop) at
        256^2 (three in four) and 512^2;
      * C4-style pools (a fraction `pools` of the scenes): a pool with 1-4 droplets at one of the C4 sizes
        (128^2 ... 768x512), 8 local forces every 30 steps.
    `live` scenes step round-robin; each lives `episode` steps and is then replaced by a scene of a fresh
    seed, so the samples span splashes and settling of many configurations.  Every step records one sample
    and one Adam step (cosine learning-rate decay from lr to lr_final) follows.  The training scenes are
    solved to `target_tolerance` (where the pressure hardly changes between steps, as in a settled pool,
    a target solved to 1e-5 is mostly the solver's own tolerance error)."""
    from .plugin import pack_obstacles
    from .rigid import RigidWorld
    big = max(768, max(w for w, _ in scenes.BATCH_SHAPES))
    net = capi.UNet(api, big, big, seed=0xC5, device=device)
    net.set_coarsening(coarse)
    rng = np.random.default_rng(seed0)
    next_seed = [seed0]

    def spawn():
        seed = next_seed[0]
        next_seed[0] += 1
        if rng.uniform() < pools:
            bs = scenes.batch(1, seed=seed)
            bs.force_every = 30
            sc = bs.scenes[0]
            sc.cfg.projection.method = capi.PROJECTION_MGPCG
            rigid = None
        else:
            sz = 256 if rng.uniform() < 0.75 else 512
            bs = None
            sc = scenes.coupled(sz, seed=seed, method=capi.PROJECTION_MGPCG)
            rigid = RigidWorld(copy.deepcopy(list(sc.bodies)), (sz, sz), gravity=9.8 * scenes.LENGTH_UNIT,
                               grid_length=1.0 / scenes.LENGTH_UNIT)
        sc.cfg.device = device
        sc.cfg.projection.tolerance = target_tolerance
        sc.cfg.projection.max_iterations = 200
        sim = sc.make(api)
        sim.step(sc.dt)
        net.attach(sim, warm_start=False, record=True)
        return [sc, sim, rigid, bs, 0]

    live_sims = [spawn() for _ in range(live)]
    tl = TrainLog()
    t0 = time.time()
    while tl.samples < samples:
        for slot in range(live):
            sc, sim, rigid, bs, age = live_sims[slot]
            if bs is not None:
                f = bs.forces(0, age + 1)
                if f:
                    sim.set_local_forces(f)
            sim.step(sc.dt)
            if rigid is not None:
                rigid.apply_fluid_forces(sim.solid_forces(), sc.dt)
                rigid.step(sc.dt)
                sim.set_obstacles(pack_obstacles(rigid.bodies))
            frac = tl.samples / samples
            rate = lr_final + 0.5 * (lr - lr_final) * (1.0 + math.cos(math.pi * frac))
            tl.losses.append(net.train_step(rate))
            tl.samples += 1
            live_sims[slot][4] = age + 1
            if age + 1 >= episode:
                net.attach(sim, warm_start=False, record=False)
                sim.close()
                live_sims[slot] = spawn()
            if tl.samples % 5000 == 0 and log:
                log(f"{tl.samples} samples, {time.time() - t0:.0f} s, median relative loss of the last 1000 "
                    f"{np.median(tl.losses[-1000:]):.4f}")
            if tl.samples >= samples:
                break
    tl.seconds = time.time() - t0
    for _, sim, _, _, _ in live_sims:
        net.attach(sim, warm_start=False, record=False)
        sim.close()
    return net, tl


def main():
    import argparse
    ap = argparse.ArgumentParser(description="offline training of the learned warm start's weights")
    ap.add_argument("--samples", type=int, default=50000)
    ap.add_argument("--coarse", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--pools", type=float, default=0.0, help="share of C4-style pool scenes")
    ap.add_argument("--target-tolerance", type=float, default=1e-5)
    ap.add_argument("--out", default=WEIGHTS_PATH)
    args = ap.parse_args()
    api = capi.load()
    net, tl = pretrain(api, samples=args.samples, coarse=args.coarse, lr=args.lr, pools=args.pools,
                       target_tolerance=args.target_tolerance)
    q = max(1, len(tl.losses) // 10)
    info = {"samples": tl.samples, "seconds": round(tl.seconds, 1), "coarse": args.coarse,
            "scenes": f"C2-style coupled (256^2, 512^2) and, {args.pools:.0%} of them, C4-style pools (C4 sizes), "
                      f"seeds from 1000, MGPCG to {args.target_tolerance:g}",
            "median_relative_loss_by_tenth": [round(float(np.median(tl.losses[i * q:(i + 1) * q])), 4)
                                              for i in range(10)]}
    save_weights(net, args.coarse, info, args.out)
    print(info)


if __name__ == "__main__":
    main()

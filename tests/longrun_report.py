"""Long-run mass drift and post-projection divergence, GPU next to the CPU oracle.

Test infrastructure (run by hand, not collected by pytest).  One backend per
run, so the slow oracle arm can run on any host while the GPU arm runs on the
GPU machine; --compare then reads both series.

  C1  dam_break_256: 600 steps, Gauss-Seidel 20 at weight 1.9, FIM(10).
  C2  coupled_512: 1000 steps, 24 bodies, jump flooding, RBGS to 1e-5, the
      two-way coupling loop (force read-back, host rigid integration,
      obstacle upload every step).

Every step runs the stages one by one so that the divergence the projection
leaves can be read between EFL_STAGE_SOLVE_VELOCITY and the extrapolation:
the operator of divergence.wgsl:16-42 on the projected velocity over the
cells the residual counts (efl_divergence_norms).  After the step: the fluid
volume (cells with levelset_air < 0, calculate_volume.wgsl:11-75), and every
`--hash-every` steps a CRC of the pressure and level-set fields.

  python -m tests.longrun_report --backend gpu --scene c1 --out c1_gpu.json
  python -m tests.longrun_report --backend oracle --scene c2 --out c2_oracle.json
  python -m tests.longrun_report --compare c1_gpu.json c1_oracle.json
"""
from __future__ import annotations

import argparse
import copy
import json
import os
import sys
import time
import zlib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

import numpy as np  # noqa: E402

from bevy_eulerian_fluid_b200 import _capi as capi  # noqa: E402
from bevy_eulerian_fluid_b200 import scenes  # noqa: E402
from bevy_eulerian_fluid_b200.plugin import pack_obstacles  # noqa: E402
from bevy_eulerian_fluid_b200.rigid import RigidWorld  # noqa: E402

SCENES = {"c1": (lambda: scenes.dam_break(256), 600), "c2": (lambda: scenes.coupled(512), 1000)}


def run(backend: str, scene: str, steps: int, hash_every: int) -> dict:
    if backend == "gpu":
        api = capi.load()
    else:
        from oracle import py_oracle
        api = py_oracle.load()
        py_oracle.set_threads(os.cpu_count() or 1)
    sc = SCENES[scene][0]()
    sim = sc.make(api)
    rigid = None
    if sc.bodies:
        rigid = RigidWorld(copy.deepcopy(list(sc.bodies)), (sc.cfg.nx, sc.cfg.ny), gravity=9.8 * scenes.LENGTH_UNIT,
                           grid_length=1.0 / scenes.LENGTH_UNIT)
    sim.step(sc.dt)  # init sequence
    out = {"backend": backend, "scene": sc.name, "steps": steps, "cells": sc.cells, "volume0": sim.fluid_volume(),
           "iterations": [], "converged": [], "residual": [], "volume": [], "div_l2": [], "div_linf": [],
           "hashes": {}}
    t0 = time.perf_counter()
    for k in range(1, steps + 1):
        st = None
        for stage in range(capi.STAGE_UPDATE_SOLID, capi.STAGE_SOLID_FORCES + 1):
            r = sim.run_stage(stage, sc.dt)
            if stage == capi.STAGE_PROJECTION:
                st = r
            if stage == capi.STAGE_SOLVE_VELOCITY:
                l2, linf = sim.divergence_norms()
        out["iterations"].append(int(st.pressure_iterations))
        out["converged"].append(int(st.converged))
        out["residual"].append(float(st.residual))
        out["volume"].append(int(sim.fluid_volume()))
        out["div_l2"].append(l2)
        out["div_linf"].append(linf)
        if rigid is not None:
            rigid.apply_fluid_forces(sim.solid_forces(), sc.dt)
            rigid.step(sc.dt)
            sim.set_obstacles(pack_obstacles(rigid.bodies))
        if k % hash_every == 0 or k == steps:
            h = 0
            for f in (capi.FIELD_PRESSURE, capi.FIELD_LEVELSET_AIR, capi.FIELD_U, capi.FIELD_V):
                h = zlib.crc32(np.ascontiguousarray(sim.get(f)).tobytes(), h)
            out["hashes"][str(k)] = h
    out["seconds"] = time.perf_counter() - t0
    sim.close()
    return out


def summary(s: dict) -> dict:
    v0 = s["volume0"]
    vol = np.array(s["volume"], dtype=np.float64)
    drift = (vol - v0) / v0
    return {"volume0": v0, "volume_end": int(vol[-1]), "drift_end": float(drift[-1]),
            "drift_max_abs": float(np.max(np.abs(drift))), "div_l2_max": float(np.max(s["div_l2"])),
            "div_l2_mean": float(np.mean(s["div_l2"])), "div_linf_max": float(np.max(s["div_linf"])),
            "iterations_total": int(np.sum(s["iterations"])), "unconverged_steps": int(len(s["converged"]) -
                                                                                       np.sum(s["converged"])),
            "seconds": s["seconds"]}


def compare(a: dict, b: dict) -> str:
    sa, sb = summary(a), summary(b)
    same = {k: a[k] == b[k] for k in ("iterations", "volume", "div_linf", "hashes")}
    l2 = np.array(a["div_l2"]), np.array(b["div_l2"])
    l2_rel = float(np.max(np.abs(l2[0] - l2[1]) / np.maximum(np.abs(l2[1]), 1e-300)))
    rows = [f"| quantity | {a['backend']} | {b['backend']} |", "|---|---|---|"]
    for k in sa:
        fa, fb = sa[k], sb[k]
        fmt = (lambda x: f"{x:.6g}") if isinstance(fa, float) else str
        rows.append(f"| {k} | {fmt(fa)} | {fmt(fb)} |")
    lines = [f"scene {a['scene']} ({a['cells']} cells), {a['steps']} steps", "", *rows, "",
             f"identical series: iterations {same['iterations']}, volume {same['volume']}, "
             f"divergence Linf {same['div_linf']}, field CRCs every {len(a['hashes'])} checkpoints {same['hashes']}; "
             f"divergence L2 max relative difference {l2_rel:.3g} (FP64 sums in different orders)"]
    return "\n".join(lines)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--backend", choices=["gpu", "oracle"])
    ap.add_argument("--scene", choices=sorted(SCENES))
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--hash-every", type=int, default=50)
    ap.add_argument("--out")
    ap.add_argument("--compare", nargs=2)
    args = ap.parse_args()
    if args.compare:
        a, b = (json.load(open(p)) for p in args.compare)
        print(compare(a, b))
        return 0
    steps = args.steps or SCENES[args.scene][1]
    res = run(args.backend, args.scene, steps, args.hash_every)
    with open(args.out, "w") as f:
        json.dump(res, f)
    print(json.dumps(summary(res)))
    return 0


if __name__ == "__main__":
    sys.exit(main())

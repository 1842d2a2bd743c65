"""Benchmark of the per-step fluid hot path (one JSON line on rank 0).

Workload (configs[1] of the reference benchmark list): coupled_512 -- a
512x512 MAC grid, water in the lower 40 %, 24 rigid bodies drawn from seed
0xC2 (6 circles, rectangles, capsules, triangles), jump-flooding level-set
reinitialisation every step, and a pressure solve that iterates red-black
Gauss-Seidel (SOR 1.9) on an FP64 iterate until ||b - A p|| / ||b|| <= 1e-5.

metric: cell-steps/s to 1e-5 relative residual = cells x steps / time.
  value  -- device-resident state, obstacles fixed, CUDA events on the
            simulation's stream around every step, L2 flushed (256 MiB
            write) between steps and excluded from the time.
  e2e    -- the same steps through the plugin API with the two-way
            coupling loop: H2D upload of the 24 packed obstacles, the step,
            D2H read-back of the force bins, host rigid integration.
  roofline -- the sweep kernel alone (efl_pressure_sweeps, 64-bit iterate)
            at the workload's state, 32 algorithmic bytes per cell per
            red-black iteration (p read+write 8, div 4, phi 4, area
            fractions 16), against the measured HBM copy bandwidth.
  microbench -- f32 reference sweeps on the 4096^2 all-fluid pressure
            microbench (N(0,1) divergence, mean removed).
  cpu_baseline -- the CPU oracle (a C++ port of the reference's kernels)
            on the host cores, one full step of the same scene.

Multi-GPU (torchrun): one independent replica per rank (a single fluid
domain does not shard here), weak scaling, max-over-ranks device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

import numpy as np  # noqa: E402

FLUSH_BYTES = 256 << 20
ALGO_BYTES_PER_CELL_ITER = 32  # one red + one black sweep


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-microbench", action="store_true")
    ap.add_argument("--only", choices=["coupled", "microbench"], default=None,
                    help="profiling aid: run one part only and print its numbers")
    return ap.parse_args()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """Per-launch DRAM bytes of the sweep kernel from the committed ncu summary, if any."""
    p = os.path.join(REPO, "profiles", "gs_sweep_f64_coupled_512.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_rb_iteration:"):
            return float(line.split(":")[1])
    return None


class ClockSampler:
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([c.strip() for c in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi samples"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 5 + i and s[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def coupled_cpu_run(size: int, warmup: int, steps: int, budget_s: float):
    """The CPU oracle through the same coupled loop as the GPU arm: init, `warmup`
    untimed steps, then up to `steps` timed steps (stopping early past budget_s)."""
    from bevy_eulerian_fluid_b200 import scenes
    from bevy_eulerian_fluid_b200.plugin import pack_obstacles
    from bevy_eulerian_fluid_b200.rigid import RigidWorld
    from oracle import py_oracle
    api = py_oracle.load()
    py_oracle.set_threads(os.cpu_count() or 1)
    sc = scenes.coupled(size)
    sim = sc.make(api)
    rigid = RigidWorld(list(sc.bodies), (size, size), gravity=9.8 * scenes.LENGTH_UNIT,
                       grid_length=1.0 / scenes.LENGTH_UNIT)

    def coupled_step():
        st = sim.step(sc.dt)
        rigid.apply_fluid_forces(sim.solid_forces(), sc.dt)
        rigid.step(sc.dt)
        sim.set_obstacles(pack_obstacles(rigid.bodies))
        return st

    sim.step(sc.dt)
    for _ in range(warmup):
        coupled_step()
    t0 = time.perf_counter()
    n, iters = 0, []
    while n < steps:
        st = coupled_step()
        n += 1
        iters.append(int(st.pressure_iterations))
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    sim.close()
    return sc.cells * n / el, n, iters, el, py_oracle.get_threads()


def cpu_baseline(size: int, warmup: int, steps: int):
    val, n, iters, el, cores = coupled_cpu_run(size, warmup, steps, 60.0)
    return {"value": val, "unit": "cell-steps/s", "cores": cores, "kind": "port",
            "sample": f"the first {n} timed step(s) of the GPU arm's coupled loop (same scene, same {warmup} warm-up "
                      f"steps) on the CPU oracle, {cores} host threads, {el:.1f} s, pressure iterations/step {iters}"}


def run_reference(args, world, rank):
    """The reference's algorithm on the host cores (the CPU oracle), same workload and metric."""
    if world > 1 and rank != 0:
        return 0
    budget = 150.0
    val, n, iters, el, cores = coupled_cpu_run(args.size, args.warmup, args.steps, budget)
    line = {"impl": "reference", "metric": "cell-steps/s to 1e-5 rel. residual", "value": val, "unit": "cell-steps/s",
            "n_gpus": world, "steps": n, "warmup": args.warmup, "ms_per_step": 1000 * el / n,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": f"coupled_{args.size}", "cells": args.size * args.size, "bodies": 24,
                       "reinit": "jump flooding",
                       "solver": "RBGS (SOR 1.9) on an FP64 iterate to 1e-5 relative residual",
                       "pressure_iterations_per_step": iters},
            "cpu_baseline": {"value": val, "unit": "cell-steps/s", "cores": cores, "kind": "port",
                             "sample": f"{n} coupled steps after {args.warmup} warm-up steps (budget {budget:.0f} s)"},
            "e2e": {"value": val, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, world, rank)

    import torch
    from bevy_eulerian_fluid_b200 import _capi as capi
    from bevy_eulerian_fluid_b200 import scenes
    from bevy_eulerian_fluid_b200.plugin import pack_obstacles
    from bevy_eulerian_fluid_b200.rigid import RigidWorld

    torch.cuda.set_device(local)
    if args.only == "microbench":
        print(json.dumps(microbench(capi.load(), None, torch, measured_peaks()[0])), flush=True)
        return 0
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    api = capi.load()
    sc = scenes.coupled(args.size)
    sc.cfg.device = local
    sim = sc.make(api)
    stream = torch.cuda.ExternalStream(sim.stream(), device=f"cuda:{local}")
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")

    bodies = [b for b in sc.bodies]
    rigid = RigidWorld(bodies, (args.size, args.size), gravity=9.8 * scenes.LENGTH_UNIT,
                       grid_length=1.0 / scenes.LENGTH_UNIT)

    def coupled_step():
        st = sim.step(sc.dt)
        forces = sim.solid_forces()  # D2H: FluidToSolidForce[256]
        rigid.apply_fluid_forces(forces, sc.dt)
        rigid.step(sc.dt)
        sim.set_obstacles(pack_obstacles(rigid.bodies))  # H2D: packed obstacles
        return st

    sim.step(sc.dt)  # init sequence
    for _ in range(args.warmup):
        coupled_step()
    torch.cuda.synchronize()

    # ---- one coupled loop: per step, events around the device step (value) and
    # around the whole coupled iteration (e2e); L2 flushed before each step, outside both.
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    iters = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = api.kernel_launches()
    launches = 0
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            ev[k][0].record(stream)
            l0 = api.kernel_launches()
            st = sim.step(sc.dt)
            launches += api.kernel_launches() - l0
            ev[k][1].record(stream)
            forces = sim.solid_forces()  # D2H: FluidToSolidForce[256]
            rigid.apply_fluid_forces(forces, sc.dt)
            rigid.step(sc.dt)
            sim.set_obstacles(pack_obstacles(rigid.bodies))  # H2D: packed obstacles
            ev[k][2].record(stream)
            iters.append(int(st.pressure_iterations))
            if not st.converged:
                print(f"warning: step {k} not converged (residual {st.residual})", file=sys.stderr)
        torch.cuda.synchronize()
    dev_ms = sum(e[0].elapsed_time(e[1]) for e in ev)
    e2e_ms = sum(e[0].elapsed_time(e[2]) for e in ev)
    if dist:
        t = torch.tensor([dev_ms, e2e_ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms, e2e_ms = float(t[0].item()), float(t[1].item())
        dist.barrier()
    value = world * sc.cells * args.steps / (dev_ms / 1e3)
    e2e_value = world * sc.cells * args.steps / (e2e_ms / 1e3)
    h2d = len(bodies) * 176
    d2h = capi.MAX_SOLIDS * 16

    # ---- roofline of the sweep kernel (FP64 iterate) at this state
    n_sw = 400
    sim.pressure_sweeps(64, 20)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    sim.pressure_sweeps(64, n_sw)
    e1.record(stream)
    torch.cuda.synchronize()
    it_ms = e0.elapsed_time(e1) / n_sw
    peak, peak_kind = measured_peaks()
    achieved = ALGO_BYTES_PER_CELL_ITER * sc.cells / (it_ms / 1e3) / 1e9
    traffic = profile_traffic()
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "kernel": "k_gs_color<double> red+black (one RB iteration)",
                "iteration_us": round(it_ms * 1e3, 3), "peak_kind": peak_kind,
                "note": f"32 B/cell/RB-iteration x {sc.cells} cells; working set is L2-resident at this size"}

    micro = None
    if not args.no_microbench and rank == 0 and args.only is None:
        micro = microbench(api, stream, torch, peak)

    sim.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.size, args.warmup, min(args.steps, 3))

    line = {
        "metric": "cell-steps/s to 1e-5 rel. residual", "value": value, "unit": "cell-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
        "config": {"workload": f"coupled_{args.size}", "cells": sc.cells, "bodies": len(bodies),
                   "reinit": "jump flooding", "solver": "RBGS (SOR 1.9) on an FP64 iterate to 1e-5 relative residual",
                   "pressure_iterations_per_step": iters, "l2": "flushed (256 MiB write) between timed steps",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_ms / args.steps},
        "roofline": roofline, "cpu_baseline": cpu, "clocks": clk.summary(), "gpu_launches": int(launches),
    }
    if micro:
        line["microbench"] = micro
    print(json.dumps(line), flush=True)
    return 0


def microbench(api, stream, torch, peak):
    """f32 reference RB sweeps on the 4096^2 all-fluid pressure microbench."""
    from bevy_eulerian_fluid_b200 import _capi as capi
    from bevy_eulerian_fluid_b200 import scenes
    n = 4096
    cfg = scenes.base_config(n, n)
    sim = capi.Sim(api, cfg)
    phi, b = scenes.microbench_inputs(n)
    sim.run_stage(capi.STAGE_UPDATE_SOLID, scenes.DT)  # walls only
    sim.run_stage(capi.STAGE_AREA_FRACTION, scenes.DT)
    sim.set(capi.FIELD_LEVELSET_AIR, phi)
    sim.set(capi.FIELD_DIVERGENCE, b)
    sim.set(capi.FIELD_PRESSURE, np.zeros((n, n), np.float32))
    s2 = torch.cuda.ExternalStream(sim.stream(), device=torch.cuda.current_device())
    sim.pressure_sweeps(32, 5)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    iters = 50
    torch.cuda.synchronize()
    e0.record(s2)
    sim.pressure_sweeps(32, iters)
    e1.record(s2)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / iters
    gbs = ALGO_BYTES_PER_CELL_ITER * n * n / (ms / 1e3) / 1e9
    sim.close()
    return {"workload": "pressure microbench 4096^2 all-fluid, N(0,1) rhs (seed 0xC3)", "kernel": "k_gs32_tma (TMA-streamed, 2 RB iterations per pass)",
            "ms_per_rb_iteration": round(ms, 4), "achieved_gbs": round(gbs, 1), "frac_of_hbm": round(gbs / peak, 4),
            "bytes_per_cell": ALGO_BYTES_PER_CELL_ITER}


if __name__ == "__main__":
    sys.exit(main())

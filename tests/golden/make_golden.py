"""Generates the committed golden fixtures from the CPU oracle.

The reference publishes no golden vectors and cannot run here, so these
fixtures pin the oracle (and, through tests/test_golden.py, the CUDA
library) to recorded outputs of two small seeded scenes:
  dam_break_64   64^2 water-surface scene, Gauss-Seidel 20, FIM(10): init + 8 steps
  coupled_64     64^2, lower 40 % water, 4 rigid bodies (seed 0xC2), jump
                 flooding, RBGS to 1e-5 (mixed-precision refinement): init + 3 steps
Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from bevy_eulerian_fluid_b200 import _capi as capi  # noqa: E402
from bevy_eulerian_fluid_b200 import scenes  # noqa: E402

FIELDS = {"u": capi.FIELD_U, "v": capi.FIELD_V, "p": capi.FIELD_PRESSURE, "phi": capi.FIELD_LEVELSET_AIR,
          "phi_solid": capi.FIELD_LEVELSET_SOLID, "solid_id": capi.FIELD_SOLID_ID}


def scene(name):
    if name == "dam_break_64":
        return scenes.dam_break(64), 8
    sc = scenes.coupled(64, tolerance=1e-5, n_per_shape=1)
    return sc, 3


def run(api, name):
    sc, steps = scene(name)
    sim = sc.make(api)
    sim.step(sc.dt)
    iters = []
    for _ in range(steps):
        iters.append(sim.step(sc.dt).pressure_iterations)
    out = {k: sim.get(f) for k, f in FIELDS.items()}
    out["bins"] = sim.force_bins()
    out["iterations"] = np.array(iters, np.int64)
    if sc.cfg.reinit.method == capi.REINIT_JUMP_FLOODING:
        out["seeds"] = sim.get(capi.FIELD_JFA_SEEDS)
    sim.close()
    return out


if __name__ == "__main__":
    from oracle import py_oracle
    api = py_oracle.load()
    for name in ("dam_break_64", "coupled_64"):
        out = run(api, name)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, {k: v.shape for k, v in out.items()})

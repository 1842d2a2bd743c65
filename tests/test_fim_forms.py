"""The three forms of the fast iterative method on the GPU -- the temporally blocked tile kernel with a
20-cell halo (the 10 iterations in one launch), the one with a 4-cell halo (2 iterations per launch) and
the per-phase launches -- against the CPU oracle on small grids.  The size rule picks the wide halo on
large grids, and on the others the narrow one for batch members and the per-phase launches for a
simulation alone; EFL_FIM_TILED (read once per process) forces one form, so each case runs in a child
process with the variable set.  Each tiled launch reads one pair of planes and writes the other, so that
no tile sees a neighbour's results of the same launch in its halo: the 1280 x 960 grid has 1200 tiles of
32 x 32, more CTAs of either tiled kernel than fit on the GPU at once."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import numpy as np
from bevy_eulerian_fluid_b200 import _capi as capi, scenes
from oracle import py_oracle

gpu, ora = capi.load(), py_oracle.load()
for nx, ny, steps in ((128, 128, 25), (96, 160, 12), (200, 72, 12), (1280, 960, 4)):
    cfg = scenes.base_config(nx, ny)  # the dam break of examples/water_surface.rs on a ragged grid
    src = scenes.aabb_source((0.0, -0.2 * ny), (0.5 * nx, 0.3 * ny))
    sc = scenes.Scene(f"dam_break_{nx}x{ny}", cfg, oneshot=[src])
    assert sc.cfg.reinit.method == capi.REINIT_FAST_ITERATIVE
    g, o = sc.make(gpu), sc.make(ora)
    for _ in range(steps + 1):
        sg, so = g.step(sc.dt), o.step(sc.dt)
        assert sg.pressure_iterations == so.pressure_iterations
    for f in (capi.FIELD_LEVELSET_AIR, capi.FIELD_U, capi.FIELD_V, capi.FIELD_PRESSURE):
        assert np.array_equal(g.get(f), o.get(f)), (nx, ny, f)
    g.close()
    o.close()
print("ok")
"""


@pytest.mark.parametrize("form", ["2", "1", "0"])
def test_fim_form_bit_exact(form):
    env = dict(os.environ, EFL_FIM_TILED=form)
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-2000:] + r.stderr[-4000:]

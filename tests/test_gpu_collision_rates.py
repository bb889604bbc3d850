"""The reference's homogeneous-gas collision-rate convergence table, run on the engine.

CUDADSMC checks its collision step against the analytic event rate per atom of a homogeneous
gas, 1/2 n sigma <v_r> with <v_r> = sqrt(16 kT / (pi m)): 1e10 atoms in a (2 mm)^3 periodic box at
20 uK give 43.5568 /s, and its table (homogeneousGasCollisions.py:27-35, transcribed in
tests/golden/reference_collision_rates.json) lists the rate it measured with 1e3 .. 1e6 test atoms
on 5^3 and 10^3 cells.  The same sweep runs here on the GPU engine: every (test atoms, cells) entry
must give the analytic rate within four statistical errors and 0.5 %.  The 5^3-cell rows at 5e5 and
1e6 test atoms hold 4000 and 8000 atoms per cell, more than a tile stages: they run through the
dense-cell path (cells split across tiles, collided by dense_collide).
"""
import json
import math
import os

import numpy as np
import pytest

from cudadsmc_b200 import F_COLLIDE, Simulation, preset

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_collision_rates.json")
KB, M_RB = 1.3806503e-23, 1.443160648e-25
DT = 5e-6
MIN_EVENTS = 30000


def homogeneous_run(n_test, cells, seed):
    with open(GOLDEN) as f:
        g = json.load(f)
    setup = g["analytic_setup"]
    run, c = preset(1)  # the periodic box
    run.dt = DT
    c.n_atoms = c.capacity = int(n_test)
    c.cells[0] = c.cells[1] = c.cells[2] = cells
    c.flags = F_COLLIDE
    c.alpha = setup["atoms_real"] / n_test
    c.temperature = setup["temperature_K"]
    half = setup["box_m"] / 2
    for a in range(3):
        c.grid_min[a], c.grid_max[a] = -half, half
    sim = Simulation(run, c)
    sim.init_cloud(seed)
    d0 = sim.diagnostics()
    rate0 = g["analytic_rate"] * DT * n_test  # expected events per step
    steps = max(200, int(math.ceil(MIN_EVENTS / rate0)))
    sim.step(steps)
    d = sim.diagnostics()
    assert d["error"] == 0 and d["n_alive"] == n_test
    events = d["collisions"] - d0["collisions"]
    rate = events / (steps * DT) / n_test
    occ = np.diff(sim.cell_starts())[:-1]
    out = dict(n_test=int(n_test), cells=cells, steps=steps, events=int(events), rate=rate,
               temperature_drift=(d["temperature"] - d0["temperature"]) / d0["temperature"],
               max_atoms_per_cell=int(occ.max()))
    sim.close()
    return out, g


@pytest.mark.parametrize("cells", [5, 10])
def test_collision_rate_convergence_table(cells):
    rows = []
    with open(GOLDEN) as f:
        g = json.load(f)
    ref = g["measured_nc5"] if cells == 5 else g["measured_nc10"]
    for i, n_test in enumerate(g["n_test"]):
        r, g = homogeneous_run(n_test, cells, seed=100 + i)
        r["reference_measured"] = ref[i]
        rows.append(r)
        sigma = r["rate"] / math.sqrt(r["events"])
        assert abs(r["rate"] - g["analytic_rate"]) < 4 * sigma + 5e-3 * g["analytic_rate"], r
        assert abs(r["temperature_drift"]) < 0.01, r
    print(json.dumps({"cells": cells, "analytic_rate": g["analytic_rate"], "rows": rows}))
    if cells == 5:  # 8000 atoms per cell: the dense-cell path ran
        assert rows[-1]["max_atoms_per_cell"] > 4000

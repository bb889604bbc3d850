"""The engine at the benchmark size (1e7 atoms, 128^3 cells): size-independent properties, and
the drift of the FP32 engine's diagnostics against an FP64 run of the same cloud."""
import numpy as np
import pytest

from cudadsmc_b200 import FP32, FP64, Simulation, preset

pytestmark = pytest.mark.gpu


def test_full_size_invariants():
    run, c = preset(2)
    sim = Simulation(run, c)
    sim.init_cloud(1234)
    d0 = sim.diagnostics()
    sim.step(30)
    d = sim.diagnostics()
    assert d["error"] == 0
    # atom accounting and energy accounting (what stays plus what was evaporated)
    assert d["n_alive"] + d["n_evaporated"] == c.n_atoms
    e0 = d0["e_kin"] + d0["e_pot"]
    e1 = d["e_kin"] + d["e_pot"] + d["e_evaporated"]
    assert abs(e1 - e0) / e0 < 1e-4
    assert d["atom_steps"] > 0 and d["collisions"] > 0
    st = sim.get_state()
    pos = st["pos"]
    ids = pos[:, 3].view(np.uint32)
    assert ids.size == d["n_alive"] and np.unique(ids).size == ids.size
    # the order is sorted by cell: recompute every cell in float32 with the engine's formula
    lo = np.array([c.grid_min[a] for a in range(3)], np.float32)
    inv = np.array([np.float32(1.0 / ((c.grid_max[a] - c.grid_min[a]) / c.cells[a])) for a in range(3)], np.float32)
    f = (pos[:, :3] - lo) * inv
    n = np.array(c.cells)
    inside = np.all((f >= 0) & (f < n), axis=1)
    idx = np.floor(np.where(inside[:, None], f, 0)).astype(np.int64)
    cell = np.where(inside, (idx[:, 2] * n[1] + idx[:, 1]) * n[0] + idx[:, 0], n.prod())
    assert np.all(np.diff(cell) >= 0)
    starts = sim.cell_starts()
    assert np.array_equal(np.bincount(cell, minlength=n.prod() + 1), np.diff(starts))


def test_fp32_drift_against_fp64():
    # the same 1e6-atom cloud (FP64 initial state, rounded to FP32) advanced 200 steps in both
    run, c = preset(2)
    c.n_atoms = c.capacity = 1_000_000
    run64 = run.copy()
    run64.precision = FP64
    s64 = Simulation(run64, c)
    s64.init_cloud(77)
    st = s64.get_state()
    s32 = Simulation(run, c)

    def lanes32(a):
        out = a.astype(np.float32)
        out[:, 3] = a[:, 3].view(np.uint64).astype(np.uint32).view(np.float32)  # id / flag bits
        return out

    s32.set_state(lanes32(st["pos"]), lanes32(st["vel"]), st["psi"].astype(np.float32), st["cloud_counts"])
    s64.step(200)
    s32.step(200)
    a, b = s32.diagnostics(), s64.diagnostics()
    rel = {k: abs(a[k] - b[k]) / abs(b[k]) for k in ("n_alive", "temperature", "e_kin", "e_pot", "e_evaporated")}
    print("FP32 vs FP64 relative drift after 200 steps:", rel,
          "collisions", a["collisions"], b["collisions"])
    assert rel["n_alive"] < 1e-3 and rel["temperature"] < 1e-3 and rel["e_kin"] < 2e-3


def test_homogeneous_box_full_config():
    # the homogeneous-gas check as configured (homogeneousGasCollisions.py / collisionComparison.py
    # setting): 1e6 test atoms standing for 1e10 (alpha = 1e4) in a periodic 1 mm^3 box at 10 uK,
    # 100^3 cells (one atom per cell on average), dt = 5 us, 2000 steps, FP32.  The collision rate
    # per atom equals 1/2 n sigma <v_r>, <v_r> = sqrt(16 kT / (pi m)), within four statistical
    # errors and 1 %, and elastic collisions keep the temperature constant.
    run, c = preset(1)
    assert run.precision == FP32 and c.n_atoms == 1_000_000 and c.cells[0] == 100
    sim = Simulation(run, c)
    sim.init_cloud(11)
    d0 = sim.diagnostics()
    steps = 2000
    sim.step(steps)
    d = sim.diagnostics()
    assert d["error"] == 0 and d["n_alive"] == c.n_atoms
    kb, m = 1.3806503e-23, 1.443160648e-25
    volume = np.prod([c.grid_max[a] - c.grid_min[a] for a in range(3)])
    n_real = c.alpha * c.n_atoms / volume
    sigma = 8 * np.pi * (5.3e-9) ** 2
    analytic = 0.5 * n_real * sigma * np.sqrt(16 * kb * c.temperature / (np.pi * m))
    events = d["collisions"] - d0["collisions"]
    rate = events / (steps * run.dt) / c.n_atoms
    assert abs(rate - analytic) < 4 * rate / np.sqrt(events) + 0.01 * analytic, (rate, analytic, events)
    assert abs(d["temperature"] - d0["temperature"]) / d0["temperature"] < 0.01


def test_batched_ensemble_5000_steps_matches_single_runs():
    # the batched workload as specified: 256 clouds (atoms log-uniform in [1e3, 1e5], B' in
    # [1.5, 4] T/m, T in [5, 50] uK, grids 20^3-64^3), autotuned tiles, 5000 steps in one handle;
    # every cloud's diagnostics equal those of the same cloud run alone for 5000 steps
    from cudadsmc_b200.workloads import batched_ensemble
    run, clouds = batched_ensemble()
    batch = Simulation(run, clouds)
    batch.init_cloud(run.seed)
    tile, _ = batch.autotune(3)
    done = batch.diagnostics()["step"]
    batch.step(5000 - done)
    assert batch.diagnostics()["error"] == 0
    for k, c in enumerate(clouds):
        s = Simulation(run, c)
        s.init_cloud(run.seed)
        s.step(5000)
        a, b = s.diagnostics(), batch.diagnostics(k)
        for f in ("step", "n_alive", "sum_v2", "sum_absB", "collisions", "candidates", "n_evaporated"):
            assert a[f] == b[f], (k, f, a[f], b[f])
        s.close()

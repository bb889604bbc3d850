"""The command-line driver (cudadsmc_b200/dsmc_driver, the call structure of CUDADSMC's main())
on the GPU: its printed diagnostics and .npy snapshots against the same run through the Python
binding of the C ABI, bit for bit in FP64."""
import json
import os
import subprocess

import numpy as np
import pytest

from cudadsmc_b200 import FP64, F_MCWF, Simulation, preset

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cudadsmc_b200", "dsmc_driver")


def test_driver_snapshots_match_the_abi_run(tmp_path):
    nc, n, prints, per = 20, 20000, 2, 15
    out = tmp_path / "snap"
    res = subprocess.run([DRIVER, str(nc), str(n), "--prints", str(prints), "--steps-per-print", str(per),
                          "--loops-per-collision", "5", "--mcwf", "--fp64", "--out", str(out), "--seed", "99"],
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    lines = [json.loads(x) for x in res.stdout.splitlines() if x.startswith("{")]
    assert [x["print"] for x in lines] == list(range(prints + 1))
    assert all(x["error"] == 0 for x in lines)

    # the same run through the binding: preset 0 with the driver's argv mapping (main.cu:53-64)
    run, c = preset(0)
    run.precision = FP64
    run.collide_every = 5
    c.cells[0] = c.cells[1] = c.cells[2] = nc
    c.n_atoms = c.capacity = n
    c.alpha = 3e6 / n
    c.flags |= F_MCWF
    sim = Simulation(run, c)
    sim.init_cloud(99)
    for frame in range(prints + 1):
        if frame:
            sim.step(per)
        st = sim.get_state()
        m = st["pos"].shape[0]
        load = lambda name: np.load(out / f"{name}_{frame}.npy")
        assert load("atomNumber")[0] == m == lines[frame]["N"]
        np.testing.assert_array_equal(load("positions"), st["pos"][:, :3])
        np.testing.assert_array_equal(load("velocities"), st["vel"][:, :3])
        np.testing.assert_array_equal(load("psiUp"), st["psi"][:, :2])
        np.testing.assert_array_equal(load("psiDn"), st["psi"][:, 2:])
        ids = load("atomID")
        np.testing.assert_array_equal(ids, st["pos"][:, 3].view(np.uint64).astype(np.int32))
        assert np.unique(ids).size == m
        spin = load("atomIsSpinUp")
        np.testing.assert_array_equal(spin, 1 - (st["vel"][:, 3].view(np.uint64) & 1).astype(np.uint8))
        cell = load("cellID")
        assert np.all(np.diff(cell) >= 0)  # sorted by cell
        counts = load("atomCount")
        np.testing.assert_array_equal(counts, np.diff(sim.cell_starts()))
        assert load("simuatedTime")[0] == pytest.approx(frame * per * run.dt)


def test_driver_snapshot_records_match_the_oracle(tmp_path):
    """The driver's evapPos / evapVel / collisionCount datasets (recorded by the GPU step) and the
    state frames, read back as (N, k, t) arrays, against the oracle's run with its own records:
    the trapped workload's physics (Larmor, Majorana, knife, collisions) scaled to 20000 atoms on
    24^3 cells, FP32, bit for bit."""
    import oracle
    from cudadsmc_b200.snapshots import read_snapshots
    nc, n, prints, per = 24, 20000, 3, 6
    out = tmp_path / "snap"
    res = subprocess.run([DRIVER, str(nc), str(n), "--preset", "2", "--prints", str(prints), "--steps-per-print",
                          str(per), "--out", str(out), "--seed", "7"], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    data = read_snapshots(str(out))
    run, c = preset(2)
    c.cells[0] = c.cells[1] = c.cells[2] = nc
    c.n_atoms = c.capacity = n
    c.alpha = 3e6 / n
    orc = oracle.Oracle(run, c)
    orc.init_cloud(7)
    orc.set_recording(3)
    for frame in range(prints + 1):
        if frame:
            orc.step(per)
        st = orc.get_state()
        m = st["pos"].shape[0]
        assert data["atomNumber"][0, 0, frame] == m
        np.testing.assert_array_equal(data["positions"][:m, :, frame], st["pos"][:, :3].astype(np.float64))
        np.testing.assert_array_equal(data["velocities"][:m, :, frame], st["vel"][:, :3].astype(np.float64))
        ev = orc.evaporated(0)
        np.testing.assert_array_equal(data["evapPos"][:, :, frame], ev["pos"])
        np.testing.assert_array_equal(data["evapVel"][:, :, frame], ev["vel"])
        np.testing.assert_array_equal(data["collisionCount"][:, 0, frame], orc.cell_collisions())
    assert np.count_nonzero(ev["step"] >= 0) > 0  # atoms were lost


@pytest.mark.parametrize("cells", [24, 3])
def test_step_records_match_the_oracle_with_collisions(cells):
    """The records through the Python binding with enough collisions to count (alpha 2e4): lost
    atoms by id and per-cell collision counts after every step, bit for bit with the oracle.  On
    3^3 cells the central cells are dense (more atoms than a tile stages): their counts come from
    dense_collide."""
    import oracle
    from cudadsmc_b200 import F_COLLIDE, F_KNIFE, F_LARMOR, F_MAJORANA, F_NORMALISE
    run, c = preset(2)
    c.n_atoms = c.capacity = 30000
    c.cells[0] = c.cells[1] = c.cells[2] = cells
    c.alpha = 2e4
    c.flags |= F_COLLIDE | F_LARMOR | F_NORMALISE | F_MAJORANA | F_KNIFE
    sim = Simulation(run, c)
    orc = oracle.Oracle(run, c)
    sim.init_cloud(3)
    orc.init_cloud(3)
    sim.set_recording(3)
    orc.set_recording(3)
    total = 0
    for _ in range(4):
        sim.step(2)
        orc.step(2)
        cg, co = sim.cell_collisions(), orc.cell_collisions()
        np.testing.assert_array_equal(cg, co)
        total += int(cg.sum())
        eg, eo = sim.evaporated(0), orc.evaporated(0)
        for k in ("pos", "vel", "step", "fate"):
            np.testing.assert_array_equal(eg[k], eo[k])
    assert total > 0 and np.count_nonzero(eg["step"] >= 0) > 0
    if cells == 3:
        assert np.diff(sim.cell_starts())[:-1].max() > 769

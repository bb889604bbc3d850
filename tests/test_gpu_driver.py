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

"""A bounded device-side wait that runs out ends in an error bit the host reads, not in a hang.

The cell scan's look-back waits for the prefix of the scan block before it; dsmc_check_wait_timeout
runs the scan with its first block withheld, so that prefix never comes. The test checks that the
call returns in seconds with the timeout bit set, and that the context and the simulation stay
usable: the run then continues bit for bit like a twin run that never saw the check."""
import time

import numpy as np
import pytest

from cudadsmc_b200 import Simulation, preset

pytestmark = pytest.mark.gpu

EB_TIMEOUT = 64  # device error bit: a bounded wait gave up


def test_scan_wait_gives_up_and_the_run_continues():
    run, c = preset(2)
    c.n_atoms = c.capacity = 30000
    c.cells[0] = c.cells[1] = c.cells[2] = 24  # 24^3 + 1 cells: four scan blocks
    a, b = Simulation(run, c), Simulation(run, c)
    a.init_cloud(5)
    b.init_cloud(5)
    a.step(3)
    b.step(3)
    t0 = time.perf_counter()
    bits = a.check_wait_timeout()
    assert time.perf_counter() - t0 < 30
    assert bits & EB_TIMEOUT, bits
    a.step(5)
    b.step(5)
    da, db = a.diagnostics(), b.diagnostics()
    assert da["error"] == 0 and db["error"] == 0
    for k in ("step", "n_alive", "sum_v2", "sum_absB", "collisions", "candidates", "n_evaporated"):
        assert da[k] == db[k], (k, da[k], db[k])
    sa, sb = a.get_state(), b.get_state()
    for k in ("pos", "vel", "psi"):
        np.testing.assert_array_equal(sa[k], sb[k])

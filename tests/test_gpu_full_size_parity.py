"""Bit parity with the oracle at the benchmark sizes (GPU).

The measured workloads themselves, not scaled-down copies: the engine and the oracle's OpenMP
path (the same order built in parallel; bit-identical to the serial path by
test_fast_path_is_bit_identical_to_serial) start from the same seed and must agree bit for bit
in every atom's position, velocity and spinor, in the cell starts (the sorted order), in
(sigma v_r)max and in every diagnostic:

  * the full trapped step: 1e7 atoms, 128^3 cells, FP32, collisions + Larmor + Majorana + knife
    (the loop body of CUDADSMC/src/main.cu:416-523), 3 steps;
  * the batched ensemble: 256 clouds (5.66e6 atoms, 20^3..64^3 cells each) with autotuned tiles,
    then 20 steps;
  * the homogeneous periodic box (1e6 atoms, 100^3 cells) and the adjoint workload's cloud
    (1e6 atoms, 0.1 mT bias, 8-knot knife), 5 steps each.
"""
import numpy as np
import pytest

import oracle
from cudadsmc_b200 import Simulation, preset
from cudadsmc_b200.workloads import batched_ensemble

pytestmark = pytest.mark.gpu


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)


def assert_same(sim, orc, nclouds=1):
    assert sim.diagnostics()["error"] == 0
    g, o = sim.get_state(), orc.get_state()
    assert list(g["cloud_counts"]) == list(o["cloud_counts"])
    for key in ("pos", "vel", "psi"):
        assert g[key].shape == o[key].shape, key
        bad = np.nonzero(np.any(bits(g[key]) != bits(o[key]), axis=1))[0]
        assert bad.size == 0, f"{key}: {bad.size} atoms differ, first {bad[:5]}"
    del g, o
    np.testing.assert_array_equal(sim.cell_starts(), orc.cell_starts())
    np.testing.assert_array_equal(bits(sim.sigvrmax()), bits(orc.sigvrmax()))
    keys = ("step", "n_alive", "sum_v2", "sum_absB", "n_evaporated", "n_majorana", "n_knife", "collisions",
            "candidates", "e_kin", "e_pot", "e_evaporated", "temperature", "atom_steps")
    for k in [-1] + list(range(nclouds if nclouds > 1 else 0)):
        dg, do = sim.diagnostics(k), orc.diagnostics(k)
        for key in keys:
            assert dg[key] == do[key], (k, key, dg[key], do[key])


def test_full_trapped_step_at_ten_million_atoms_bit_exact():
    run, c = preset(2)
    assert c.n_atoms == 10_000_000 and tuple(c.cells) == (128, 128, 128)
    sim = Simulation(run, c)
    orc = oracle.Oracle(run, c, fast=True)
    sim.init_cloud(1234)
    orc.init_cloud(1234)
    assert_same(sim, orc)
    sim.step(3)
    orc.step(3)
    assert_same(sim, orc)
    d = sim.diagnostics()
    assert d["collisions"] > 0 and d["n_evaporated"] > 0


def test_batched_ensemble_autotuned_bit_exact():
    run, clouds = batched_ensemble()
    assert len(clouds) == 256
    sim = Simulation(run, clouds)
    orc = oracle.Oracle(run, clouds, fast=True)
    sim.init_cloud(run.seed)
    orc.init_cloud(run.seed)
    sim.autotune(1)  # advances the simulation while it times the tile sizes
    orc.step(sim.diagnostics()["step"])
    sim.step(20)
    orc.step(20)
    assert_same(sim, orc, nclouds=len(clouds))


@pytest.mark.parametrize("which", [1, 4])
def test_box_and_adjoint_workloads_at_full_size_bit_exact(which):
    run, c = preset(which)
    assert c.n_atoms == 1_000_000
    sim = Simulation(run, c)
    orc = oracle.Oracle(run, c, fast=True)
    sim.init_cloud(77)
    orc.init_cloud(77)
    sim.step(5)
    orc.step(5)
    assert_same(sim, orc)

"""The pathwise adjoint on the GPU (dsmc_adjoint_run) against the CPU oracle's smoothed model
and its adjoint on the same recorded run, and against common-random-number central finite
differences of each loss term.  The cloud has Larmor precession and Majorana loss, so the gradient
runs through the spin rotation and the sigmoid Majorana weight as well as Verlet, the knife and the
collisions.  The loss oscillates in B' and B0 through the Larmor phase (about 4 rad per step at
0.1 mT), so a central difference's error falls as h^2 from about 1e-4 relative at h = 1e-4; the
checks on B' and B0 use h = 1e-5 relative and the knots h = 1e-4."""
import numpy as np
import pytest

import oracle
from cudadsmc_b200 import F_MAJORANA, FP32, FP64, Simulation, preset

pytestmark = pytest.mark.gpu


def adjoint_cloud(n=20000, steps=300, majorana=True):
    run, c = preset(4)
    c.n_atoms = c.capacity = n
    c.alpha = 2e4  # enough collisions in a short run to exercise their adjoint
    if majorana:
        c.flags |= F_MAJORANA
    for k in range(9):
        c.knife_step[k] = steps * k / 8.0
        c.knife_eta[k] = 6.0 - 0.25 * k
    return run, c


def theta_of(c):
    return np.array([c.dBdz, c.B0] + [c.knife_eta[k] for k in range(9)])


@pytest.fixture(scope="module")
def recorded():
    run, c = adjoint_cloud()
    sim = Simulation(run, c)
    sim.init_cloud(2468)
    g = sim.adjoint_run(300, checkpoint_every=64, precision=FP64, sigmoid_width_kT=0.2)
    return run, c, sim, g


def test_gpu_smoothed_run_matches_oracle(recorded):
    run, c, sim, g = recorded
    rec = sim.adjoint_export()
    assert g["collisions"] == rec["ij"].shape[0] > 0
    loss_o, parts_o, ge_o, gn_o = oracle.smooth_loss(run, c, theta_of(c), 0.2, rec["x0"], rec["v0"], rec["psi0"],
                                                     rec["steps"], rec["off"], rec["ij"], rec["n"], grad=True,
                                                     fp64=True, majorana_width=0.05)
    # exact sums, same per-atom arithmetic
    assert g["mean_energy_kT"] == parts_o[0] and g["retained_fraction"] == parts_o[1]
    assert g["loss"] == loss_o
    for mine, ref in ((g["dE_dtheta"], ge_o), (g["dN_dtheta"], gn_o)):
        np.testing.assert_allclose(np.array(mine), ref, rtol=1e-9, atol=1e-12 * np.max(np.abs(ref)))
    grad_g = np.array([g["dL_dBp"], g["dL_dB0"]] + g["dL_deta"])
    np.testing.assert_allclose(grad_g, ge_o + gn_o, rtol=1e-9, atol=1e-12 * np.max(np.abs(ge_o + gn_o)))


def test_gradients_repeat_bit_for_bit(recorded):
    # the parameter adjoints are summed per block and reduced in a fixed order, and each step's
    # collisions are applied with every atom's collisions in recorded order: evaluating the
    # gradient again on the same recorded run gives the same bits, in FP64 and in FP32
    run, c, sim, g = recorded
    th = theta_of(c)
    first = sim.adjoint_loss_parts(th, grad=True)
    again = sim.adjoint_loss_parts(th, grad=True)
    for a, b in zip(first, again):
        assert np.array_equal(a, b)
    np.testing.assert_array_equal(first[1], np.array(g["dE_dtheta"]))
    np.testing.assert_array_equal(first[2], np.array(g["dN_dtheta"]))
    s32 = Simulation(run, c)
    s32.init_cloud(2468)
    g32 = s32.adjoint_run(300, checkpoint_every=64, precision=FP32, sigmoid_width_kT=0.2)
    assert g32["collisions"] > 0
    for _ in range(2):  # the smoothed model again in the run's precision, on its record
        parts, ge, gn = s32.adjoint_loss_parts(th, grad=True)
        assert parts[0] == g32["mean_energy_kT"] and parts[1] == g32["retained_fraction"]
        np.testing.assert_array_equal(ge, np.array(g32["dE_dtheta"]))
        np.testing.assert_array_equal(gn, np.array(g32["dN_dtheta"]))
    s32.close()


def test_recorded_collisions_of_dense_cells():
    # a 2^3 grid: the central cells hold thousands of atoms and are collided by dense_collide, which
    # records its collisions (atom ids through the permutation) like the tiles do; the smoothed
    # model on the GPU equals the oracle's on that record
    run, c = adjoint_cloud(n=20000, steps=100)
    c.cells[0] = c.cells[1] = c.cells[2] = 2
    sim = Simulation(run, c)
    sim.init_cloud(97)
    assert np.diff(sim.cell_starts())[:-1].max() > 769
    g = sim.adjoint_run(100, checkpoint_every=32, precision=FP64, sigmoid_width_kT=0.2)
    rec = sim.adjoint_export()
    ij = rec["ij"]
    assert ij.shape[0] == g["collisions"] > 0
    assert np.all(ij >= 0) and np.all(ij < c.n_atoms) and np.all(ij[:, 0] != ij[:, 1])
    loss_o, parts_o, ge_o, gn_o = oracle.smooth_loss(run, c, theta_of(c), 0.2, rec["x0"], rec["v0"], rec["psi0"],
                                                     rec["steps"], rec["off"], rec["ij"], rec["n"], grad=True,
                                                     fp64=True, majorana_width=0.05)
    assert g["mean_energy_kT"] == parts_o[0] and g["retained_fraction"] == parts_o[1]
    np.testing.assert_allclose(np.array(g["dE_dtheta"]), ge_o, rtol=1e-9, atol=1e-12 * np.max(np.abs(ge_o)))


def check_terms_against_differences(sim, th, g, min_checked):
    """Every term's gradient against central differences of that term, 1e-3 relative."""
    grads = (np.array(g["dE_dtheta"]), np.array(g["dN_dtheta"]))
    parts = sim.adjoint_loss_parts(th)
    checked = 0
    for p in range(11):
        h = (1e-5 if p < 2 else 1e-4) * abs(th[p])
        tp, tm = th.copy(), th.copy()
        tp[p] += h
        tm[p] -= h
        fd = (sim.adjoint_loss_parts(tp) - sim.adjoint_loss_parts(tm)) / (2 * h)
        for q in range(2):
            if abs(fd[q] * th[p]) < 1e-6 * max(abs(parts[q]), 1e-3):
                continue  # a knot the run never reached
            assert abs(grads[q][p] - fd[q]) <= 1e-3 * abs(fd[q]), (p, q, grads[q][p], fd[q])
            checked += 1
    assert checked >= min_checked


def test_adjoint_matches_finite_differences(recorded):
    run, c, sim, g = recorded
    check_terms_against_differences(sim, theta_of(c), g, 10)


def test_fp32_adjoint_close_to_fp64():
    run, c = adjoint_cloud(n=20000, steps=200)
    a = Simulation(run, c)
    a.init_cloud(99)
    g64 = a.adjoint_run(200, checkpoint_every=50, precision=FP64)
    b = Simulation(run, c)
    b.init_cloud(99)
    g32 = b.adjoint_run(200, checkpoint_every=50, precision=FP32)
    assert abs(g32["loss"] - g64["loss"]) < 1e-5 * abs(g64["loss"])
    for key in ("dE_dtheta", "dN_dtheta"):
        v64, v32 = np.array(g64[key]), np.array(g32[key])
        big = np.abs(v64) > 1e-3 * np.max(np.abs(v64))
        np.testing.assert_allclose(v32[big], v64[big], rtol=2e-2)


def test_torch_autograd_function():
    import torch
    from cudadsmc_b200.autograd import smoothed_knife_loss, smoothed_loss_terms
    run, c = adjoint_cloud(n=10000, steps=120)
    th = torch.tensor(theta_of(c), dtype=torch.float64, requires_grad=True)
    loss = smoothed_knife_loss(th, run, c, steps=120, checkpoint_every=40, seed=5)
    loss.backward()
    sim = Simulation(run, c)
    sim.init_cloud(5)
    g = sim.adjoint_run(120, checkpoint_every=40)
    assert loss.item() == g["loss"]
    ref = np.array([g["dL_dBp"], g["dL_dB0"]] + g["dL_deta"])
    np.testing.assert_allclose(th.grad.numpy(), ref, rtol=1e-9, atol=1e-14)
    # the terms apart: a weighted sum differentiates through both gradients
    th2 = torch.tensor(theta_of(c), dtype=torch.float64, requires_grad=True)
    terms = smoothed_loss_terms(th2, run, c, steps=120, checkpoint_every=40, seed=5)
    (2.0 * terms[0] - 3.0 * terms[1]).backward()
    assert terms[0].item() == g["mean_energy_kT"] and terms[1].item() == g["retained_fraction"]
    np.testing.assert_allclose(th2.grad.numpy(), 2.0 * np.array(g["dE_dtheta"]) - 3.0 * np.array(g["dN_dtheta"]),
                               rtol=1e-9, atol=1e-14)


def test_adjoint_workload_scale_finite_differences():
    # the adjoint workload as configured (1e6 atoms, 0.1 mT bias, 30 uK, 8-segment ramp over 2000
    # steps, K = 100, sigmoid width 0.2 kT, Larmor precession) with Majorana smoothing on: FP64
    # adjoint of each loss term against common-random-number central differences of that term,
    # 1e-3 relative on every parameter the run is sensitive to
    run, c = preset(4)
    c.flags |= F_MAJORANA
    sim = Simulation(run, c)
    sim.init_cloud(4321)
    g = sim.adjoint_run(2000, checkpoint_every=100, precision=FP64, sigmoid_width_kT=0.2)
    assert g["collisions"] > 0
    th = theta_of(c)
    assert sim.adjoint_loss(th) == g["loss"]
    check_terms_against_differences(sim, th, g, 14)

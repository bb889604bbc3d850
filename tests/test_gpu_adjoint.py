"""The pathwise adjoint on the GPU (dsmc_adjoint_run) against the CPU oracle's smoothed model
and its adjoint on the same recorded run, and against common-random-number central finite
differences of the smoothed loss (h = 1e-4 relative)."""
import numpy as np
import pytest

import oracle
from cudadsmc_b200 import FP32, FP64, Simulation, preset

pytestmark = pytest.mark.gpu


def adjoint_cloud(n=20000, steps=300):
    run, c = preset(4)
    c.n_atoms = c.capacity = n
    c.alpha = 2e4  # enough collisions in a short run to exercise their adjoint
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
    loss_o, grad_o = oracle.smooth_loss(run, c, theta_of(c), 0.2, rec["x0"], rec["v0"], rec["steps"], rec["off"],
                                        rec["ij"], rec["n"], grad=True, fp64=True)
    assert g["loss"] == loss_o  # exact sums, same per-atom arithmetic
    grad_g = np.array([g["dL_dBp"], g["dL_dB0"]] + g["dL_deta"])
    np.testing.assert_allclose(grad_g, grad_o, rtol=1e-9, atol=1e-12 * np.max(np.abs(grad_o)))


def test_adjoint_matches_finite_differences(recorded):
    run, c, sim, g = recorded
    th = theta_of(c)
    grad = np.array([g["dL_dBp"], g["dL_dB0"]] + g["dL_deta"])
    checked = 0
    for p in range(11):
        h = 1e-4 * abs(th[p])
        tp, tm = th.copy(), th.copy()
        tp[p] += h
        tm[p] -= h
        fd = (sim.adjoint_loss(tp) - sim.adjoint_loss(tm)) / (2 * h)
        if abs(fd) < 1e-6 * np.max(np.abs(grad * th)) / max(abs(th[p]), 1e-30):
            continue  # a knot the run never reached
        assert abs(grad[p] - fd) <= 1e-3 * abs(fd), (p, grad[p], fd)
        checked += 1
    assert checked >= 5


def test_fp32_adjoint_close_to_fp64():
    run, c = adjoint_cloud(n=20000, steps=200)
    a = Simulation(run, c)
    a.init_cloud(99)
    g64 = a.adjoint_run(200, checkpoint_every=50, precision=FP64)
    b = Simulation(run, c)
    b.init_cloud(99)
    g32 = b.adjoint_run(200, checkpoint_every=50, precision=FP32)
    assert abs(g32["loss"] - g64["loss"]) < 1e-5 * abs(g64["loss"])
    v64 = np.array([g64["dL_dBp"], g64["dL_dB0"]] + g64["dL_deta"])
    v32 = np.array([g32["dL_dBp"], g32["dL_dB0"]] + g32["dL_deta"])
    big = np.abs(v64) > 1e-3 * np.max(np.abs(v64))
    np.testing.assert_allclose(v32[big], v64[big], rtol=2e-2)


def test_torch_autograd_function():
    import torch
    from cudadsmc_b200.autograd import smoothed_knife_loss
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


def test_adjoint_workload_scale_finite_differences():
    # the adjoint workload as configured (1e6 atoms, 0.1 mT bias, 30 uK, 8-segment ramp over 2000
    # steps, K = 100, sigmoid width 0.2 kT): FP64 adjoint against common-random-number central
    # differences (h = 1e-4 relative) of the smoothed loss, 1e-3 relative on every parameter the
    # run is sensitive to
    run, c = preset(4)
    sim = Simulation(run, c)
    sim.init_cloud(4321)
    g = sim.adjoint_run(2000, checkpoint_every=100, precision=FP64, sigmoid_width_kT=0.2)
    assert g["collisions"] > 0
    th = theta_of(c)
    assert sim.adjoint_loss(th) == g["loss"]
    grad = np.array([g["dL_dBp"], g["dL_dB0"]] + g["dL_deta"])
    scale = np.max(np.abs(grad * th))
    checked = 0
    for p in range(11):
        h = 1e-4 * abs(th[p])
        tp, tm = th.copy(), th.copy()
        tp[p] += h
        tm[p] -= h
        fd = (sim.adjoint_loss(tp) - sim.adjoint_loss(tm)) / (2 * h)
        if abs(fd * th[p]) < 1e-6 * scale:
            continue  # a knot whose weight no atom feels
        assert abs(grad[p] - fd) <= 1e-3 * abs(fd), (p, grad[p], fd)
        checked += 1
    assert checked >= 8

"""The oracle's smoothed model with spin (Larmor precession, sigmoid Majorana weight) and its
hand-written adjoint against central finite differences, on CPU.

A short synthetic run of a few hundred atoms in the biased quadrupole (the field's zero sits inside
the cloud, so the Majorana weights move), with recorded collisions between random pairs: the
adjoint's gradients of the two loss terms -- the final mean energy per retained atom (L_E) and the
retained fraction (L_N) -- must match central differences of each term (h = 1e-5 relative; the
Larmor phase makes the loss oscillate in B', and the differences' error falls as h^2) to 1e-5
relative, on B', the bias and every knife knot the run reaches.  The same gradients with Larmor
precession switched off must differ (the spin path carries gradient).
"""
import numpy as np

import oracle
from cudadsmc_b200 import F_LARMOR, F_MAJORANA


def synthetic_run(n=300, steps=60, seed=3, flags=F_LARMOR | F_MAJORANA):
    run, c = oracle.preset(4)
    c.n_atoms = c.capacity = n
    c.flags |= flags
    c.B0 = 2e-5  # the field's zero at z = B0/B' = 8 um, inside the cloud
    for k in range(9):
        c.knife_step[k] = steps * k / 8.0
        c.knife_eta[k] = 5.0 - 0.2 * k
    rng = np.random.default_rng(seed)
    kT = 1.380649e-23 * c.temperature
    r0 = kT / c.moment / c.dBdz  # thermal length of the linear trap
    x = rng.normal(0.0, r0, size=(n, 3)) * np.array([2.0, 2.0, 1.0])
    v = rng.normal(0.0, np.sqrt(kT / c.mass), size=(n, 3))
    # spinors near the local field direction, tilted so that some atoms are close to flipping
    B = np.stack([0.5 * c.dBdz * x[:, 0], 0.5 * c.dBdz * x[:, 1], c.B0 - c.dBdz * x[:, 2]], axis=1)
    b = B / np.linalg.norm(B, axis=1, keepdims=True)
    th = np.arccos(np.clip(b[:, 2], -1, 1)) + rng.normal(0.0, 0.6, n)
    ph = np.arctan2(b[:, 1], b[:, 0])
    psi = np.stack([np.cos(th / 2), np.zeros(n), np.sin(th / 2) * np.cos(ph), np.sin(th / 2) * np.sin(ph)], axis=1)
    # two recorded collisions per step between random distinct atoms, isotropic directions
    off = np.arange(steps + 1, dtype=np.int32) * 2
    ij = np.stack([rng.choice(n, 2, replace=False) for _ in range(2 * steps)]).astype(np.int32)
    nv = rng.normal(size=(2 * steps, 3))
    nv /= np.linalg.norm(nv, axis=1, keepdims=True)
    theta = np.array([c.dBdz, c.B0] + [c.knife_eta[k] for k in range(9)])
    return run, c, theta, dict(x=x, v=v, psi=psi, steps=steps, off=off, ij=ij, nv=nv)


def loss_parts(run, c, theta, rec, grad=False):
    return oracle.smooth_loss(run, c, theta, 0.2, rec["x"], rec["v"], rec["psi"], rec["steps"], rec["off"], rec["ij"],
                              rec["nv"], grad=grad, fp64=True, majorana_width=0.1)


def test_spin_adjoint_matches_finite_differences_per_term():
    run, c, theta, rec = synthetic_run()
    loss, parts, ge, gn = loss_parts(run, c, theta, rec, grad=True)
    assert abs(loss - parts.sum()) < 1e-15 * abs(loss)
    assert 0.2 < parts[1] < 0.999  # the weights moved
    checked = 0
    for p in range(11):
        h = 1e-5 * abs(theta[p])
        tp, tm = theta.copy(), theta.copy()
        tp[p] += h
        tm[p] -= h
        fd = (loss_parts(run, c, tp, rec)[1] - loss_parts(run, c, tm, rec)[1]) / (2 * h)
        for q, g in ((0, ge), (1, gn)):
            if abs(fd[q] * theta[p]) < 1e-9 * max(abs(parts[q]), 1.0):
                continue  # a knot the run never reaches
            assert abs(g[p] - fd[q]) <= 1e-5 * abs(fd[q]), (p, q, g[p], fd[q])
            checked += 1
    assert checked >= 12


def test_spin_path_carries_gradient():
    run, c, theta, rec = synthetic_run()
    _, _, ge, gn = loss_parts(run, c, theta, rec, grad=True)
    run2, c2, theta2, rec2 = synthetic_run(flags=F_MAJORANA)
    c2.flags &= ~F_LARMOR
    _, _, ge2, gn2 = loss_parts(run2, c2, theta2, rec2, grad=True)
    assert abs(gn[0] - gn2[0]) > 1e-3 * abs(gn[0])

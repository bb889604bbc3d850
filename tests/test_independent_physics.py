"""The oracle's per-atom step and per-cell collisions against a numpy FP64 restatement written in
this file from the physics alone (CPU only).

The engine and the oracle share their per-atom and per-cell arithmetic (dsmc_physics.h), so
GPU-vs-oracle bit equality proves the GPU's orchestration, not the physics.  This file pins that
shared arithmetic to code that includes none of it: complex 2x2 matrices for the spin, analytic
gradients for the field, and its own Philox4x32-10 (checked against the published known-answer
vectors of Salmon et al., SC'11) for the random words of the no-time-counter collisions.

  one step of an atom in the linear quadrupole trap (the benchmark's trap):
    Larmor rotation psi <- exp(-i theta s.B^) psi, theta = mu |B| dt / hbar, renormalised
                                           (CUDADSMC/src/wavefunction.cu:39-73, 279-299)
    velocity Verlet with a = -(mu/m) grad|B| (+ for anti-trapped atoms)
                                           (CUDADSMC/src/moveAtoms.cu:51-65, 93-116)
    Majorana test <psi| s.B^ |psi> < 0     (CUDADSMC/src/evaporation.cu:86-95)
    energy knife  v^2 + (2 mu/m)|B| > 2 eta kB T / m
    cell index    floor((x - xmin)/dx), z*nx*ny + y*nx + x, overflow cell  (collisions.cu:194-219)
  one cell of Bird's no-time-counter scheme:
    Ncand = ceil(Mc alpha dt_c (sigma v_r)max / V), Mc = n(n-1)/2, a uniform distinct pair per
    candidate, accepted with sigma v_r alpha dt_c Mc / (V Ncand), isotropic rescatter about the
    centre of mass                         (collisions.cu:319-322, 422-437, 529-546)
"""
import numpy as np
import pytest

import oracle
from cudadsmc_b200._abi import F_COLLIDE, F_KNIFE, F_LARMOR, F_MAJORANA, F_NORMALISE, FP64

MASK32 = np.uint64(0xFFFFFFFF)


# ------------------------------------------------------------------------------ Philox4x32-10
def philox(ctr, key):
    """Philox4x32-10 of counters ctr (m, 4) under key (2,), as uint64 arrays holding 32-bit words."""
    c = [np.asarray(ctr[:, i], np.uint64) & MASK32 for i in range(4)]
    k0, k1 = np.uint64(key[0]) & MASK32, np.uint64(key[1]) & MASK32
    for _ in range(10):
        p0 = np.uint64(0xD2511F53) * c[0]
        p1 = np.uint64(0xCD9E8D57) * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK32
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK32
        c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
        k0 = (k0 + np.uint64(0x9E3779B9)) & MASK32
        k1 = (k1 + np.uint64(0xBB67AE85)) & MASK32
    return np.stack(c, axis=1)


def test_philox_known_answers():
    # the known-answer vectors published with the Random123 library for philox4x32 with 10 rounds
    kat = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
           ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
           ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
            (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for ctr, key, want in kat:
        got = philox(np.array([ctr], np.uint64), key)[0]
        assert [int(x) for x in got] == list(want)
        assert [int(x) for x in oracle.philox4x32_10(ctr, key)] == list(want)


def u01d(a, b):
    """Uniform in (0, 1) from 53 bits of two words: ((a << 21) ^ (b >> 11) + 1/2) 2^-53."""
    m = (np.uint64(a) << np.uint64(21)) ^ (np.uint64(b) >> np.uint64(11))
    return (float(m) + 0.5) * 2.0 ** -53


# ------------------------------------------------------------------------------ one quadrupole step
HBAR = 1.05457148e-34
KB = 1.3806503e-23


def quad_field(c, x):
    """B, |B|, B^ and grad|B| of B = (B'x/2, B'y/2, B0 - B'z) at points x (m, 3)."""
    h = 0.5 * c.dBdz
    B = np.stack([h * x[:, 0], h * x[:, 1], c.B0 - c.dBdz * x[:, 2]], axis=1)
    absB = np.linalg.norm(B, axis=1)
    bhat = B / absB[:, None]
    grad = np.stack([h * h * x[:, 0], h * h * x[:, 1], -c.dBdz * B[:, 2]], axis=1) / absB[:, None]
    return absB, bhat, grad


def sigma_dot(bhat):
    """s.B^ as (m, 2, 2) complex matrices."""
    bx, by, bz = bhat[:, 0], bhat[:, 1], bhat[:, 2]
    return np.stack([np.stack([bz + 0j, bx - 1j * by], -1), np.stack([bx + 1j * by, -bz + 0j], -1)], -2)


def numpy_step(run, c, pos, vel, psi, anti, cut_v2):
    """One FP64 timestep of each atom; returns (pos, vel, psi, fate, cell)."""
    dt, mu, m = run.dt, c.moment, c.mass
    absB, bhat, grad = quad_field(c, pos)
    spinor = np.stack([psi[:, 0] + 1j * psi[:, 1], psi[:, 2] + 1j * psi[:, 3]], axis=1)
    theta = mu * absB * dt / HBAR
    U = np.cos(theta)[:, None, None] * np.eye(2)[None] - 1j * np.sin(theta)[:, None, None] * sigma_dot(bhat)
    spinor = np.einsum("nij,nj->ni", U, spinor)
    spinor /= np.linalg.norm(spinor, axis=1)[:, None]
    sgn = np.where(anti, 1.0, -1.0)[:, None]
    v_half = vel + 0.5 * dt * sgn * (mu / m) * grad
    x1 = pos + dt * v_half
    absB1, bhat1, grad1 = quad_field(c, x1)
    v1 = v_half + 0.5 * dt * sgn * (mu / m) * grad1
    proj = np.einsum("ni,nij,nj->n", spinor.conj(), sigma_dot(bhat1), spinor).real
    v2 = np.sum(v1 * v1, axis=1)
    energy = v2 + (2.0 * mu / m) * absB1
    fate = np.where(proj < 0, 1, np.where(energy > cut_v2, 2, 0))
    lo = np.array(c.grid_min[:3])
    n = np.array(c.cells[:3])
    d = (np.array(c.grid_max[:3]) - lo) / n
    f = (x1 - lo) / d
    inside = np.all((f >= 0) & (f < n), axis=1)
    idx = np.floor(np.where(inside[:, None], f, 0)).astype(np.int64)
    cell = np.where(inside, (idx[:, 2] * n[1] + idx[:, 1]) * n[0] + idx[:, 0], n.prod())
    near_face = np.any(np.abs(f - np.rint(f)) < 1e-9, axis=1)
    out_psi = np.stack([spinor[:, 0].real, spinor[:, 0].imag, spinor[:, 1].real, spinor[:, 1].imag], axis=1)
    return x1, v1, out_psi, fate, cell, near_face


def trapped_cloud(n, seed):
    run, c = oracle.preset(2)
    run.precision = FP64
    c.flags = F_LARMOR | F_NORMALISE | F_MAJORANA | F_KNIFE
    rng = np.random.default_rng(seed)
    rz = KB * c.temperature / (c.moment * c.dBdz)
    pos = rng.normal(0.0, 1.0, (n, 3)) * np.array([2 * rz, 2 * rz, rz])
    pos[-20:] *= 4.0  # a few atoms beyond the grid's +-5 thermal lengths: the overflow cell
    vel = rng.normal(0.0, np.sqrt(KB * c.temperature / c.mass), (n, 3))
    # spinors near the local field direction, some far from it (Majorana candidates)
    _, bhat, _ = quad_field(c, pos)
    up = np.sqrt(0.5 * (1 + bhat[:, 2]))
    aligned = np.stack([up + 0j, (bhat[:, 0] + 1j * bhat[:, 1]) / (2 * up)], axis=1)
    noise = rng.normal(size=(n, 2)) + 1j * rng.normal(size=(n, 2))
    w = rng.uniform(0.0, 1.5, n)[:, None]
    s = aligned + w * noise
    s /= np.linalg.norm(s, axis=1)[:, None]
    psi = np.stack([s[:, 0].real, s[:, 0].imag, s[:, 1].real, s[:, 1].imag], axis=1)
    anti = rng.uniform(size=n) < 0.1
    return run, c, pos, vel, psi, anti


def test_quadrupole_step_matches_numpy_restatement():
    n = 1000
    run, c, pos, vel, psi, anti = trapped_cloud(n, 11)
    cut_v2 = 2.0 * 5.0 * KB * c.temperature / c.mass  # eta = 5
    p4 = np.zeros((n, 4)); p4[:, :3] = pos
    v4 = np.zeros((n, 4)); v4[:, :3] = vel
    v4[:, 3] = anti.astype(np.uint64).view(np.float64)  # flag bit 0 in the fourth lane's integer bits
    op, ov, opsi, ofate, ocell = oracle.step_atoms(run, c, p4, v4, psi, cut_v2)
    x1, v1, s1, fate, cell, near = numpy_step(run, c, pos, vel, psi, anti, cut_v2)
    scale_x = np.max(np.abs(x1))
    scale_v = np.max(np.abs(v1))
    assert np.max(np.abs(op[:, :3] - x1)) <= 1e-12 * scale_x
    assert np.max(np.abs(ov[:, :3] - v1)) <= 1e-12 * scale_v
    assert np.max(np.abs(opsi - s1)) <= 1e-12
    assert np.array_equal(ofate, fate)
    assert np.all((ocell == cell) | near)
    # the sample exercises every branch: Majorana, knife, survivors, anti-trapped atoms, overflow cell
    assert (fate == 1).sum() > 10 and (fate == 2).sum() > 10 and (fate == 0).sum() > 100
    assert anti.sum() > 10 and (cell == np.prod(c.cells[:3])).sum() >= 1


# ------------------------------------------------------------------------------ one NTC cell
def numpy_collide(run, c, vel, sigvrmax, local_cell, step):
    """Bird's no-time-counter collisions of one cell with this file's Philox; returns
    (vel, sigvrmax, candidates, pairs, directions)."""
    vel = vel.copy()
    n = vel.shape[0]
    d = (np.array(c.grid_max[:3]) - np.array(c.grid_min[:3])) / np.array(c.cells[:3])
    cand_pref = c.alpha * run.dt * run.collide_every / np.prod(d)
    Mc = 0.5 * n * (n - 1)
    ncand = int(np.ceil(Mc * cand_pref * sigvrmax))
    pacc = cand_pref * Mc / ncand
    key = (run.seed & 0xFFFFFFFF, run.seed >> 32)
    purpose = (3 << 24) | (c.stream_id & 0xFFFFFF)
    pairs, dirs = [], []
    for k in range(ncand):
        w = philox(np.array([[local_cell, step, purpose, 2 * k]], np.uint64), key)[0]
        i = (int(w[0]) * n) >> 32
        j = (int(w[1]) * (n - 1)) >> 32
        j += 1 if j >= i else 0
        vr = np.linalg.norm(vel[i] - vel[j])
        sigvrmax = max(sigvrmax, c.sigma * vr)
        if u01d(w[2], w[3]) < c.sigma * vr * pacc:
            w2 = philox(np.array([[local_cell, step, purpose, 2 * k + 1]], np.uint64), key)[0]
            ct = 2.0 * u01d(w2[0], w2[1]) - 1.0
            phi = 2.0 * np.pi * u01d(w2[2], w2[3])
            st = np.sqrt(max(1.0 - ct * ct, 0.0))
            nhat = np.array([st * np.cos(phi), st * np.sin(phi), ct])
            cm = 0.5 * (vel[i] + vel[j])
            vel[i], vel[j] = cm + 0.5 * vr * nhat, cm - 0.5 * vr * nhat
            pairs.append((i, j))
            dirs.append(nhat)
    return vel, sigvrmax, ncand, np.array(pairs, np.int64).reshape(-1, 2), np.array(dirs).reshape(-1, 3)


@pytest.mark.parametrize("alpha", [1.0, 2e5])
def test_ntc_cells_match_numpy_restatement(alpha):
    run, c = oracle.preset(2)
    run.precision = FP64
    run.seed = 0x1234_5678_9ABC
    c.flags = F_COLLIDE
    c.alpha = alpha  # 2e5: many candidates per cell and frequent acceptance
    c.stream_id = 5
    rng = np.random.default_rng(3)
    sv0 = c.sigma * np.sqrt(16 * KB * c.temperature / (np.pi * c.mass))
    accepted = 0
    for cell in range(50):
        n = int(rng.integers(2, 41))
        vel = rng.normal(0.0, np.sqrt(KB * c.temperature / c.mass), (n, 3))
        local, step = int(rng.integers(0, 128 ** 3)), int(rng.integers(0, 10 ** 5))
        ov, osv, ocand, oij, onv = oracle.collide_cell(run, c, vel, sv0, local, step)
        nv, nsv, ncand, nij, nnv = numpy_collide(run, c, vel, sv0, local, step)
        assert ocand == ncand
        assert np.array_equal(oij, nij), cell
        assert np.max(np.abs(onv - nnv), initial=0.0) <= 1e-12
        assert np.max(np.abs(ov - nv)) <= 1e-12 * np.max(np.abs(nv))
        assert abs(osv - nsv) <= 1e-12 * nsv
        accepted += len(nij)
    if alpha > 1.0:
        assert accepted > 100

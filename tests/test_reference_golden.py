"""The oracle's per-atom physics against the reference's own kernels (CPU only).

tests/golden/reference_ip_motion.npz was produced by tests/golden/make_reference_vectors.py,
which compiles CUDADSMC/src/moveAtoms.cu and CUDADSMC/src/wavefunction.cu for the host from
the reference tree (oracle/ref_host/Makefile) and iterates evolveWavefunction + moveAtoms
(CUDADSMC/src/main.cu:465-476) in the reference's Ioffe-Pritchard trap.  The oracle runs the
same FP64 step (Larmor rotation about B^(x), then velocity Verlet) from the same inputs; the
two differ only in the order of floating-point operations, so agreement is to rounding.
"""
import os

import numpy as np
import pytest

import oracle
from cudadsmc_b200._abi import FP64, F_LARMOR, TRAP_IOFFE_PRITCHARD

GOLD = os.path.join(os.path.dirname(__file__), "golden", "reference_ip_motion.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def ip_cloud(g):
    run, c = oracle.preset(0)
    run.precision = FP64
    run.dt = float(g["dt"])
    c.trap = TRAP_IOFFE_PRITCHARD
    c.B0, c.dBdz, c.d2Bdz2 = float(g["B0"]), float(g["dBdz"]), float(g["d2Bdz2"])
    c.moment = float(g["moment"])
    c.mass = float(g["mass"])
    c.flags = F_LARMOR  # no renormalisation: the reference normalises once per collision step
    for a in range(3):
        c.grid_min[a], c.grid_max[a] = -1e-3, 1e-3
    return run, c


def pack(g, n):
    pos = np.zeros((n, 4)); vel = np.zeros((n, 4)); psi = np.zeros((n, 4))
    pos[:, :3] = g["pos0"]; vel[:, :3] = g["vel0"]
    psi[:, :2] = g["up0"]; psi[:, 2:] = g["dn0"]
    return pos, vel, psi


@pytest.mark.parametrize("steps,rtol", [(1, 1e-13), (200, 1e-10)])
def test_motion_and_larmor_match_reference_kernels(gold, steps, rtol):
    run, c = ip_cloud(gold)
    n = gold["pos0"].shape[0]
    pos, vel, psi = pack(gold, n)
    p, v, s, fate = oracle.advance_atoms(run, c, pos, vel, psi, steps)
    scale_x = np.max(np.abs(gold[f"pos_{steps}"]))
    scale_v = np.max(np.abs(gold[f"vel_{steps}"]))
    assert np.max(np.abs(p[:, :3] - gold[f"pos_{steps}"])) <= rtol * scale_x
    assert np.max(np.abs(v[:, :3] - gold[f"vel_{steps}"])) <= rtol * scale_v
    assert np.max(np.abs(s[:, :2] - gold[f"up_{steps}"])) <= 50 * rtol
    assert np.max(np.abs(s[:, 2:] - gold[f"dn_{steps}"])) <= 50 * rtol


def test_projection_matches_reference_local_populations(gold):
    # getLocalPopulations (wavefunction.cu:156-173): P_up - P_dn = <s.B^>, the Majorana test quantity
    run, c = ip_cloud(gold)
    n = gold["pos0"].shape[0]
    pos, vel, psi = pack(gold, n)
    p, v, s, fate = oracle.advance_atoms(run, c, pos, vel, psi, 200)
    f = oracle.field(run, c, p[:, :3])
    u = s[:, 0] + 1j * s[:, 1]
    d = s[:, 2] + 1j * s[:, 3]
    proj = 2 * f[:, 0] * (np.conj(u) * d).real + 2 * f[:, 1] * (np.conj(u) * d).imag + f[:, 2] * (abs(u) ** 2 - abs(d) ** 2)
    pops = gold["pops_end"]
    assert np.max(np.abs(proj - (pops[:, 0] - pops[:, 1]))) < 1e-9

"""Generates tests/golden/reference_ip_motion.npz from the reference's own kernels.

Runs in a container where the reference tree is present: builds CUDADSMC/src/moveAtoms.cu
and CUDADSMC/src/wavefunction.cu for the host (oracle/ref_host/Makefile -> oracle/_ref/) and
records, for seeded atoms in the reference's Ioffe-Pritchard trap (B0 = 0.01 T,
B' = 20 T/m, B'' = 4e4 T/m^2, include/deviceSystemParameters.cuh:25-27; moment
g_s muB / 2 with g_s = 0.5, moveAtoms.cu:102; dt = 1e-7 s, wavefunction.cu:45), the state
after 1 and after 200 iterations of evolveWavefunction + moveAtoms (main.cu:465-476).

    python tests/golden/make_reference_vectors.py /root/reference/CUDADSMC

The argument is the CUDADSMC project tree (read only; nothing is written there).
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")

MUB, M_RB, KB = 9.27400915e-24, 1.443160648e-25, 1.3806503e-23


def build(ref_tree):
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle", "ref_host"), "CXX=/usr/bin/g++", f"REF={ref_tree}"],
                   check=True, capture_output=True)


def main(ref_tree, n=256, steps=(1, 200), seed=2024):
    build(ref_tree)
    mv = C.CDLL(os.path.join(REF_DIR, "libref_move.so"))
    wv = C.CDLL(os.path.join(REF_DIR, "libref_wave.so"))
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
    rng = np.random.default_rng(seed)
    pos0 = rng.uniform(-2e-4, 2e-4, (n, 3))
    vel0 = rng.normal(0, np.sqrt(KB * 20e-6 / M_RB), (n, 3))
    up = rng.normal(size=(n, 2))
    dn = rng.normal(size=(n, 2))
    norm = np.sqrt(np.sum(up ** 2, 1) + np.sum(dn ** 2, 1))
    up0, dn0 = up / norm[:, None], dn / norm[:, None]
    out = {"pos0": pos0, "vel0": vel0, "up0": up0, "dn0": dn0, "dt": 1e-7, "moment": 0.25 * MUB,
           "B0": 0.01, "dBdz": 20.0, "d2Bdz2": 4e4, "mass": M_RB, "steps": np.array(steps)}
    mv.ref_set_dt(C.c_double(1e-7))
    pos, vel = pos0.copy(), vel0.copy()
    u, d = up0.copy(), dn0.copy()
    acc = np.zeros_like(pos)
    mv.ref_update_acc(dp(pos), dp(acc), n)
    ids = np.arange(n, dtype=np.int32)
    spin = np.ones(n, np.uint8)
    done = 0
    for s in steps:
        for _ in range(s - done):
            wv.ref_evolve_wavefunction(dp(pos), dp(u), dp(d), ip(ids), n)
            mv.ref_move_atoms(dp(pos), dp(vel), dp(acc), spin.ctypes.data_as(C.c_void_p), ip(ids), n)
        done = s
        out[f"pos_{s}"], out[f"vel_{s}"], out[f"up_{s}"], out[f"dn_{s}"] = pos.copy(), vel.copy(), u.copy(), d.copy()
    pops = np.zeros((n, 2))
    wv.ref_local_populations(dp(pos), dp(u), dp(d), dp(pops), ip(ids), n)
    out["pops_end"] = pops
    np.savez_compressed(os.path.join(HERE, "reference_ip_motion.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])

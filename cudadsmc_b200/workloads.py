"""Named workloads beyond the single-cloud presets of dsmc_preset.

``batched_ensemble`` -- the batched configuration: independent clouds with atom counts
log-uniform in [1e3, 1e5], field gradients B' uniform in [1.5, 4] T/m, temperatures uniform in
[5, 50] uK and cubic cell meshes of 20^3..64^3 spanning +-5 thermal radii, each with its own
Philox stream (stream_id = index) so that a cloud gives the same result inside the batch and
run alone.
"""
from __future__ import annotations

import numpy as np

from . import _abi
from .engine import preset

KB = 1.3806503e-23


def quadrupole_grid(c: _abi.CloudParams, radii: float, cells: int) -> None:
    rz = KB * c.temperature / (c.moment * c.dBdz)
    rx = 2.0 * rz
    z0 = c.B0 / c.dBdz
    for a, r, centre in ((0, rx, 0.0), (1, rx, 0.0), (2, rz, z0)):
        c.grid_min[a] = centre - radii * r
        c.grid_max[a] = centre + radii * r
        c.cells[a] = cells


def batched_ensemble(n_clouds: int = 256, seed: int = 2024, atoms_lo: float = 1e3, atoms_hi: float = 1e5):
    """(run, [cloud params]) of the batched workload."""
    rng = np.random.default_rng(seed)
    run, base = preset(2)
    clouds = []
    for k in range(n_clouds):
        c = base.copy()
        c.n_atoms = int(round(np.exp(rng.uniform(np.log(atoms_lo), np.log(atoms_hi)))))
        c.capacity = c.n_atoms
        c.dBdz = float(rng.uniform(1.5, 4.0))
        c.temperature = float(rng.uniform(5e-6, 50e-6))
        c.alpha = 3e6 / c.n_atoms  # real atoms per test atom, as CUDADSMC/src/main.cu:53
        c.flags = _abi.F_COLLIDE | _abi.F_LARMOR | _abi.F_NORMALISE | _abi.F_MAJORANA
        c.knife_nknots = 0
        quadrupole_grid(c, 5.0, int(rng.integers(20, 65)))
        c.stream_id = k
        clouds.append(c)
    return run, clouds

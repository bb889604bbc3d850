"""Snapshots in the layout of CUDADSMC's output file, as .npy files, and their reader.

The reference writes /atomData/<name> datasets into one HDF5 file, each extendible along its last
axis: every print appends a frame of shape (N, k) to an (N, k, t) dataset (CUDADSMC/src/main.cu:
209-383 create and fill them, CUDADSMC/src/hdf5Helpers.cu:13-163 extend them).  HDF5 is not
available here, so a frame of dataset <name> is the file <dir>/<name>_<frame>.npy (the C++ driver
writes the same files), and read_snapshots() stacks the frames back into (N, k, t) arrays.

Datasets (reference names, including its spelling of simuatedTime):
  per atom of the frame: positions, velocities (N, 3); psiUp, psiDn (N, 2) as (Re, Im); atomID,
    atomIsSpinUp, cellID (N, 1)
  per atom id: evapPos, evapVel (N0, 3) -- where each atom was lost and its velocity then, zeros
    for atoms not lost (evaporation.cu:86-100 keeps them by atom)
  per cell of the cloud (its grid cells then the overflow cell): atomCount, collisionCount (Nc+1, 1)
  per frame: atomNumber, simuatedTime (1, 1)
Frames whose atom count fell (atoms were lost) are padded at the end of the atom axis: NaN for
floating-point datasets, -1 for atomID and cellID, 0 for atomIsSpinUp.
save_npz() packs the stacked (N, k, t) datasets of a directory into one .npz archive under the
same names (the file the reference's single HDF5 output stands for), and load_npz() reads it back.
"""
from __future__ import annotations

import glob
import os
import re

import numpy as np

from ._abi import REC_CELL_COLLISIONS, REC_EVAPORATED

PER_ATOM = ("positions", "velocities", "psiUp", "psiDn", "atomID", "atomIsSpinUp", "cellID")
PER_ID = ("evapPos", "evapVel")
PER_CELL = ("atomCount", "collisionCount")
PER_FRAME = ("atomNumber", "simuatedTime")
DATASETS = PER_ATOM + PER_ID + PER_CELL + PER_FRAME


def enable_records(sim) -> None:
    """Turns on the records the evapPos / evapVel / collisionCount datasets need."""
    sim.set_recording(REC_EVAPORATED | REC_CELL_COLLISIONS)


def snapshot_frame(sim, cloud: int = 0) -> dict:
    """One frame of every dataset for a cloud of `sim` (a Simulation, or the oracle, which has
    the same interface); the records must be on (enable_records)."""
    st = sim.get_state()
    counts = np.asarray(st["cloud_counts"], np.int64)
    a0 = int(counts[:cloud].sum())
    n = int(counts[cloud])
    pos, vel, psi = (st[k][a0:a0 + n] for k in ("pos", "vel", "psi"))
    bits = np.uint32 if pos.dtype == np.float32 else np.uint64
    starts = sim.cell_starts()
    # the cloud's cells: its grid cells then its overflow cell
    cell_of_cloud = [0]
    for c in sim.clouds:
        cell_of_cloud.append(cell_of_cloud[-1] + int(c.cells[0]) * int(c.cells[1]) * int(c.cells[2]) + 1)
    c0, c1 = cell_of_cloud[cloud], cell_of_cloud[cloud + 1]
    count = np.diff(starts)[c0:c1].astype(np.int32)
    cell = np.repeat(np.arange(c1 - c0, dtype=np.int32), count)
    ev = sim.evaporated(cloud)
    d = sim.diagnostics(cloud)
    return {
        "positions": pos[:, :3].astype(np.float64),
        "velocities": vel[:, :3].astype(np.float64),
        "psiUp": psi[:, 0:2].astype(np.float64),
        "psiDn": psi[:, 2:4].astype(np.float64),
        "atomID": (pos[:, 3].view(bits) & 0xFFFFFFFF).astype(np.int32),
        "atomIsSpinUp": ((vel[:, 3].view(bits) & 1) == 0).astype(np.uint8),  # flag bit 0: anti-trapped
        "cellID": cell,
        "evapPos": ev["pos"],
        "evapVel": ev["vel"],
        "atomCount": count,
        "collisionCount": sim.cell_collisions()[c0:c1].astype(np.int32),
        "atomNumber": np.array([n], np.int32),
        "simuatedTime": np.array([d["time"]], np.float64),
    }


def write_snapshot(sim, directory: str, frame: int, cloud: int = 0) -> dict:
    """Writes one frame of every dataset as <directory>/<name>_<frame>.npy; returns the frame."""
    os.makedirs(directory, exist_ok=True)
    f = snapshot_frame(sim, cloud)
    for name, arr in f.items():
        np.save(os.path.join(directory, f"{name}_{frame}.npy"), arr)
    return f


def _pad(arr: np.ndarray, rows: int) -> np.ndarray:
    if arr.shape[0] == rows:
        return arr
    fill = np.nan if arr.dtype.kind == "f" else (0 if arr.dtype == np.uint8 else -1)
    out = np.full((rows,) + arr.shape[1:], fill, dtype=arr.dtype)
    out[:arr.shape[0]] = arr
    return out


def read_snapshots(directory: str) -> dict:
    """Every dataset of the frames in `directory` as an (N, k, t) array, frames in order."""
    frames: dict[str, dict[int, np.ndarray]] = {}
    pat = re.compile(r"^(?P<name>[A-Za-z]+)_(?P<frame>\d+)\.npy$")
    for path in glob.glob(os.path.join(directory, "*_*.npy")):
        m = pat.match(os.path.basename(path))
        if not m or m["name"] not in DATASETS:
            continue
        frames.setdefault(m["name"], {})[int(m["frame"])] = np.load(path)
    out = {}
    for name, by_frame in frames.items():
        order = sorted(by_frame)
        if order != list(range(len(order))):
            raise ValueError(f"{name}: frames {order} are not 0..{len(order) - 1}")
        arrs = [a.reshape(a.shape[0], -1) for a in (by_frame[k] for k in order)]
        rows = max(a.shape[0] for a in arrs)
        out[name] = np.stack([_pad(a, rows) for a in arrs], axis=-1)
    return out


def save_npz(directory: str, path: str) -> dict:
    """Every dataset of the frames in `directory`, stacked as (N, k, t), into the archive `path`."""
    data = read_snapshots(directory)
    np.savez(path, **data)
    return data


def load_npz(path: str) -> dict:
    """The (N, k, t) datasets of an archive written by save_npz."""
    with np.load(path) as z:
        return {name: z[name] for name in z.files}

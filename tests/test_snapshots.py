"""Snapshot writer and reader round trip on CPU, with the oracle as the simulation.

cudadsmc_b200.snapshots writes one .npy file per dataset and frame under the reference's
/atomData names and reads the frames back as the reference's extendible (N, k, t) arrays
(CUDADSMC/src/main.cu:209-383, CUDADSMC/src/hdf5Helpers.cu:13-163).  The oracle has the engine's
interface, so the writer runs on it here: a small trapped cloud with the knife and Majorana loss
over three frames, every dataset read back and checked against the oracle's own state, its lost
atoms and its per-cell collision counts.
"""
import numpy as np

import oracle
from cudadsmc_b200 import F_COLLIDE, F_KNIFE, F_LARMOR, F_MAJORANA, F_NORMALISE
from cudadsmc_b200.snapshots import enable_records, load_npz, read_snapshots, save_npz, write_snapshot


def small_cloud():
    run, c = oracle.preset(2)
    c.n_atoms = c.capacity = 6000
    c.cells[0] = c.cells[1] = c.cells[2] = 16
    c.alpha = 5e4  # collisions in every step
    c.flags |= F_COLLIDE | F_LARMOR | F_NORMALISE | F_MAJORANA | F_KNIFE
    return run, c


def test_snapshot_round_trip_on_the_oracle(tmp_path):
    run, c = small_cloud()
    orc = oracle.Oracle(run, c)
    orc.init_cloud(11)
    enable_records(orc)
    frames = []
    for frame in range(3):
        if frame:
            orc.step(4)
        frames.append((write_snapshot(orc, str(tmp_path), frame), orc.get_state(), orc.diagnostics()))
    data = read_snapshots(str(tmp_path))
    assert sorted(data) == sorted(frames[0][0])
    n0 = c.n_atoms
    assert data["positions"].shape == (n0, 3, 3)
    assert data["evapPos"].shape == (n0, 3, 3)
    assert data["collisionCount"].shape == (16 ** 3 + 1, 1, 3)
    assert data["atomNumber"].shape == (1, 1, 3)
    for t, (_, st, d) in enumerate(frames):
        n = st["pos"].shape[0]
        assert data["atomNumber"][0, 0, t] == n == d["n_alive"]
        np.testing.assert_array_equal(data["positions"][:n, :, t], st["pos"][:, :3])
        assert np.all(np.isnan(data["positions"][n:, :, t]))  # padding after losses
        assert np.all(data["atomID"][n:, 0, t] == -1)
        np.testing.assert_array_equal(data["psiDn"][:n, :, t], st["psi"][:, 2:])
        assert data["simuatedTime"][0, 0, t] == d["time"]
        assert data["atomCount"][:, 0, t].sum() == n
    # lost atoms: exactly the ids missing from the last frame, at a position where they were lost
    last = frames[-1][1]
    alive = set((last["pos"][:, 3].view(np.uint32)).tolist())
    ev = orc.evaporated(0)
    lost = np.flatnonzero(ev["step"] >= 0)
    assert len(lost) == n0 - len(alive) > 0
    assert alive.isdisjoint(lost.tolist())
    np.testing.assert_array_equal(data["evapPos"][:, :, 2], ev["pos"])
    assert np.all(data["evapPos"][np.setdiff1d(np.arange(n0), lost), :, 2] == 0.0)
    d = frames[-1][2]
    assert set(np.unique(ev["fate"][lost]).tolist()) <= {1, 2}
    assert int((ev["fate"] == 1).sum()) == d["n_majorana"]
    # collision counts of the last collision step (step 7): each frame's counts add up to that
    # step's accepted collisions
    cc = data["collisionCount"][:, 0, 2]
    assert cc[-1] == 0  # the overflow cell never collides
    assert cc.sum() > 0
    orc2 = oracle.Oracle(run, c)
    orc2.init_cloud(11)
    orc2.step(7)
    before = orc2.diagnostics()["collisions"]
    orc2.step(1)
    assert cc.sum() == orc2.diagnostics()["collisions"] - before


def test_npz_archive_holds_the_stacked_frames(tmp_path):
    run, c = small_cloud()
    orc = oracle.Oracle(run, c)
    orc.init_cloud(5)
    enable_records(orc)
    for frame in range(2):
        if frame:
            orc.step(3)
        write_snapshot(orc, str(tmp_path / "frames"), frame)
    data = save_npz(str(tmp_path / "frames"), str(tmp_path / "atomData.npz"))
    back = load_npz(str(tmp_path / "atomData.npz"))
    assert sorted(back) == sorted(data)
    for name, arr in data.items():
        assert back[name].shape == arr.shape and back[name].dtype == arr.dtype, name
        np.testing.assert_array_equal(back[name], arr)
    assert back["positions"].shape[-1] == 2

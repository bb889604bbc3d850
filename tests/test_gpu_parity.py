"""GPU engine vs CPU oracle on the same seeded inputs, through the C ABI.

The engine and the oracle share the IEEE-exact per-atom arithmetic, so the bar is bit
equality of the whole state (positions, velocities, spinors, atom ids), of the cell
bookkeeping (cell starts = sorted order), of (sigma v_r)max and of the exact fixed-point
diagnostics, in FP32 and in FP64.
"""
import numpy as np
import pytest

import oracle
from cudadsmc_b200 import (FP32, FP64, F_COLLIDE, F_KNIFE, F_KNIFE_FIXED_T, F_LARMOR, F_MAJORANA, F_MCWF,
                           F_NORMALISE, TRAP_BOX, TRAP_IOFFE_PRITCHARD, INIT_THERMAL, Simulation, preset)
from cudadsmc_b200.engine import DSMCError

pytestmark = pytest.mark.gpu

ALL = F_COLLIDE | F_LARMOR | F_NORMALISE | F_MAJORANA | F_KNIFE | F_KNIFE_FIXED_T


def scaled(which, n=None, cells=None, precision=None, flags=None, **kw):
    run, c = preset(which)
    if precision is not None:
        run.precision = precision
    if n is not None:
        c.n_atoms = n
        c.capacity = n
    if cells is not None:
        c.cells[0] = c.cells[1] = c.cells[2] = cells
    if flags is not None:
        c.flags = flags
    for k, v in kw.items():
        if hasattr(run, k):
            setattr(run, k, v)
        else:
            setattr(c, k, v)
    return run, c


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)


def assert_same(sim, orc, diag=True):
    err = sim.diagnostics()["error"]
    assert err == 0, f"device error bits 0x{err:x}"
    g, o = sim.get_state(), orc.get_state()
    assert list(g["cloud_counts"]) == list(o["cloud_counts"])
    for key in ("pos", "vel", "psi"):
        assert g[key].shape == o[key].shape, key
        bad = np.nonzero(np.any(bits(g[key]) != bits(o[key]), axis=1))[0]
        assert bad.size == 0, f"{key}: {bad.size} atoms differ, first {bad[:5]}: {g[key][bad[:2]]} vs {o[key][bad[:2]]}"
    np.testing.assert_array_equal(sim.cell_starts(), orc.cell_starts())
    np.testing.assert_array_equal(bits(sim.sigvrmax()), bits(orc.sigvrmax()))
    if diag:
        dg, do = sim.diagnostics(), orc.diagnostics()
        for k in ("step", "n_alive", "sum_v2", "sum_absB", "n_evaporated", "n_majorana", "n_knife", "collisions",
                  "candidates", "e_kin", "e_pot", "e_evaporated", "temperature"):
            assert dg[k] == do[k], (k, dg[k], do[k])
        assert dg["error"] == 0


def run_pair(run, clouds, steps, check_every=None, seed=1234):
    sim = Simulation(run, clouds)
    orc = oracle.Oracle(run, clouds)
    sim.init_cloud(seed)
    orc.init_cloud(seed)
    assert_same(sim, orc)
    done = 0
    for s in (check_every or [steps]):
        sim.step(s)
        orc.step(s)
        done += s
        assert_same(sim, orc)
    return sim, orc


@pytest.mark.parametrize("precision", [FP32, FP64])
def test_init_bit_exact(precision):
    run, c = scaled(0, n=30000, precision=precision)
    sim = Simulation(run, c)
    orc = oracle.Oracle(run, c)
    sim.init_cloud(99)
    orc.init_cloud(99)
    assert_same(sim, orc)
    st = sim.get_state()
    ids = st["pos"][:, 3].view(np.uint32 if precision == FP32 else np.uint64).astype(np.int64)
    assert np.array_equal(np.sort(ids), np.arange(30000))


@pytest.mark.parametrize("precision", [FP32, FP64])
def test_small_trap_steps_bit_exact(precision):
    # the small trapped configuration (1e4 atoms, 50^3 cells, alpha = 300), 120 steps
    run, c = scaled(0, precision=precision)
    run_pair(run, c, 120, check_every=[1, 1, 18, 100])


def test_small_configuration_as_specified_bit_exact():
    # the small trapped configuration exactly as specified: 1e4 atoms, 50^3 cells, FP64, 1000
    # steps with collisions, run by the serial C++ step and by the GPU: identical after every decade
    run, c = scaled(0, precision=FP64)
    assert c.n_atoms == 10000 and c.cells[0] == 50
    run_pair(run, c, 1000, check_every=[1, 9, 90, 900])


@pytest.mark.parametrize("precision", [FP32, FP64])
def test_motion_and_spin_over_ten_thousand_steps_bit_exact(precision):
    # motion + Larmor precession + renormalisation over 10^4 steps (no collisions): the GPU state
    # equals the serial oracle's bit for bit at 10^2, 10^3 and 10^4 steps
    run, c = scaled(0, n=2000, precision=precision, flags=F_LARMOR | F_NORMALISE)
    run_pair(run, c, 10000, check_every=[100, 900, 9000])


@pytest.mark.parametrize("precision", [FP32, FP64])
def test_full_step_with_evaporation_bit_exact(precision):
    # Larmor + Majorana + knife ramp; a hotter cloud and a tight knife so atoms are removed
    run, c = scaled(2, n=60000, cells=40, precision=precision, flags=ALL, alpha=4000.0)
    c.knife_eta[0] = 6.0
    c.knife_eta[1] = 3.0
    c.knife_step[1] = 200
    sim, orc = run_pair(run, c, 60, check_every=[1, 9, 50])
    d = sim.diagnostics()
    assert d["n_knife"] > 0 and d["collisions"] > 0


def test_box_bit_exact():
    run, c = scaled(1, n=120000, cells=24)
    sim, orc = run_pair(run, c, 40, check_every=[1, 39])
    assert sim.diagnostics()["collisions"] > 0


def test_ioffe_pritchard_reference_trap_bit_exact():
    # the trap of CUDADSMC/src/moveAtoms.cu:135-142 with its constants
    # (include/deviceSystemParameters.cuh:25-27), 1 mm grid, 20 uK, rejection-sampled cloud
    run, c = scaled(0, n=8000, precision=FP64)
    c.trap = TRAP_IOFFE_PRITCHARD
    c.B0, c.dBdz, c.d2Bdz2 = 0.01, 20.0, 40000.0
    c.moment = 0.25 * 9.27400915e-24
    for a in range(3):
        c.grid_min[a], c.grid_max[a] = -1e-3, 1e-3
    c.cells[0] = c.cells[1] = c.cells[2] = 64
    c.flags = F_COLLIDE | F_LARMOR | F_NORMALISE | F_MAJORANA
    sim, orc = run_pair(run, c, 30, check_every=[1, 29])
    assert np.diff(sim.cell_starts())[:-1].max() < 513


def test_running_temperature_knife_bit_exact():
    # the knife of the running temperature (F_KNIFE_FIXED_T off) feeds the exact fixed-point T of
    # each step into the next cut
    run, c = scaled(2, n=30000, cells=32, flags=ALL & ~F_KNIFE_FIXED_T, alpha=4000.0)
    c.knife_eta[0] = c.knife_eta[1] = 7.0
    run_pair(run, c, 20, check_every=[1, 19])


def test_collide_every_and_odd_steps_graph_vs_plain():
    run, c = scaled(2, n=40000, cells=32, flags=ALL, alpha=4000.0, collide_every=3)
    a = Simulation(run, c)
    run2 = run.copy()
    run2.use_graphs = 0
    b = Simulation(run2, c)
    orc = oracle.Oracle(run, c)
    for s in (a, b, orc):
        s.init_cloud(5)
    for n in (1, 4, 7):
        a.step(n)
        b.step(n)
        orc.step(n)
        assert_same(a, orc)
        assert_same(b, orc)


def test_profiling_mode_identical():
    run, c = scaled(2, n=30000, cells=32, flags=ALL)
    a = Simulation(run, c)
    orc = oracle.Oracle(run, c)
    a.init_cloud(3)
    orc.init_cloud(3)
    a.set_profiling(True)
    a.step(5)
    orc.step(5)
    assert_same(a, orc)
    t = a.kernel_times()
    assert len(t) == a.launches_per_step() == 5  # dense_collide, step_pass, scan_cells, permute_pass, mover_rank
    assert all(v[1] == 5 for v in t.values())


@pytest.mark.parametrize("precision", [FP32, FP64])
def test_batched_clouds_match_oracle_and_single_runs(precision):
    rng = np.random.default_rng(7)
    clouds = []
    for k in range(5):
        run, c = scaled(2, n=int(rng.integers(500, 20000)), cells=int(rng.integers(8, 24)), flags=ALL, alpha=2000.0,
                        precision=precision)
        c.dBdz = float(rng.uniform(1.5, 4.0))
        c.temperature = float(rng.uniform(5e-6, 50e-6))
        from cudadsmc_b200.engine import load_library  # noqa
        # grid of +-5 thermal radii for this cloud
        rz = 1.3806503e-23 * c.temperature / (c.moment * c.dBdz)
        for a, r in ((0, 2 * rz), (1, 2 * rz), (2, rz)):
            c.grid_min[a], c.grid_max[a] = -5 * r, 5 * r
        c.stream_id = 11 + k
        clouds.append(c)
    clouds[2].n_atoms = clouds[2].capacity = 0  # an empty cloud
    sim, orc = run_pair(run, clouds, 25, check_every=[1, 24])
    batched = sim.get_state()
    off = np.concatenate([[0], np.cumsum(batched["cloud_counts"])])
    for k, c in enumerate(clouds):
        single = Simulation(run, c)
        single.init_cloud(1234)
        single.step(25)
        s = single.get_state()
        for key in ("pos", "vel", "psi"):
            assert np.array_equal(bits(s[key]), bits(batched[key][off[k]:off[k + 1]])), (k, key)
        ds, db = single.diagnostics(), sim.diagnostics(k)
        for f in ("n_alive", "sum_v2", "sum_absB", "collisions", "n_evaporated"):
            assert ds[f] == db[f], (k, f)
    # the batched entry points are the same engine: dsmc_batch_create + dsmc_batch_step
    import ctypes as C
    from cudadsmc_b200 import _abi
    from cudadsmc_b200.engine import load_library
    lib = load_library()
    arr = (_abi.CloudParams * len(clouds))(*clouds)
    h = C.c_void_p()
    assert lib.dsmc_batch_create(C.byref(run), arr, len(clouds), C.byref(h)) == 0
    try:
        assert lib.dsmc_init_cloud(h, C.c_uint64(1234)) == 0
        assert lib.dsmc_batch_step(h, 25) == 0
        d = _abi.Diag()
        assert lib.dsmc_diagnostics(h, -1, C.byref(d)) == 0
        assert d.n_alive == sim.diagnostics()["n_alive"] and d.sum_v2 == sim.diagnostics()["sum_v2"]
    finally:
        lib.dsmc_destroy(h)


def test_set_state_unsorted_input():
    run, c = scaled(2, n=30000, cells=24, flags=ALL)
    src = Simulation(run, c)
    src.init_cloud(21)
    src.step(3)
    st = src.get_state()
    perm = np.random.default_rng(3).permutation(st["pos"].shape[0])
    sim = Simulation(run, c)
    orc = oracle.Oracle(run, c)
    for s in (sim, orc):
        s.set_state(st["pos"][perm], st["vel"][perm], st["psi"][perm], st["cloud_counts"])
    assert_same(sim, orc, diag=False)
    sim.step(10)
    orc.step(10)
    assert_same(sim, orc, diag=False)


def test_overflow_spanning_many_tiles():
    # a grid much smaller than the cloud: most atoms live in the overflow cell, which is split
    # across tiles and carries its stayer count from tile to tile
    run, c = scaled(2, n=50000, cells=8, flags=ALL, tile_atoms=256)
    for a in range(3):
        c.grid_min[a] *= 0.15
        c.grid_max[a] *= 0.15
    sim, orc = run_pair(run, c, 20, check_every=[1, 19])
    starts = sim.cell_starts()
    assert starts[-1] - starts[-2] > 20000


def test_dense_cells_and_tiny_clouds():
    # hundreds of atoms per central cell of an 8^3 grid, next to a one-atom cloud
    run, c = scaled(2, n=12000, cells=8, flags=ALL, alpha=1.0)
    run2, c1 = scaled(2, n=1, cells=4, flags=ALL)
    c1.stream_id = 1
    sim, orc = run_pair(run, [c, c1], 12, check_every=[1, 11])
    occ = np.diff(sim.cell_starts())
    assert occ[:-1].max() > 300


DENSE_FP32 = 1280 + 1 - 512  # grid cells above this many atoms are split across tiles (FP32)


@pytest.mark.parametrize("precision,n,alpha", [(FP32, 4000, 2e7), (FP64, 4000, 2e7), (FP32, 16000, 2e6),
                                             (FP64, 8000, 5e6)])
def test_one_dense_cell_bit_exact(precision, n, alpha):
    # one cell holding most of the atoms, more than a tile stages: the cell is split across tiles,
    # its collisions run in dense_collide -- its velocities gathered into shared memory, or (16000
    # atoms in FP32, 8000 in FP64: more than the 12800 / 6400 that fit) into its slots of the step's
    # output buffer -- and the result is the oracle's
    run, c = scaled(2, n=n, cells=1, flags=F_COLLIDE | F_LARMOR, precision=precision, alpha=alpha)
    sim, orc = run_pair(run, c, 12, check_every=[1, 5, 6])
    occ = np.diff(sim.cell_starts())
    assert occ[0] > 0.75 * n
    assert sim.diagnostics()["collisions"] > 50


def test_dense_cells_split_across_small_tiles():
    # a coarse grid: dozens of cells above the dense threshold, each split across several
    # 256-atom tiles, beside ordinary cells and the overflow cell, with every step process on;
    # two clouds in one handle so that the split cells of both carry their ranks separately
    run, c = scaled(2, n=60000, cells=6, flags=ALL, tile_atoms=256, alpha=2e4)
    run2, c1 = scaled(2, n=20000, cells=5, flags=ALL, alpha=1e4)
    c1.stream_id = 1
    sim, orc = run_pair(run, [c, c1], 16, check_every=[1, 1, 6, 8])
    occ = np.diff(sim.cell_starts())
    grid = np.delete(occ, [6 ** 3, 6 ** 3 + 1 + 5 ** 3])  # the two overflow cells left out
    assert (grid > DENSE_FP32).sum() >= 6
    assert sim.diagnostics(0)["collisions"] > 0 and sim.diagnostics(1)["collisions"] > 0


@pytest.mark.parametrize("precision,threshold", [(FP32, 769), (FP64, 1025)])
def test_cells_crossing_the_dense_threshold(precision, threshold):
    # a hot periodic box whose 27 cells hold the dense threshold on average: every step some cells
    # become dense (split across tiles, collided by dense_collide) and others stop being
    # dense, while their stayers in later tiles still carry their ranks; bit-exact throughout
    run, c = scaled(1, n=27 * threshold, cells=3, flags=F_COLLIDE, precision=precision, temperature=2e-3,
                    alpha=3e5)
    sim = Simulation(run, c)
    orc = oracle.Oracle(run, c)
    sim.init_cloud(5)
    orc.init_cloud(5)
    seen_dense, flips, prev = 0, 0, None
    for _ in range(8):
        sim.step(5)
        orc.step(5)
        assert_same(sim, orc)
        d = np.diff(sim.cell_starts())[:-1] > threshold
        seen_dense += int(d.sum())
        flips += 0 if prev is None else int((d != prev).sum())
        prev = d
    assert seen_dense > 0 and flips > 0
    assert sim.diagnostics()["collisions"] > 1000


def test_dense_cells_default_tiles_and_collide_every():
    # the default (adaptive) tiling, collisions every third step, the MCWF flips at the
    # collision periods' ends: dense cells only change which kernel collides them
    run, c = scaled(2, n=80000, cells=8, flags=ALL | F_MCWF, collide_every=3, alpha=2e4)
    sim, orc = run_pair(run, c, 12, check_every=[2, 10])
    occ = np.diff(sim.cell_starts())
    assert occ[:-1].max() > DENSE_FP32


def test_autotune_changes_speed_not_results():
    # the tiling is a performance choice only: after the autotuner has stepped with every tile
    # size the state is bit-identical to the oracle's after the same number of steps
    run, c = scaled(2, n=60000, cells=32, flags=ALL, alpha=4000.0)
    sim = Simulation(run, c)
    orc = oracle.Oracle(run, c)
    sim.init_cloud(17)
    orc.init_cloud(17)
    tile, ms = sim.autotune(2)
    assert 128 <= tile <= 1024 and ms > 0
    # the table holds every (tile size, blocks per SM) candidate timed; the choice is its fastest
    table = sim.autotune_table()
    assert len(table["tile_atoms"]) >= 20 and len(set(table["blocks_per_sm"])) >= 2
    best = int(np.argmin(table["ms_per_step"]))
    assert table["tile_atoms"][best] == tile and table["blocks_per_sm"][best] == table["chosen_blocks_per_sm"]
    assert table["ms_per_step"][best] == ms
    orc.step(sim.diagnostics()["step"])
    assert_same(sim, orc)
    sim.step(3)
    orc.step(3)
    assert_same(sim, orc)


@pytest.mark.parametrize("precision,period", [(FP32, 1), (FP32, 3), (FP64, 3)])
def test_mcwf_flips_and_decoherence_bit_exact(precision, period):
    # MCWF (flip + decoherence + renormalisation once per collision period) with collisions,
    # starting from half-population spinors, half the atoms anti-trapped: flips happen, and the
    # GPU state, order and diagnostics equal the oracle's bit for bit
    run, c = scaled(2, n=30000, cells=24, precision=precision, flags=ALL | F_MCWF, alpha=4000.0)
    run.collide_every = period
    src = Simulation(run, c)
    src.init_cloud(5)
    st = src.get_state()
    pos, vel = st["pos"].astype(np.float64), st["vel"].copy()
    B = np.stack([0.5 * c.dBdz * pos[:, 0], 0.5 * c.dBdz * pos[:, 1], c.B0 - c.dBdz * pos[:, 2]], 1)
    b = B / np.linalg.norm(B, axis=1)[:, None]
    nrm = np.sqrt(2.0 * (1.0 + b[:, 2]))
    up_p, dn_p = (1.0 + b[:, 2]) / nrm, (b[:, 0] + 1j * b[:, 1]) / nrm
    up_m, dn_m = -(b[:, 0] - 1j * b[:, 1]) / nrm, (1.0 + b[:, 2]) / nrm
    u, d = np.sqrt(0.5) * (up_p + up_m), np.sqrt(0.5) * (dn_p + dn_m)
    psi = np.stack([u.real, u.imag, d.real, d.imag], 1).astype(st["psi"].dtype)
    w = vel[:, 3].view(np.uint32 if vel.dtype == np.float32 else np.uint64)
    w[::2] |= 1  # anti-trapped
    sim = Simulation(run, c)
    orc = oracle.Oracle(run, c)
    for s in (sim, orc):
        s.set_state(st["pos"], vel, psi, st["cloud_counts"])
    assert_same(sim, orc)
    flags0 = bits(sim.get_state()["vel"])[:, 3] & 1
    for n in (period, 2 * period + 1, 12):
        sim.step(n)
        orc.step(n)
        assert_same(sim, orc)
    g = sim.get_state()
    assert int(np.sum(bits(g["vel"])[:, 3] & 1)) != int(np.sum(flags0))  # spins flipped


def test_reinit_with_another_seed_matches_a_fresh_handle():
    # the step graphs carry the kernel parameters (the seed among them): a handle initialised
    # again with another seed steps like a fresh handle with that seed, for even and odd counts
    run, c = scaled(2, n=20000, cells=16, flags=ALL)
    a, b = Simulation(run, c), Simulation(run, c)
    a.init_cloud(1)
    a.step(4)
    a.step(3)
    a.init_cloud(2)
    b.init_cloud(2)
    for n in (4, 3, 1):
        a.step(n)
        b.step(n)
    da, db = a.diagnostics(), b.diagnostics()
    for k in ("step", "n_alive", "sum_v2", "sum_absB", "collisions", "candidates", "n_evaporated"):
        assert da[k] == db[k], (k, da[k], db[k])
    sa, sb = a.get_state(), b.get_state()
    for k in ("pos", "vel", "psi"):
        np.testing.assert_array_equal(sa[k], sb[k])


def test_diagnostics_enqueued_each_step_equal_the_synchronous_ones():
    # dsmc_diagnostics_enqueue copies a step's totals without waiting; collecting them afterwards
    # gives, slot by slot, exactly what dsmc_diagnostics returned after the same step of a twin run
    run, c = scaled(2, n=30000, cells=24, flags=ALL, alpha=4000.0)
    a, b = Simulation(run, c), Simulation(run, c)
    a.init_cloud(21)
    b.init_cloud(21)
    a.reserve_diagnostics(6)
    sync = []
    for k in range(6):
        a.step(1)
        a.diagnostics_enqueue(k)
        b.step(1)
        sync.append(b.diagnostics())
    for k in range(6):
        assert a.diagnostics_collect(k) == sync[k], k
    with pytest.raises(DSMCError):
        a.diagnostics_collect(6)  # outside the reserve
    a.reserve_diagnostics(8)  # grows: the new slots were never enqueued
    with pytest.raises(DSMCError):
        a.diagnostics_collect(7)
    assert a.diagnostics_copy_bytes() > 0


def test_every_atom_lost_then_empty_steps():
    # a knife at 0.02 kT removes the whole cloud in the first step; the empty cloud keeps
    # stepping (no tiles, no cells occupied) beside a second cloud that keeps its atoms, the
    # evaporated energy and counts equal the oracle's, and a state of zero atoms can be set
    run, c = scaled(2, n=5000, cells=16, flags=ALL, alpha=2e4)
    c.knife_nknots = 1
    c.knife_step[0] = 0.0
    c.knife_eta[0] = 0.02
    run2, c1 = scaled(2, n=3000, cells=12, flags=F_COLLIDE | F_LARMOR, alpha=2e4)
    c1.stream_id = 1
    sim, orc = run_pair(run, [c, c1], 6, check_every=[1, 1, 4])
    assert sim.diagnostics(0)["n_alive"] == 0 and sim.diagnostics(0)["n_evaporated"] == 5000
    assert sim.diagnostics(1)["n_alive"] == 3000
    # set_state with no atoms at all, then steps
    z = np.zeros((0, 4), dtype=np.float32)
    for s in (sim, orc):
        s.set_state(z, z, z, [0, 0])
    sim.step(2)
    orc.step(2)
    assert_same(sim, orc)
    assert sim.diagnostics()["n_alive"] == 0

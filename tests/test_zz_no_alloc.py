"""The allocation-free cell sort (dsmc_sort_cells_noalloc) against the oracle and the engine's sort.

Callers whose GPU memory belongs to another allocator (a PyTorch process, for example) cannot
count on cudaMalloc, and cudaMalloc / cudaFree would stall every stream of the device; this
entry point sorts caller-owned device positions with a fixed scratch array inside the library.
Its result must equal the CPU oracle's stable sort by (cell, input index) of the same atoms
(oracle set_state, then its state and cell starts), and what the engine's own entry points
produce: dsmc_set_state (which sorts its input stably by cell) followed by dsmc_get_state and
dsmc_get_cell_starts.  Two calls in a row check that the shared scratch is reset between calls.
The cases reach the limits of the scratch (262144 atoms, a 64^3 grid, atoms outside it), the
periodic box, and every atom in one cell (the sort's time must not grow with a cell's size).
This file is collected last so that a failure here never hides the other tests.
"""
import ctypes as C
import time

import numpy as np
import pytest

import oracle
from cudadsmc_b200 import FP32, FP64, TRAP_BOX, Simulation, load_library, preset

pytestmark = pytest.mark.gpu

MAX_ATOMS = 1 << 18


def cloud(precision, n=50000, cells=20):
    run, c = preset(2)
    run.precision = precision
    c.n_atoms = c.capacity = n
    c.cells[0] = c.cells[1] = c.cells[2] = cells
    return run, c


def noalloc_sort(run, c, pos_host, offset=0):
    """Calls the entry point on device copies of pos_host (offset: elements of padding in front)."""
    import torch
    lib = load_library()
    dev = torch.device("cuda", torch.cuda.current_device())
    n = pos_host.shape[0]
    buf = torch.zeros((n * 4 + offset,), dtype=torch.float32 if pos_host.dtype == np.float32 else torch.float64,
                      device=dev)
    buf[offset:] = torch.from_numpy(np.ascontiguousarray(pos_host).reshape(-1)).to(dev)
    ncells = c.cells[0] * c.cells[1] * c.cells[2]
    order = torch.full((max(n, 1),), -1, dtype=torch.int32, device=dev)
    starts = torch.full((ncells + 2,), -1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    st = lib.dsmc_sort_cells_noalloc(C.byref(run), C.byref(c), C.c_void_p(buf.data_ptr() + offset * buf.element_size()),
                                     n, C.c_void_p(order.data_ptr()), C.c_void_p(starts.data_ptr()),
                                     C.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    return st, order.cpu().numpy()[:n], starts.cpu().numpy()


def oracle_sort(run, c, pos, vel, psi):
    orc = oracle.Oracle(run, c)
    orc.set_state(pos, vel, psi, [pos.shape[0]])
    out = orc.get_state()["pos"], orc.cell_starts()
    orc.close()
    return out


def check_against_oracle(run, c, pos, vel, psi, view):
    st, order, starts = noalloc_sort(run, c, pos)
    assert st == 0
    n = pos.shape[0]
    expect_pos, expect_starts = oracle_sort(run, c, pos, vel, psi)
    assert np.array_equal(np.sort(order), np.arange(n))
    assert np.array_equal(starts, expect_starts)
    assert np.array_equal(pos[order].view(view), expect_pos.view(view))
    return order, starts


@pytest.mark.parametrize("precision", [FP32, FP64])
def test_noalloc_sort_matches_engine_and_oracle(precision):
    run, c = cloud(precision)
    src = Simulation(run, c)
    src.init_cloud(4321)
    src.step(3)
    state = src.get_state()
    n = state["pos"].shape[0]
    view = np.uint32 if precision == FP32 else np.uint64
    for call, seed in enumerate((1, 2)):  # two calls in a row, different inputs
        perm = np.random.default_rng(seed).permutation(n)
        shuffled = {k: state[k][perm] for k in ("pos", "vel", "psi")}
        ref = Simulation(run, c)
        ref.set_state(shuffled["pos"], shuffled["vel"], shuffled["psi"], state["cloud_counts"])
        expect_pos = ref.get_state()["pos"]
        expect_starts = ref.cell_starts()
        order, starts = check_against_oracle(run, c, shuffled["pos"], shuffled["vel"], shuffled["psi"], view)
        assert np.array_equal(starts, expect_starts), call
        assert np.array_equal(shuffled["pos"][order].view(view), expect_pos.view(view)), call
        ref.close()


def random_state(rng, n, lo, hi, dtype):
    pos = np.zeros((n, 4), dtype=dtype)
    pos[:, :3] = rng.uniform(lo, hi, size=(n, 3))
    pos[:, 3] = np.arange(n).astype(np.uint32).view(np.float32) if dtype == np.float32 else \
        np.arange(n).astype(np.uint64).view(np.float64)
    vel = np.zeros((n, 4), dtype=dtype)
    vel[:, :3] = rng.normal(0.0, 0.05, size=(n, 3))
    psi = np.zeros((n, 4), dtype=dtype)
    psi[:, 0] = 1.0
    return pos, vel, psi


def test_noalloc_sort_at_capacity_with_atoms_outside_the_grid():
    run, c = cloud(FP32, n=MAX_ATOMS, cells=64)
    rng = np.random.default_rng(7)
    lo = np.array(c.grid_min[:])
    hi = np.array(c.grid_max[:])
    span = hi - lo
    pos, vel, psi = random_state(rng, MAX_ATOMS, lo - 0.1 * span, hi + 0.1 * span, np.float32)
    for _ in range(2):
        order, starts = check_against_oracle(run, c, pos, vel, psi, np.uint32)
    assert starts[-1] == MAX_ATOMS
    assert starts[-1] - starts[-2] > 1000  # many atoms in the overflow cell


def test_noalloc_sort_periodic_box():
    run, c = preset(1)
    c.n_atoms = c.capacity = 100000
    c.cells[0] = c.cells[1] = c.cells[2] = 40
    assert c.trap == TRAP_BOX
    rng = np.random.default_rng(11)
    pos, vel, psi = random_state(rng, c.n_atoms, np.array(c.grid_min[:]), np.array(c.grid_max[:]), np.float32)
    check_against_oracle(run, c, pos, vel, psi, np.uint32)


def test_noalloc_sort_one_cell_holding_every_atom():
    """Every atom in one grid cell: the sort keeps its per-atom cost (no pass over the cell per atom)."""
    import torch
    run, c = cloud(FP32, n=MAX_ATOMS, cells=8)
    rng = np.random.default_rng(3)
    lo = np.array(c.grid_min[:])
    cell = (np.array(c.grid_max[:]) - lo) / 8
    corner = lo + 3 * cell
    pos, vel, psi = random_state(rng, MAX_ATOMS, corner + 0.25 * cell, corner + 0.75 * cell, np.float32)
    order, starts = check_against_oracle(run, c, pos, vel, psi, np.uint32)
    assert np.max(np.diff(starts)) == MAX_ATOMS
    assert np.array_equal(order, np.arange(MAX_ATOMS))  # stable: input order within the cell
    # time a call with CUDA events on the current stream: a few kernels over 2^18 atoms
    lib = load_library()
    dev = torch.device("cuda", torch.cuda.current_device())
    dpos = torch.from_numpy(pos).to(dev)
    dord = torch.empty((MAX_ATOMS,), dtype=torch.int32, device=dev)
    dst = torch.empty((8 ** 3 + 2,), dtype=torch.int32, device=dev)
    s = torch.cuda.current_stream()
    args = (C.byref(run), C.byref(c), C.c_void_p(dpos.data_ptr()), MAX_ATOMS, C.c_void_p(dord.data_ptr()),
            C.c_void_p(dst.data_ptr()), C.c_void_p(s.cuda_stream))
    assert lib.dsmc_sort_cells_noalloc(*args) == 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    assert lib.dsmc_sort_cells_noalloc(*args) == 0
    e1.record(s)
    e1.synchronize()
    assert e0.elapsed_time(e1) < 5.0  # milliseconds


def test_noalloc_rejects_misaligned_positions():
    run, c = cloud(FP32, n=1000)
    rng = np.random.default_rng(5)
    pos, _, _ = random_state(rng, 1000, np.array(c.grid_min[:]), np.array(c.grid_max[:]), np.float32)
    st, _, _ = noalloc_sort(run, c, pos, offset=1)  # 4 bytes off a 16-byte boundary
    assert st == 1  # DSMC_ERR_INVALID, before any GPU work
    st, _, _ = noalloc_sort(run, c, pos, offset=4)
    assert st == 0


def test_noalloc_rejects_oversized_input():
    run, c = cloud(FP32)
    lib = load_library()
    st = lib.dsmc_sort_cells_noalloc(C.byref(run), C.byref(c), C.c_void_p(1), MAX_ATOMS + 1, C.c_void_p(1),
                                     C.c_void_p(1), None)
    assert st == 4  # DSMC_ERR_CAPACITY, before any GPU work
    c.cells[0] = c.cells[1] = c.cells[2] = 65
    st = lib.dsmc_sort_cells_noalloc(C.byref(run), C.byref(c), C.c_void_p(1), 10, C.c_void_p(1), C.c_void_p(1), None)
    assert st == 4

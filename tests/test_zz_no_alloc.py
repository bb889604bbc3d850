"""The allocation-free cell sort (dsmc_sort_cells_noalloc) against the engine's own sort.

Callers whose GPU memory belongs to another allocator (a PyTorch process, for example) cannot
count on cudaMalloc, and cudaMalloc / cudaFree would stall every stream of the device; this
entry point sorts caller-owned device positions with a fixed scratch array inside the library.
Its result must equal what the existing entry points produce for the same atoms:
dsmc_set_state (which sorts its input stably by cell) followed by dsmc_get_state and
dsmc_get_cell_starts.  Two calls in a row check that the shared scratch is reset between calls.
This file is collected last so that a failure here never hides the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from cudadsmc_b200 import FP32, FP64, Simulation, load_library, preset

pytestmark = pytest.mark.gpu


def cloud(precision):
    run, c = preset(2)
    run.precision = precision
    c.n_atoms = c.capacity = 50000
    c.cells[0] = c.cells[1] = c.cells[2] = 20
    return run, c


def noalloc_sort(run, c, pos_host):
    import torch
    lib = load_library()
    dev = torch.device("cuda", torch.cuda.current_device())
    pos = torch.from_numpy(np.ascontiguousarray(pos_host)).to(dev)
    n = pos.shape[0]
    ncells = c.cells[0] * c.cells[1] * c.cells[2]
    order = torch.full((n,), -1, dtype=torch.int32, device=dev)
    starts = torch.full((ncells + 2,), -1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    st = lib.dsmc_sort_cells_noalloc(C.byref(run), C.byref(c), C.c_void_p(pos.data_ptr()), n,
                                     C.c_void_p(order.data_ptr()), C.c_void_p(starts.data_ptr()),
                                     C.c_void_p(stream.cuda_stream))
    assert st == 0
    torch.cuda.synchronize()
    return order.cpu().numpy(), starts.cpu().numpy()


@pytest.mark.parametrize("precision", [FP32, FP64])
def test_noalloc_sort_matches_engine_sort(precision):
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
        order, starts = noalloc_sort(run, c, shuffled["pos"])
        assert np.array_equal(starts, expect_starts), call
        assert np.array_equal(np.sort(order), np.arange(n)), call
        assert np.array_equal(shuffled["pos"][order].view(view), expect_pos.view(view)), call
        ref.close()


def test_noalloc_rejects_oversized_input():
    run, c = cloud(FP32)
    lib = load_library()
    st = lib.dsmc_sort_cells_noalloc(C.byref(run), C.byref(c), C.c_void_p(1), (1 << 18) + 1, C.c_void_p(1),
                                     C.c_void_p(1), None)
    assert st == 4  # DSMC_ERR_CAPACITY, before any GPU work
    c.cells[0] = c.cells[1] = c.cells[2] = 65
    st = lib.dsmc_sort_cells_noalloc(C.byref(run), C.byref(c), C.c_void_p(1), 10, C.c_void_p(1), C.c_void_p(1), None)
    assert st == 4

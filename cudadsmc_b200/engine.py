"""Python binding of the sm_100a DSMC engine (libdsmc_b200.so, C ABI in include/dsmc.h).

``Simulation`` follows the call structure of CUDADSMC's ``main()`` (CUDADSMC/src/main.cu):
create the handle (allocation, main.cu:83-140), ``init_cloud`` (h_initRNG +
h_generateInitialDist + initSigvrmax, setUp.cu:32-292), ``step`` (one pass of the loop body,
main.cu:416-523) and ``diagnostics`` / ``get_state`` (the snapshot copies, main.cu:526-577).
There is no CPU fallback: if the library is missing or no GPU is present the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

from . import _abi
from ._abi import AdjParams, CloudParams, Diag, Grad, RunParams, StateBuffers

_LIB = None
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libdsmc_b200.so")

# every symbol include/dsmc.h declares
EXPORTED_SYMBOLS = (
    "dsmc_abi_version", "dsmc_status_string", "dsmc_last_error", "dsmc_preset", "dsmc_create",
    "dsmc_destroy", "dsmc_set_stream", "dsmc_init_cloud", "dsmc_step", "dsmc_synchronize",
    "dsmc_batch_create", "dsmc_batch_step",
    "dsmc_diagnostics", "dsmc_diagnostics_reserve", "dsmc_diagnostics_enqueue", "dsmc_diagnostics_collect",
    "dsmc_diagnostics_copy_bytes",
    "dsmc_get_state", "dsmc_set_state", "dsmc_get_cell_starts",
    "dsmc_get_sigvrmax", "dsmc_set_sigvrmax", "dsmc_set_profiling", "dsmc_kernel_times",
    "dsmc_launches_per_step", "dsmc_autotune", "dsmc_autotune_table", "dsmc_set_recording", "dsmc_get_evaporated", "dsmc_get_cell_collisions",
    "dsmc_adjoint_run", "dsmc_adjoint_loss", "dsmc_adjoint_loss_parts",
    "dsmc_adjoint_export", "dsmc_adjoint_export_spinors",
    "dsmc_sort_cells_noalloc", "dsmc_check_wait_timeout",
)


class DSMCError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def load_library(path: str | None = None) -> C.CDLL:
    """Loads libdsmc_b200.so (raises if it has not been built); DSMC_LIB overrides the path."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or os.environ.get("DSMC_LIB") or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(f"{p} is missing: build it with `python -m cudadsmc_b200.build`")
    lib = C.CDLL(p)
    vp, i32, i64, u64 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64
    sig = {
        "dsmc_abi_version": (i32, []),
        "dsmc_status_string": (C.c_char_p, [i32]),
        "dsmc_last_error": (C.c_char_p, [vp]),
        "dsmc_preset": (i32, [i32, C.POINTER(RunParams), C.POINTER(CloudParams)]),
        "dsmc_create": (i32, [C.POINTER(RunParams), C.POINTER(CloudParams), i32, C.POINTER(vp)]),
        "dsmc_destroy": (i32, [vp]),
        "dsmc_set_stream": (i32, [vp, vp]),
        "dsmc_init_cloud": (i32, [vp, u64]),
        "dsmc_step": (i32, [vp, i32]),
        "dsmc_batch_create": (i32, [C.POINTER(RunParams), C.POINTER(CloudParams), i32, C.POINTER(vp)]),
        "dsmc_batch_step": (i32, [vp, i32]),
        "dsmc_synchronize": (i32, [vp]),
        "dsmc_diagnostics": (i32, [vp, i32, C.POINTER(Diag)]),
        "dsmc_diagnostics_reserve": (i32, [vp, i32]),
        "dsmc_diagnostics_enqueue": (i32, [vp, i32]),
        "dsmc_diagnostics_collect": (i32, [vp, i32, i32, C.POINTER(Diag)]),
        "dsmc_diagnostics_copy_bytes": (C.c_int64, [vp]),
        "dsmc_get_state": (i32, [vp, C.POINTER(StateBuffers)]),
        "dsmc_set_state": (i32, [vp, C.POINTER(StateBuffers)]),
        "dsmc_get_cell_starts": (i32, [vp, C.POINTER(C.c_int32), i64, C.POINTER(i64)]),
        "dsmc_get_sigvrmax": (i32, [vp, vp, i64]),
        "dsmc_set_sigvrmax": (i32, [vp, vp, i64]),
        "dsmc_set_profiling": (i32, [vp, i32]),
        "dsmc_kernel_times": (i32, [vp, C.POINTER(C.c_char_p), C.POINTER(C.c_double), C.POINTER(i64), i32,
                                    C.POINTER(i32)]),
        "dsmc_launches_per_step": (i32, [vp]),
        "dsmc_check_wait_timeout": (i32, [vp, C.POINTER(i32)]),
        "dsmc_autotune": (i32, [vp, i32, C.POINTER(i32), C.POINTER(C.c_double)]),
        "dsmc_adjoint_run": (i32, [vp, C.POINTER(AdjParams), C.POINTER(Grad)]),
        "dsmc_adjoint_loss": (i32, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "dsmc_adjoint_loss_parts": (i32, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double)]),
        "dsmc_adjoint_export_spinors": (i32, [vp, C.POINTER(C.c_double), i64]),
        "dsmc_set_recording": (i32, [vp, i32]),
        "dsmc_autotune_table": (i32, [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(C.c_double), i32, C.POINTER(i32),
                                      C.POINTER(i32)]),
        "dsmc_get_evaporated": (i32, [vp, i32, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(i32),
                                      C.POINTER(i32), i64]),
        "dsmc_get_cell_collisions": (i32, [vp, C.POINTER(i32), i64, C.POINTER(i64)]),
        "dsmc_adjoint_export": (i32, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), i64, C.POINTER(i32), i64,
                                      C.POINTER(i32), C.POINTER(C.c_double), i64, C.POINTER(i64), C.POINTER(i64),
                                      C.POINTER(i32)]),
        "dsmc_sort_cells_noalloc": (i32, [C.POINTER(RunParams), C.POINTER(CloudParams), vp, i64, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _LIB = lib
    return lib


def preset(which: int) -> tuple[RunParams, CloudParams]:
    """Named workloads of the engine (see dsmc_preset in include/dsmc.h)."""
    lib = load_library()
    run, cloud = RunParams(), CloudParams()
    st = lib.dsmc_preset(which, C.byref(run), C.byref(cloud))
    if st != 0:
        raise DSMCError(st, f"unknown preset {which}")
    return run, cloud


def real_dtype(run: RunParams):
    return np.float32 if run.precision == _abi.FP32 else np.float64


class Simulation:
    """One engine handle: one or more clouds advanced together on the current GPU."""

    def __init__(self, run: RunParams, clouds: CloudParams | Sequence[CloudParams]):
        self.lib = load_library()
        if isinstance(clouds, CloudParams):
            clouds = [clouds]
        self.run = run.copy()
        self.clouds = [c.copy() for c in clouds]
        arr = (CloudParams * len(self.clouds))(*self.clouds)
        h = C.c_void_p()
        st = self.lib.dsmc_create(C.byref(self.run), arr, len(self.clouds), C.byref(h))
        if st != 0:
            raise DSMCError(st, self.lib.dsmc_last_error(None).decode())
        self._h = h
        self.dtype = real_dtype(run)

    # -- lifecycle ---------------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.dsmc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int) -> None:
        if st != 0:
            raise DSMCError(st, self.lib.dsmc_last_error(self._h).decode())

    # -- reference loop --------------------------------------------------------------------------
    def init_cloud(self, seed: int | None = None) -> None:
        self._check(self.lib.dsmc_init_cloud(self._h, int(self.run.seed if seed is None else seed)))

    def step(self, nsteps: int = 1) -> None:
        self._check(self.lib.dsmc_step(self._h, int(nsteps)))

    def synchronize(self) -> None:
        self._check(self.lib.dsmc_synchronize(self._h))

    def set_stream(self, stream_ptr: int) -> None:
        self._check(self.lib.dsmc_set_stream(self._h, C.c_void_p(stream_ptr)))

    def diagnostics(self, cloud: int = -1) -> dict:
        d = Diag()
        self._check(self.lib.dsmc_diagnostics(self._h, int(cloud), C.byref(d)))
        return d.as_dict()

    def reserve_diagnostics(self, nslots: int) -> None:
        """Pinned host slots for diagnostics_enqueue / diagnostics_collect."""
        self._check(self.lib.dsmc_diagnostics_reserve(self._h, int(nslots)))

    def diagnostics_enqueue(self, slot: int) -> None:
        """Copies the current step totals into `slot` on the stream, without waiting."""
        self._check(self.lib.dsmc_diagnostics_enqueue(self._h, int(slot)))

    def diagnostics_copy_bytes(self) -> int:
        """Bytes one diagnostics_enqueue copies from the device."""
        return int(self.lib.dsmc_diagnostics_copy_bytes(self._h))

    def diagnostics_collect(self, slot: int, cloud: int = -1) -> dict:
        """The diagnostics as they were when `slot` was enqueued (waits for that copy only)."""
        d = Diag()
        self._check(self.lib.dsmc_diagnostics_collect(self._h, int(slot), int(cloud), C.byref(d)))
        return d.as_dict()

    # -- state -------------------------------------------------------------------------------------
    def n_alive(self) -> int:
        return int(self.diagnostics()["n_alive"])

    def get_state(self, out: dict = None) -> dict:
        """Sorted state: pos/vel/psi as (n, 4) arrays, atom ids, cloud counts.  `out` may give
        C-contiguous (capacity, 4) arrays of the handle's precision for pos/vel/psi (pinned host
        memory, say) to be filled instead of new ones."""
        cap = int(sum(max(c.capacity, c.n_atoms) for c in self.clouds))
        if out is not None:
            pos, vel, psi = out["pos"], out["vel"], out["psi"]
            for a in (pos, vel, psi):
                if a.dtype != self.dtype or a.ndim != 2 or a.shape[1] != 4 or not a.flags["C_CONTIGUOUS"]:
                    raise ValueError("out arrays must be C-contiguous (capacity, 4) of the handle's precision")
            cap = min(a.shape[0] for a in (pos, vel, psi))
        else:
            pos = np.empty((cap, 4), self.dtype)
            vel = np.empty((cap, 4), self.dtype)
            psi = np.empty((cap, 4), self.dtype)
        counts = np.zeros(len(self.clouds), np.int64)
        b = StateBuffers(pos.ctypes.data, vel.ctypes.data, psi.ctypes.data, cap,
                         counts.ctypes.data_as(C.POINTER(C.c_int64)))
        self._check(self.lib.dsmc_get_state(self._h, C.byref(b)))
        n = int(b.n)
        return {"pos": pos[:n], "vel": vel[:n], "psi": psi[:n], "cloud_counts": counts}

    def set_state(self, pos: np.ndarray, vel: np.ndarray, psi: np.ndarray, cloud_counts) -> None:
        pos = np.ascontiguousarray(pos, self.dtype)
        vel = np.ascontiguousarray(vel, self.dtype)
        psi = np.ascontiguousarray(psi, self.dtype)
        counts = np.ascontiguousarray(np.asarray(cloud_counts, np.int64))
        n = pos.shape[0]
        b = StateBuffers(pos.ctypes.data, vel.ctypes.data, psi.ctypes.data, n,
                         counts.ctypes.data_as(C.POINTER(C.c_int64)))
        self._check(self.lib.dsmc_set_state(self._h, C.byref(b)))

    def cell_starts(self) -> np.ndarray:
        total = C.c_int64()
        self._check(self.lib.dsmc_get_cell_starts(self._h, None, 0, C.byref(total)))
        out = np.empty(total.value + 1, np.int32)
        self._check(self.lib.dsmc_get_cell_starts(self._h, out.ctypes.data_as(C.POINTER(C.c_int32)),
                                                  out.size, C.byref(total)))
        return out

    def sigvrmax(self) -> np.ndarray:
        total = C.c_int64()
        self._check(self.lib.dsmc_get_cell_starts(self._h, None, 0, C.byref(total)))
        out = np.empty(total.value, self.dtype)
        self._check(self.lib.dsmc_get_sigvrmax(self._h, out.ctypes.data, out.size))
        return out

    def set_sigvrmax(self, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, self.dtype)
        self._check(self.lib.dsmc_set_sigvrmax(self._h, v.ctypes.data, v.size))

    # -- profiling ---------------------------------------------------------------------------------
    def set_profiling(self, on: bool) -> None:
        self._check(self.lib.dsmc_set_profiling(self._h, 1 if on else 0))

    def kernel_times(self) -> dict:
        names = (C.c_char_p * 32)()
        ms = (C.c_double * 32)()
        launches = (C.c_int64 * 32)()
        cnt = C.c_int32()
        self._check(self.lib.dsmc_kernel_times(self._h, names, ms, launches, 32, C.byref(cnt)))
        return {names[i].decode(): (ms[i], launches[i]) for i in range(cnt.value)}

    def launches_per_step(self) -> int:
        return int(self.lib.dsmc_launches_per_step(self._h))

    def check_wait_timeout(self) -> int:
        """Runs the coming step's cell scan with its first block withheld (dsmc_check_wait_timeout):
        returns the device error bits it left, 64 (a bounded wait gave up) among them."""
        bits = C.c_int32(0)
        self._check(self.lib.dsmc_check_wait_timeout(self._h, C.byref(bits)))
        return int(bits.value)

    # -- snapshot records ---------------------------------------------------------------------------
    def set_recording(self, flags: int) -> None:
        """Turns the snapshot records on (cleared) or off: REC_EVAPORATED, REC_CELL_COLLISIONS."""
        self._check(self.lib.dsmc_set_recording(self._h, int(flags)))

    def evaporated(self, cloud: int = 0) -> dict:
        """The lost atoms of a cloud by atom id: position, velocity, step and fate (1 Majorana,
        2 knife) at the step each was lost in (step -1 and zeros for atoms never lost)."""
        c = self.clouds[cloud]
        n = int(c.capacity if c.capacity > 0 else c.n_atoms)
        pos, vel = np.zeros((max(n, 1), 3)), np.zeros((max(n, 1), 3))
        step, fate = np.zeros(max(n, 1), np.int32), np.zeros(max(n, 1), np.int32)
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        self._check(self.lib.dsmc_get_evaporated(self._h, int(cloud), dp(pos), dp(vel), ip(step), ip(fate), max(n, 1)))
        return {"pos": pos[:n], "vel": vel[:n], "step": step[:n], "fate": fate[:n]}

    def cell_collisions(self) -> np.ndarray:
        """Accepted collisions of every global cell in the last step that ran the collisions."""
        total = C.c_int64()
        self._check(self.lib.dsmc_get_cell_collisions(self._h, None, 0, C.byref(total)))
        out = np.zeros(max(total.value, 1), np.int32)
        self._check(self.lib.dsmc_get_cell_collisions(self._h, out.ctypes.data_as(C.POINTER(C.c_int32)), out.size,
                                                      C.byref(total)))
        return out[:total.value]

    # -- pathwise adjoint -----------------------------------------------------------------------------
    def adjoint_run(self, steps: int, checkpoint_every: int = 100, precision: int = _abi.FP64,
                    sigmoid_width_kT: float = 0.2, majorana_width: float = 0.05) -> dict:
        """Runs `steps` physical steps recording the collisions, then the smoothed loss and its
        gradient w.r.t. (B', B0, knife knots): of the sum (dL_*) and of each term (dE_dtheta for the
        mean energy, dN_dtheta for the retained fraction); see dsmc_adjoint_run in include/dsmc.h."""
        p = AdjParams(int(steps), int(checkpoint_every), int(precision), 0, float(sigmoid_width_kT),
                      float(majorana_width))
        g = Grad()
        self._check(self.lib.dsmc_adjoint_run(self._h, C.byref(p), C.byref(g)))
        return g.as_dict()

    def adjoint_loss(self, theta=None, grad: bool = False):
        """Smoothed loss of the recorded run at theta = (B', B0, eta_0..eta_8), same collisions."""
        loss = C.c_double()
        g = np.zeros(11, np.float64)
        th = None if theta is None else np.ascontiguousarray(theta, np.float64)
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        self._check(self.lib.dsmc_adjoint_loss(self._h, dp(th) if th is not None else None, C.byref(loss),
                                               dp(g) if grad else None))
        return (loss.value, g) if grad else loss.value

    def adjoint_loss_parts(self, theta=None, grad: bool = False):
        """The two terms (L_E, L_N) of the smoothed loss at theta and, with grad, their gradients."""
        parts = np.zeros(2, np.float64)
        ge = np.zeros(11, np.float64)
        gn = np.zeros(11, np.float64)
        th = None if theta is None else np.ascontiguousarray(theta, np.float64)
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        self._check(self.lib.dsmc_adjoint_loss_parts(self._h, dp(th) if th is not None else None, dp(parts),
                                                     dp(ge) if grad else None, dp(gn) if grad else None))
        return (parts, ge, gn) if grad else parts

    def adjoint_export(self) -> dict:
        na, nl, st = C.c_int64(), C.c_int64(), C.c_int32()
        self._check(self.lib.dsmc_adjoint_export(self._h, None, None, 0, None, 0, None, None, 0, C.byref(na),
                                                 C.byref(nl), C.byref(st)))
        n, m, steps = na.value, nl.value, st.value
        x0 = np.zeros((n, 3)); v0 = np.zeros((n, 3))
        off = np.zeros(steps + 1, np.int32); ij = np.zeros((max(m, 1), 2), np.int32); nv = np.zeros((max(m, 1), 3))
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        self._check(self.lib.dsmc_adjoint_export(self._h, dp(x0), dp(v0), n, ip(off), steps + 1, ip(ij), dp(nv),
                                                 max(m, 1), C.byref(na), C.byref(nl), C.byref(st)))
        psi0 = np.zeros((max(n, 1), 4))
        self._check(self.lib.dsmc_adjoint_export_spinors(self._h, dp(psi0), max(n, 1)))
        return {"x0": x0, "v0": v0, "psi0": psi0[:n], "off": off, "ij": ij[:m], "n": nv[:m], "steps": steps}

    def autotune(self, steps_per_candidate: int = 5) -> tuple[int, float]:
        """Chooses the tile size by timing (advances the simulation); returns (tile, ms/step)."""
        t = C.c_int32()
        ms = C.c_double()
        self._check(self.lib.dsmc_autotune(self._h, int(steps_per_candidate), C.byref(t), C.byref(ms)))
        return int(t.value), float(ms.value)

    def autotune_table(self) -> dict:
        """The last autotune's candidates: tile sizes, step-kernel blocks per SM, ms per step, and
        the blocks per SM chosen."""
        n, b = C.c_int32(), C.c_int32()
        self._check(self.lib.dsmc_autotune_table(self._h, None, None, None, 0, C.byref(n), C.byref(b)))
        T = np.zeros(max(n.value, 1), np.int32)
        B = np.zeros(max(n.value, 1), np.int32)
        ms = np.zeros(max(n.value, 1))
        self._check(self.lib.dsmc_autotune_table(self._h, T.ctypes.data_as(C.POINTER(C.c_int32)),
                                                 B.ctypes.data_as(C.POINTER(C.c_int32)),
                                                 ms.ctypes.data_as(C.POINTER(C.c_double)), n.value, C.byref(n),
                                                 C.byref(b)))
        return {"tile_atoms": T[:n.value].tolist(), "blocks_per_sm": B[:n.value].tolist(),
                "ms_per_step": ms[:n.value].tolist(), "chosen_blocks_per_sm": int(b.value)}

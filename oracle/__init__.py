"""CPU oracle of the DSMC timestep -- TEST INFRASTRUCTURE ONLY.

Python binding of oracle/build/liboracle.so (dsmc_oracle.cpp, a serial C++ restatement of
CUDADSMC's timestep that shares the IEEE-exact per-atom arithmetic of the engine).  Only the
tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use it; the engine never
does.  ``Oracle`` mirrors ``cudadsmc_b200.Simulation`` method for method.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

from cudadsmc_b200._abi import CloudParams, Diag, RunParams, StateBuffers, FP32

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liboracle.so")
_LIB = None


def load() -> C.CDLL:
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            from cudadsmc_b200 import build as _b
            _b.build_oracle()
        lib = C.CDLL(LIB_PATH)
        vp, i32, i64, u64 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64
        sig = {
            "oracle_create": (i32, [C.POINTER(RunParams), C.POINTER(CloudParams), i32, i32, C.POINTER(vp)]),
            "oracle_last_error": (C.c_char_p, [vp]),
            "oracle_destroy": (None, [vp]),
            "oracle_init": (i32, [vp, u64]),
            "oracle_step": (i32, [vp, i32]),
            "oracle_diag": (i32, [vp, i32, C.POINTER(Diag)]),
            "oracle_get_state": (i32, [vp, C.POINTER(StateBuffers)]),
            "oracle_set_state": (i32, [vp, C.POINTER(StateBuffers)]),
            "oracle_get_cell_starts": (i32, [vp, C.POINTER(C.c_int32), i64, C.POINTER(i64)]),
            "oracle_get_sigvrmax": (i32, [vp, vp, i64]),
            "oracle_set_sigvrmax": (i32, [vp, vp, i64]),
            "oracle_set_recording": (i32, [vp, i32]),
            "oracle_get_evaporated": (i32, [vp, i32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                            C.POINTER(C.c_int32), C.POINTER(C.c_int32), i64]),
            "oracle_get_cell_collisions": (i32, [vp, C.POINTER(C.c_int32), i64]),
            "oracle_max_threads": (i32, []),
            "oracle_set_threads": (None, [i32]),
            "oracle_preset": (i32, [i32, C.POINTER(RunParams), C.POINTER(CloudParams)]),
            "oracle_philox": (None, [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
            "oracle_math_f": (None, [i32, C.POINTER(C.c_float), C.POINTER(C.c_float), i64]),
            "oracle_math_d": (None, [i32, C.POINTER(C.c_double), C.POINTER(C.c_double), i64]),
            "oracle_fx": (None, [i32, C.c_void_p, C.POINTER(C.c_uint64), i64]),
            "oracle_field_d": (i32, [C.POINTER(RunParams), C.POINTER(CloudParams), C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), i64]),
            "oracle_smooth_loss": (C.c_double, [C.POINTER(RunParams), C.POINTER(CloudParams), C.POINTER(C.c_double),
                                                C.c_double, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                                C.POINTER(C.c_double), i64, i32, C.POINTER(C.c_int32),
                                                C.POINTER(C.c_int32), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                                C.POINTER(C.c_double), C.POINTER(C.c_double), i32]),
            "oracle_mcwf_end_d": (i32, [C.POINTER(RunParams), C.POINTER(CloudParams), C.POINTER(C.c_double),
                                        C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                        C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), i32, i64]),
            "oracle_advance_atoms_d": (i32, [C.POINTER(RunParams), C.POINTER(CloudParams), C.POINTER(C.c_double),
                                             C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int32),
                                             i64, i32]),
            "oracle_step_atoms_d": (i32, [C.POINTER(RunParams), C.POINTER(CloudParams), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                          C.POINTER(C.c_int32), C.POINTER(C.c_int32), i64]),
            "oracle_collide_cell_d": (i32, [C.POINTER(RunParams), C.POINTER(CloudParams), C.POINTER(C.c_double), i32,
                                            C.POINTER(C.c_double), C.c_uint32, C.c_uint32, C.POINTER(C.c_int32),
                                            C.POINTER(C.c_int32), C.POINTER(C.c_double), i32]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _LIB = lib
    return _LIB


def preset(which: int) -> tuple[RunParams, CloudParams]:
    run, cloud = RunParams(), CloudParams()
    if load().oracle_preset(which, C.byref(run), C.byref(cloud)) != 0:
        raise ValueError(f"unknown preset {which}")
    return run, cloud


def philox4x32_10(ctr, key) -> np.ndarray:
    c = (C.c_uint32 * 4)(*[int(x) & 0xFFFFFFFF for x in ctr])
    k = (C.c_uint32 * 2)(*[int(x) & 0xFFFFFFFF for x in key])
    o = (C.c_uint32 * 4)()
    load().oracle_philox(c, k, o)
    return np.array(list(o), np.uint32)


def fixed_point(x: np.ndarray) -> list:
    """The diagnostics' exact fixed-point value floor(min(x, 2^38) * 2^64) of each element (float32
    elements through the float form, float64 through the double form), as Python ints."""
    x = np.ascontiguousarray(x)
    out = np.zeros(2 * x.size, np.uint64)
    prec = 0 if x.dtype == np.float32 else 1
    load().oracle_fx(prec, x.ctypes.data, out.ctypes.data_as(C.POINTER(C.c_uint64)), x.size)
    vals = []
    for lo, hi in zip(out[0::2], out[1::2]):
        v = int(lo) | (int(hi) << 64)
        vals.append(v - (1 << 128) if v >> 127 else v)
    return vals


def math(which: str, x: np.ndarray) -> np.ndarray:
    code = {"sin": 0, "cos": 1, "log": 2, "exp": 3, "rsqrt": 4}[which]
    x = np.ascontiguousarray(x)
    y = np.empty_like(x)
    if x.dtype == np.float32:
        load().oracle_math_f(code, x.ctypes.data_as(C.POINTER(C.c_float)), y.ctypes.data_as(C.POINTER(C.c_float)), x.size)
    else:
        x = x.astype(np.float64)
        y = np.empty_like(x)
        load().oracle_math_d(code, x.ctypes.data_as(C.POINTER(C.c_double)), y.ctypes.data_as(C.POINTER(C.c_double)), x.size)
    return y


def field(run: RunParams, cloud: CloudParams, xyz: np.ndarray) -> np.ndarray:
    xyz = np.ascontiguousarray(xyz, np.float64)
    out = np.empty((xyz.shape[0], 7), np.float64)
    load().oracle_field_d(C.byref(run), C.byref(cloud), xyz.ctypes.data_as(C.POINTER(C.c_double)),
                          out.ctypes.data_as(C.POINTER(C.c_double)), xyz.shape[0])
    return out


def mcwf_end(run: RunParams, cloud: CloudParams, pos, vel, psi, x0, flags, ids, step: int):
    """The MCWF period end (spin flip, decoherence, renormalisation) of each atom, FP64: pos/vel
    (n, 3), psi (n, 4), x0 the trapped population at the period start, flags bit 0 anti-trapped.
    Returns (vel, psi, flags) after the period end."""
    pos = np.ascontiguousarray(pos, np.float64); vel = np.array(vel, np.float64, order="C")
    psi = np.array(psi, np.float64, order="C"); x0 = np.ascontiguousarray(x0, np.float64)
    fl = np.array(flags, np.uint32, order="C"); ids = np.ascontiguousarray(ids, np.uint32)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    up = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint32))
    load().oracle_mcwf_end_d(C.byref(run), C.byref(cloud), dp(pos), dp(vel), dp(psi), dp(x0), up(fl), up(ids),
                             int(step), pos.shape[0])
    return vel, psi, fl


def advance_atoms(run: RunParams, cloud: CloudParams, pos, vel, psi, nsteps: int):
    """FP64 per-atom advance (Larmor, Verlet, evaporation tests) without collisions or sort."""
    pos = np.array(pos, np.float64, order="C", copy=True)
    vel = np.array(vel, np.float64, order="C", copy=True)
    psi = np.array(psi, np.float64, order="C", copy=True)
    fate = np.zeros(pos.shape[0], np.int32)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    load().oracle_advance_atoms_d(C.byref(run), C.byref(cloud), dp(pos), dp(vel), dp(psi),
                                  fate.ctypes.data_as(C.POINTER(C.c_int32)), pos.shape[0], int(nsteps))
    return pos, vel, psi, fate


def step_atoms(run: RunParams, cloud: CloudParams, pos, vel, psi, cut_v2: float):
    """One FP64 timestep of each atom (Larmor, Verlet, Majorana and knife tests with the cut
    cut_v2 = 2 eta kB T / m, new cell) without collisions or sort: pos/vel/psi (n, 4), the fourth
    lane of vel the flag bits.  Returns (pos, vel, psi, fate, cell)."""
    pos = np.array(pos, np.float64, order="C", copy=True)
    vel = np.array(vel, np.float64, order="C", copy=True)
    psi = np.array(psi, np.float64, order="C", copy=True)
    n = pos.shape[0]
    fate = np.zeros(n, np.int32)
    cell = np.zeros(n, np.int32)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    load().oracle_step_atoms_d(C.byref(run), C.byref(cloud), dp(pos), dp(vel), dp(psi), float(cut_v2), ip(fate),
                               ip(cell), n)
    return pos, vel, psi, fate, cell


def collide_cell(run: RunParams, cloud: CloudParams, vel, sigvrmax: float, local_cell: int, step: int):
    """The NTC collisions of one grid cell in FP64: vel (n, 3) of the cell's atoms in sorted order.
    Returns (vel, sigvrmax, candidates, pairs (k, 2), directions (k, 3)) after the cell's candidates."""
    vel = np.asarray(vel, np.float64)
    n = vel.shape[0]
    v4 = np.zeros((n, 4), np.float64)
    v4[:, :3] = vel
    sv = C.c_double(float(sigvrmax))
    cand = C.c_int32(0)
    cap = 4096
    ij = np.zeros((cap, 2), np.int32)
    nv = np.zeros((cap, 3), np.float64)
    acc = load().oracle_collide_cell_d(C.byref(run), C.byref(cloud), v4.ctypes.data_as(C.POINTER(C.c_double)), n,
                                       C.byref(sv), int(local_cell), int(step), C.byref(cand),
                                       ij.ctypes.data_as(C.POINTER(C.c_int32)),
                                       nv.ctypes.data_as(C.POINTER(C.c_double)), cap)
    k = min(acc, cap)
    return v4[:, :3].copy(), sv.value, cand.value, ij[:k].copy(), nv[:k].copy()


def smooth_loss(run, cloud, theta, width_kT, x, v, psi, steps, log_off, log_ij, log_n, grad=False, fp64=True,
                majorana_width=0.05):
    """Smoothed loss of the recorded run (mean energy term + retained fraction).

    Returns (loss, parts) -- parts = (L_E, L_N) -- and with grad=True also (grad_E, grad_N), the
    gradients of each part w.r.t. (B', B0, knots)."""
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    theta = np.ascontiguousarray(theta, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    v = np.ascontiguousarray(v, np.float64)
    psi = np.ascontiguousarray(psi, np.float64)
    off = np.ascontiguousarray(log_off, np.int32)
    ij = np.ascontiguousarray(log_ij, np.int32)
    ln = np.ascontiguousarray(log_n, np.float64)
    parts = np.zeros(2, np.float64)
    ge = np.zeros(11, np.float64)
    gn = np.zeros(11, np.float64)
    loss = load().oracle_smooth_loss(C.byref(run), C.byref(cloud), dp(theta), float(width_kT), float(majorana_width),
                                     dp(x), dp(v), dp(psi), x.shape[0], int(steps), ip(off), ip(ij), dp(ln), dp(parts),
                                     dp(ge) if grad else None, dp(gn) if grad else None, 1 if fp64 else 0)
    if grad:
        return loss, parts, ge, gn
    return loss, parts


def max_threads() -> int:
    return int(load().oracle_max_threads())


def set_threads(n: int) -> None:
    load().oracle_set_threads(int(n))


class Oracle:
    """CPU restatement with the Simulation interface. fast=True selects the OpenMP path."""

    def __init__(self, run: RunParams, clouds: CloudParams | Sequence[CloudParams], fast: bool = False):
        self.lib = load()
        if isinstance(clouds, CloudParams):
            clouds = [clouds]
        self.run = run.copy()
        self.clouds = [c.copy() for c in clouds]
        arr = (CloudParams * len(self.clouds))(*self.clouds)
        h = C.c_void_p()
        if self.lib.oracle_create(C.byref(self.run), arr, len(self.clouds), 1 if fast else 0, C.byref(h)) != 0:
            raise ValueError(self.lib.oracle_last_error(None).decode())
        self._h = h
        self.dtype = np.float32 if run.precision == FP32 else np.float64

    def close(self):
        if getattr(self, "_h", None):
            self.lib.oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            raise RuntimeError(self.lib.oracle_last_error(self._h).decode())

    def init_cloud(self, seed: int | None = None):
        self._check(self.lib.oracle_init(self._h, int(self.run.seed if seed is None else seed)))

    def step(self, n: int = 1):
        self._check(self.lib.oracle_step(self._h, int(n)))

    def synchronize(self):
        """The CPU steps complete before step() returns: nothing to wait for."""

    def diagnostics(self, cloud: int = -1) -> dict:
        d = Diag()
        self._check(self.lib.oracle_diag(self._h, int(cloud), C.byref(d)))
        return d.as_dict()

    def get_state(self) -> dict:
        cap = int(sum(max(c.capacity, c.n_atoms) for c in self.clouds))
        cap = max(cap, 1)
        pos = np.empty((cap, 4), self.dtype)
        vel = np.empty((cap, 4), self.dtype)
        psi = np.empty((cap, 4), self.dtype)
        counts = np.zeros(len(self.clouds), np.int64)
        b = StateBuffers(pos.ctypes.data, vel.ctypes.data, psi.ctypes.data, cap,
                         counts.ctypes.data_as(C.POINTER(C.c_int64)))
        self._check(self.lib.oracle_get_state(self._h, C.byref(b)))
        n = int(b.n)
        return {"pos": pos[:n], "vel": vel[:n], "psi": psi[:n], "cloud_counts": counts}

    def set_state(self, pos, vel, psi, cloud_counts):
        pos = np.ascontiguousarray(pos, self.dtype)
        vel = np.ascontiguousarray(vel, self.dtype)
        psi = np.ascontiguousarray(psi, self.dtype)
        counts = np.ascontiguousarray(np.asarray(cloud_counts, np.int64))
        b = StateBuffers(pos.ctypes.data, vel.ctypes.data, psi.ctypes.data, pos.shape[0],
                         counts.ctypes.data_as(C.POINTER(C.c_int64)))
        self._check(self.lib.oracle_set_state(self._h, C.byref(b)))

    def set_recording(self, flags: int) -> None:
        self._check(self.lib.oracle_set_recording(self._h, int(flags)))

    def evaporated(self, cloud: int = 0) -> dict:
        c = self.clouds[cloud]
        n = int(c.capacity if c.capacity > 0 else c.n_atoms)
        pos, vel = np.zeros((max(n, 1), 3)), np.zeros((max(n, 1), 3))
        step, fate = np.zeros(max(n, 1), np.int32), np.zeros(max(n, 1), np.int32)
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        self._check(self.lib.oracle_get_evaporated(self._h, int(cloud), dp(pos), dp(vel), ip(step), ip(fate),
                                                   max(n, 1)))
        return {"pos": pos[:n], "vel": vel[:n], "step": step[:n], "fate": fate[:n]}

    def cell_collisions(self) -> np.ndarray:
        total = C.c_int64()
        self._check(self.lib.oracle_get_cell_starts(self._h, None, 0, C.byref(total)))
        out = np.zeros(max(total.value, 1), np.int32)
        self._check(self.lib.oracle_get_cell_collisions(self._h, out.ctypes.data_as(C.POINTER(C.c_int32)), out.size))
        return out[:total.value]

    def cell_starts(self) -> np.ndarray:
        total = C.c_int64()
        self._check(self.lib.oracle_get_cell_starts(self._h, None, 0, C.byref(total)))
        out = np.empty(total.value + 1, np.int32)
        self._check(self.lib.oracle_get_cell_starts(self._h, out.ctypes.data_as(C.POINTER(C.c_int32)), out.size,
                                                    C.byref(total)))
        return out

    def sigvrmax(self) -> np.ndarray:
        total = C.c_int64()
        self._check(self.lib.oracle_get_cell_starts(self._h, None, 0, C.byref(total)))
        out = np.empty(total.value, self.dtype)
        self._check(self.lib.oracle_get_sigvrmax(self._h, out.ctypes.data, out.size))
        return out

    def set_sigvrmax(self, values):
        v = np.ascontiguousarray(values, self.dtype)
        self._check(self.lib.oracle_set_sigvrmax(self._h, v.ctypes.data, v.size))

"""ctypes mirror of include/dsmc.h (structs, enums, flags)."""
from __future__ import annotations

import ctypes as C

DSMC_OK = 0
STATUS_NAMES = {
    0: "DSMC_OK", 1: "DSMC_ERR_INVALID", 2: "DSMC_ERR_CUDA", 3: "DSMC_ERR_ALLOC",
    4: "DSMC_ERR_CAPACITY", 5: "DSMC_ERR_CELL_FULL", 6: "DSMC_ERR_NAN", 7: "DSMC_ERR_STATE",
    8: "DSMC_ERR_UNSUPPORTED", 9: "DSMC_ERR_TIMEOUT",
}

FP32, FP64 = 0, 1
TRAP_QUADRUPOLE, TRAP_IOFFE_PRITCHARD, TRAP_BOX = 0, 1, 2
F_COLLIDE, F_LARMOR, F_MAJORANA, F_KNIFE, F_NORMALISE, F_KNIFE_FIXED_T, F_MCWF = 1, 2, 4, 8, 16, 32, 64
INIT_THERMAL, INIT_UNIFORM = 0, 1
REC_EVAPORATED, REC_CELL_COLLISIONS = 1, 2  # dsmc_set_recording
MAX_KNOTS = 9

# named workloads (dsmc_preset)
PRESET_SMALL_FP64 = 0
PRESET_BOX = 1
PRESET_TRAPPED_1E7 = 2
PRESET_ADJOINT = 4


class CloudParams(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int64),
        ("capacity", C.c_int64),
        ("trap", C.c_int32),
        ("flags", C.c_int32),
        ("cells", C.c_int32 * 3),
        ("init_mode", C.c_int32),
        ("grid_min", C.c_double * 3),
        ("grid_max", C.c_double * 3),
        ("mass", C.c_double),
        ("moment", C.c_double),
        ("B0", C.c_double),
        ("dBdz", C.c_double),
        ("d2Bdz2", C.c_double),
        ("temperature", C.c_double),
        ("alpha", C.c_double),
        ("sigma", C.c_double),
        ("sigvrmax_init", C.c_double),
        ("knife_nknots", C.c_int32),
        ("stream_id", C.c_int32),
        ("knife_step", C.c_double * MAX_KNOTS),
        ("knife_eta", C.c_double * MAX_KNOTS),
    ]

    def copy(self) -> "CloudParams":
        c = CloudParams()
        C.memmove(C.byref(c), C.byref(self), C.sizeof(CloudParams))
        return c


class RunParams(C.Structure):
    _fields_ = [
        ("precision", C.c_int32),
        ("collide_every", C.c_int32),
        ("dt", C.c_double),
        ("hbar", C.c_double),
        ("kB", C.c_double),
        ("seed", C.c_uint64),
        ("tile_atoms", C.c_int32),
        ("use_graphs", C.c_int32),
        ("step_blocks_per_sm", C.c_int32),
        ("reserved0", C.c_int32),
    ]

    def copy(self) -> "RunParams":
        r = RunParams()
        C.memmove(C.byref(r), C.byref(self), C.sizeof(RunParams))
        return r


class Diag(C.Structure):
    _fields_ = [
        ("step", C.c_int64),
        ("time", C.c_double),
        ("n_alive", C.c_int64),
        ("e_kin", C.c_double),
        ("e_pot", C.c_double),
        ("temperature", C.c_double),
        ("sum_v2", C.c_double),
        ("sum_absB", C.c_double),
        ("n_evaporated", C.c_int64),
        ("n_majorana", C.c_int64),
        ("n_knife", C.c_int64),
        ("e_evaporated", C.c_double),
        ("collisions", C.c_int64),
        ("candidates", C.c_int64),
        ("atom_steps", C.c_int64),
        ("error", C.c_int32),
        ("reserved0", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if not name.startswith("reserved")}


class StateBuffers(C.Structure):
    _fields_ = [
        ("pos", C.c_void_p),
        ("vel", C.c_void_p),
        ("psi", C.c_void_p),
        ("n", C.c_int64),
        ("cloud_counts", C.POINTER(C.c_int64)),
    ]


class AdjParams(C.Structure):
    _fields_ = [
        ("steps", C.c_int32),
        ("checkpoint_every", C.c_int32),
        ("precision", C.c_int32),
        ("reserved0", C.c_int32),
        ("sigmoid_width_kT", C.c_double),
        ("majorana_width", C.c_double),
    ]


class Grad(C.Structure):
    _fields_ = [
        ("loss", C.c_double),
        ("mean_energy_kT", C.c_double),
        ("retained_fraction", C.c_double),
        ("dL_dBp", C.c_double),
        ("dL_dB0", C.c_double),
        ("dL_deta", C.c_double * 9),
        ("collisions", C.c_int64),
        ("ms_record", C.c_double),
        ("ms_forward", C.c_double),
        ("ms_backward", C.c_double),
        ("dE_dtheta", C.c_double * 11),
        ("dN_dtheta", C.c_double * 11),
    ]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["dL_deta"] = list(self.dL_deta)
        d["dE_dtheta"] = list(self.dE_dtheta)
        d["dN_dtheta"] = list(self.dN_dtheta)
        return d

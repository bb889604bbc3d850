"""B200-native DSMC engine for trapped ultracold atoms (the CUDADSMC timestep on sm_100a).

    from cudadsmc_b200 import Simulation, preset
    run, cloud = preset(2)            # 1e7 atoms, 128^3 cells, Larmor + Majorana + knife
    sim = Simulation(run, cloud)
    sim.init_cloud(1234)
    sim.step(100)
    print(sim.diagnostics())
"""
from ._abi import (CloudParams, Diag, RunParams, StateBuffers, FP32, FP64, TRAP_QUADRUPOLE,
                   TRAP_IOFFE_PRITCHARD, TRAP_BOX, F_COLLIDE, F_LARMOR, F_MAJORANA, F_KNIFE,
                   F_NORMALISE, F_KNIFE_FIXED_T, F_MCWF, INIT_THERMAL, INIT_UNIFORM)
from .engine import DSMCError, Simulation, load_library, preset, EXPORTED_SYMBOLS

__all__ = [
    "CloudParams", "Diag", "RunParams", "StateBuffers", "Simulation", "DSMCError", "load_library",
    "preset", "EXPORTED_SYMBOLS", "FP32", "FP64", "TRAP_QUADRUPOLE", "TRAP_IOFFE_PRITCHARD",
    "TRAP_BOX", "F_COLLIDE", "F_LARMOR", "F_MAJORANA", "F_KNIFE", "F_NORMALISE", "F_KNIFE_FIXED_T", "F_MCWF",
    "INIT_THERMAL", "INIT_UNIFORM",
]

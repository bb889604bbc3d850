"""The C ABI without a GPU: the library loads, exports every symbol include/dsmc.h declares,
its structs have the layout ctypes assumes, presets work and compute entry points fail
loudly (no CPU fallback) when no device is present."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

import cudadsmc_b200 as dsmc
from cudadsmc_b200 import _abi, engine
from conftest import HAS_GPU, ROOT

HEADER = os.path.join(ROOT, "include", "dsmc.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"DSMC_API\s+[\w\s\*]+?\b(dsmc_\w+)\s*\(", text)))


def test_header_declarations_match_binding():
    assert declared_symbols() == sorted(engine.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol():
    lib = dsmc.load_library()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", engine.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (dsmc_\w+)", out))
    assert set(declared_symbols()) <= exported
    # nothing but the ABI is exported under the dsmc_ prefix
    assert exported == set(declared_symbols())


def test_struct_layout_matches_c_compiler():
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "dsmc.h"
#define P(T, f) printf(#T "." #f " %zu\n", offsetof(T, f))
int main(void) {
  printf("dsmc_cloud_params %zu\n", sizeof(dsmc_cloud_params));
  printf("dsmc_params %zu\n", sizeof(dsmc_params));
  printf("dsmc_diag %zu\n", sizeof(dsmc_diag));
  printf("dsmc_state_buffers %zu\n", sizeof(dsmc_state_buffers));
  P(dsmc_cloud_params, grid_min); P(dsmc_cloud_params, knife_step); P(dsmc_cloud_params, stream_id);
  P(dsmc_cloud_params, knife_eta); P(dsmc_params, seed); P(dsmc_params, use_graphs);
  P(dsmc_diag, atom_steps); P(dsmc_diag, error); P(dsmc_state_buffers, cloud_counts);
  return 0;
}'''
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(src, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        lines = dict(l.rsplit(" ", 1) for l in subprocess.run([exe], capture_output=True, text=True).stdout.split("\n") if l)
    assert int(lines["dsmc_cloud_params"]) == C.sizeof(_abi.CloudParams)
    assert int(lines["dsmc_params"]) == C.sizeof(_abi.RunParams)
    assert int(lines["dsmc_diag"]) == C.sizeof(_abi.Diag)
    assert int(lines["dsmc_state_buffers"]) == C.sizeof(_abi.StateBuffers)
    for key, val in lines.items():
        if "." in key:
            struct, field = key.split(".")
            cls = {"dsmc_cloud_params": _abi.CloudParams, "dsmc_params": _abi.RunParams, "dsmc_diag": _abi.Diag,
                   "dsmc_state_buffers": _abi.StateBuffers}[struct]
            assert getattr(cls, field).offset == int(val), key


def test_presets():
    run, c = dsmc.preset(2)
    assert c.n_atoms == 10_000_000 and tuple(c.cells) == (128, 128, 128)
    assert run.precision == dsmc.FP32 and run.dt == 1e-6
    assert c.flags & dsmc.F_KNIFE and c.knife_eta[0] == 6.0 and c.knife_eta[1] == 4.0
    run0, c0 = dsmc.preset(0)
    assert run0.precision == dsmc.FP64 and c0.n_atoms == 10000 and c0.alpha == 300.0
    run1, c1 = dsmc.preset(1)
    assert c1.trap == dsmc.TRAP_BOX and c1.alpha == 1e4
    with pytest.raises(dsmc.DSMCError):
        dsmc.preset(3)


def test_status_strings():
    lib = dsmc.load_library()
    assert lib.dsmc_abi_version() == 2
    assert lib.dsmc_status_string(5) == b"tile too full to stage"


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device failure path")
def test_create_without_gpu_fails_loudly():
    run, c = dsmc.preset(0)
    with pytest.raises(dsmc.DSMCError) as e:
        dsmc.Simulation(run, c)
    assert e.value.status == 2  # DSMC_ERR_CUDA: there is no CPU fallback


def test_invalid_parameters_rejected():
    lib = dsmc.load_library()
    run, c = dsmc.preset(0)
    c.temperature = -1
    h = C.c_void_p()
    st = lib.dsmc_create(C.byref(run), C.byref(c), 1, C.byref(h))
    assert st in (1, 2)  # invalid (checked first when a device exists) or no device
    assert lib.dsmc_create(None, None, 0, C.byref(h)) == 1
    assert lib.dsmc_step(None, 1) == 1

"""Primitives on the GPU: the engine's Philox4x32-10 against cuRAND's Philox4_32_10, and the
series-based elementary functions against the CUDA math library's error bounds."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT

pytestmark = pytest.mark.gpu

SRC = os.path.join(ROOT, "tests", "gpu_helpers", "curand_philox.cu")
LIB = os.path.join(ROOT, "tests", "gpu_helpers", "libcurand_check.so")


@pytest.fixture(scope="module")
def helper():
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-Xcompiler", "-fPIC",
                        "-shared", "-o", LIB, SRC], check=True)
    lib = C.CDLL(LIB)
    lib.curand_philox.argtypes = [C.c_ulonglong, C.POINTER(C.c_ulonglong), C.POINTER(C.c_uint), C.c_int, C.c_int]
    lib.cuda_math.argtypes = [C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int]
    return lib


def test_philox_matches_curand(helper):
    # cuRAND's Philox4_32_10 with (seed, subsequence s, offset 0): output block k is
    # Philox(counter = (k, 0, s_lo, s_hi), key = (seed_lo, seed_hi))
    seed = 0x0123456789ABCDEF
    subs = np.array([0, 1, 7, 12345, 2 ** 32 + 5, 2 ** 40 + 99], np.uint64)
    per = 4
    out = np.zeros((subs.size, per, 4), np.uint32)
    assert helper.curand_philox(seed, subs.ctypes.data_as(C.POINTER(C.c_ulonglong)),
                                out.ctypes.data_as(C.POINTER(C.c_uint)), subs.size, per) == 0
    for i, s in enumerate(subs):
        for k in range(per):
            mine = oracle.philox4x32_10([k, 0, int(s) & 0xFFFFFFFF, int(s) >> 32],
                                        [seed & 0xFFFFFFFF, seed >> 32])
            assert np.array_equal(mine, out[i, k]), (i, k, mine, out[i, k])


@pytest.mark.parametrize("fn", ["sin", "cos", "log", "exp"])
def test_series_functions_within_cuda_math_error(helper, fn):
    rng = np.random.default_rng(4)
    if fn in ("sin", "cos"):
        x = rng.uniform(-500, 500, 100000).astype(np.float32)
        ref = np.sin if fn == "sin" else np.cos
    elif fn == "log":
        x = rng.uniform(1e-7, 1, 100000).astype(np.float32)
        ref = np.log
    else:
        x = rng.uniform(-80, 80, 100000).astype(np.float32)
        ref = np.exp
    code = {"sin": 0, "cos": 1, "log": 2, "exp": 3}[fn]
    y = np.zeros_like(x)
    assert helper.cuda_math(code, x.ctypes.data_as(C.POINTER(C.c_float)), y.ctypes.data_as(C.POINTER(C.c_float)), x.size) == 0
    exact = ref(x.astype(np.float64))
    ours = oracle.math(fn, x).astype(np.float64)
    scale = np.maximum(np.abs(exact), 1.0) if fn in ("sin", "cos") else np.abs(exact)
    err_ours = np.max(np.abs(ours - exact) / scale)
    err_cuda = np.max(np.abs(y.astype(np.float64) - exact) / scale)
    assert err_ours <= 2.5 * max(err_cuda, 6e-8), (err_ours, err_cuda)

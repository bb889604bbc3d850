"""Arithmetic primitives shared by the engine and the oracle (CPU only): elementary functions
written from their series, Philox stream keying, uniforms, exact fixed-point sums, trap fields."""
import math

import numpy as np
import pytest

import oracle
from cudadsmc_b200._abi import FP64, TRAP_IOFFE_PRITCHARD, TRAP_QUADRUPOLE


def ulps(a, b, dtype):
    a = np.asarray(a, dtype); b = np.asarray(b, np.float64)
    spacing = np.spacing(np.abs(b).astype(dtype)).astype(np.float64)
    return np.abs(a.astype(np.float64) - b) / spacing


@pytest.mark.parametrize("fn,ref", [("sin", np.sin), ("cos", np.cos)])
def test_sincos_accuracy(fn, ref):
    x32 = np.concatenate([np.linspace(-30, 30, 300001), np.linspace(-2000, 2000, 100001)]).astype(np.float32)
    y = oracle.math(fn, x32)
    assert np.max(np.abs(y - ref(x32.astype(np.float64)))) < 2.5e-7  # ~2 ulp at |y| ~ 1
    x64 = np.linspace(-3000, 3000, 300001)
    assert np.max(np.abs(oracle.math(fn, x64) - ref(x64))) < 4e-16


def test_log_exp_accuracy():
    rng = np.random.default_rng(0)
    u32 = rng.uniform(2 ** -24, 1, 200000).astype(np.float32)
    assert np.max(ulps(oracle.math("log", u32), np.log(u32.astype(np.float64)), np.float32)) <= 3
    u64 = rng.uniform(2 ** -53, 1, 200000)
    assert np.max(ulps(oracle.math("log", u64), np.log(u64), np.float64)) <= 3
    e32 = rng.uniform(-80, 80, 200000).astype(np.float32)
    assert np.max(ulps(oracle.math("exp", e32), np.exp(e32.astype(np.float64)), np.float32)) <= 3
    e64 = rng.uniform(-700, 700, 200000)
    assert np.max(ulps(oracle.math("exp", e64), np.exp(e64), np.float64)) <= 3
    assert oracle.math("exp", np.array([-100.0], np.float32))[0] == 0.0


def test_rsqrt_accuracy():
    rng = np.random.default_rng(3)
    x32 = np.exp(rng.uniform(-80, 80, 200000)).astype(np.float32)
    x32 = x32[np.isfinite(x32) & (x32 > np.finfo(np.float32).tiny)]
    assert np.max(ulps(oracle.math("rsqrt", x32), 1 / np.sqrt(x32.astype(np.float64)), np.float32)) <= 3
    x64 = np.exp(rng.uniform(-600, 600, 200000))
    assert np.max(ulps(oracle.math("rsqrt", x64), 1 / np.sqrt(x64), np.float64)) <= 3


def test_philox_keying_and_avalanche():
    a = oracle.philox4x32_10([1, 2, 3, 4], [5, 6])
    assert np.array_equal(a, oracle.philox4x32_10([1, 2, 3, 4], [5, 6]))
    # one flipped counter or key bit changes about half of the 128 output bits
    flips = []
    for word in range(4):
        for bit in (0, 13, 31):
            c = [1, 2, 3, 4]
            c[word] ^= 1 << bit
            b = oracle.philox4x32_10(c, [5, 6])
            flips.append(sum(bin(int(x) ^ int(y)).count("1") for x, y in zip(a, b)))
    assert 50 < np.mean(flips) < 78


def test_philox_uniformity():
    out = np.array([oracle.philox4x32_10([i, 7, 3 << 24, 0], [1234, 0]) for i in range(20000)]).ravel()
    u = ((out >> 8).astype(np.float64) + 0.5) * 2.0 ** -24
    from scipy import stats
    assert stats.kstest(u, "uniform").pvalue > 1e-3


def test_fixed_point_sums_are_order_independent():
    # the diagnostics' 128-bit fixed-point sums: any order gives the same bits
    run, c = oracle.preset(2)
    c.n_atoms = c.capacity = 5000
    c.cells[0] = c.cells[1] = c.cells[2] = 12
    o = oracle.Oracle(run, c)
    o.init_cloud(3)
    d = o.diagnostics()
    st = o.get_state()
    v2 = np.sum(st["vel"][:, :3].astype(np.float32) ** 2, axis=1, dtype=np.float32)
    # recompute float v2 in the same operation order and sum exactly with Python integers
    vx, vy, vz = (st["vel"][:, k].astype(np.float32) for k in range(3))
    v2 = (vx * vx + vy * vy).astype(np.float32) + (vz * vz).astype(np.float32)
    exact = sum(int(math.floor(float(x) * 2.0 ** 64)) for x in v2.astype(np.float64))
    perm = np.random.default_rng(1).permutation(v2.size)
    exact_perm = sum(int(math.floor(float(x) * 2.0 ** 64)) for x in v2[perm].astype(np.float64))
    assert exact == exact_perm
    assert abs(exact / 2.0 ** 64 - d["sum_v2"]) <= 1e-15 * d["sum_v2"]


def test_fixed_point_float_and_double_forms_agree():
    # sign(x) floor(min(|x|, 2^38) * 2^64) from the float form equals the double form on the same
    # value, negative values (anti-trapped atoms' -|B|) included
    rng = np.random.default_rng(5)
    pos = np.concatenate([
        np.exp2(rng.uniform(-80, 40, 20000)),            # subnormal-adjacent to beyond the clamp
        rng.uniform(0, 4, 5000),
        [0.0, 2.0 ** -64, 2.0 ** -65, 1.0, 2.0 ** 38, 2.0 ** 38 * 0.999, np.inf, np.nan, 1e-45, 3e38],
    ])
    x = np.concatenate([pos, -pos[:25000], [-0.3, -1.7, -1e-3]]).astype(np.float32)
    f = oracle.fixed_point(x)
    d = oracle.fixed_point(x.astype(np.float64))
    assert f == d
    for xi, v in zip(x[:3000].astype(np.float64), f[:3000]):
        assert v == int(math.floor(min(xi, 2.0 ** 38) * 2.0 ** 64))
    for xi, v in zip(x[25010:28000].astype(np.float64), f[25010:28000]):
        assert v == -int(math.floor(min(-xi, 2.0 ** 38) * 2.0 ** 64))
    assert f[25006] == f[25007] == 2 ** 102  # inf and NaN clamp to 2^38


def field_reference(kind, p, B0, Bp, Bpp):
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    if kind == "quad":
        B = np.stack([Bp * x / 2, Bp * y / 2, B0 - Bp * z], 1)
    else:  # CUDADSMC/src/moveAtoms.cu:137-139
        B = np.stack([Bp * x - 0.5 * Bpp * x * z, -Bp * y - 0.5 * Bpp * y * z,
                      B0 + 0.5 * Bpp * (z * z - 0.5 * (x * x + y * y))], 1)
    return B


@pytest.mark.parametrize("kind", ["quad", "ip"])
def test_trap_field_and_gradient(kind):
    run, c = oracle.preset(0)
    run.precision = FP64
    if kind == "quad":
        c.trap, c.B0, c.dBdz = TRAP_QUADRUPOLE, 1e-4, 2.5
    else:
        c.trap, c.B0, c.dBdz, c.d2Bdz2 = TRAP_IOFFE_PRITCHARD, 0.01, 20.0, 4e4
    rng = np.random.default_rng(2)
    p = rng.uniform(-3e-4, 3e-4, (500, 3))
    f = oracle.field(run, c, p)
    B = field_reference(kind, p, c.B0, c.dBdz, c.d2Bdz2)
    absB = np.linalg.norm(B, axis=1)
    np.testing.assert_allclose(f[:, 3], absB, rtol=1e-13)
    np.testing.assert_allclose(f[:, :3], B / absB[:, None], atol=1e-13)
    # grad |B| by central differences
    h = 1e-9
    for a in range(3):
        dp = np.zeros(3); dp[a] = h
        num = (np.linalg.norm(field_reference(kind, p + dp, c.B0, c.dBdz, c.d2Bdz2), axis=1) -
               np.linalg.norm(field_reference(kind, p - dp, c.B0, c.dBdz, c.d2Bdz2), axis=1)) / (2 * h)
        np.testing.assert_allclose(f[:, 4 + a], num, rtol=1e-5, atol=1e-6 * c.dBdz)

"""The engine's own transcendental functions against the true functions.

The engine and the oracle evaluate log, exp and sin/cos(2 pi t) with their
own series (LogF/ExpF/SinCosTurnF and the double versions in
g4go_b200/csrc/g4b_device.cuh, restated in oracle/cpu_transport.cpp), so the
two agree bit for bit (tests/test_gpu_boundary.py) - which alone would let a
wrong coefficient pass every parity test. Here the oracle's series are held
to the true functions (numpy, float64 or long double) over the arguments the
kernels use, with stated bounds; tests/test_gpu_boundary.py holds the
device's float versions to the same bounds.

  log   uniform draws (w + 0.5) / 2^32, the clamps 1e-7 and 1 - u: <= 2 ulp
  exp   [-87.3, 0] (rise-time acceptance, facet and roughness Gaussians):
        <= 1.5 ulp; below, gradual underflow within 2^-149 of the truth
  sin, cos of 2 pi t, t in [0, 1): <= 2 ulp where |value| > 1e-3, and within
        1.2e-7 absolutely everywhere
  double: log <= 2.5 ulp, exp <= 1.5 ulp, sin/cos within 5e-16 absolutely
"""
import ctypes as C

import numpy as np

FLOAT_DRAWS = 200_000


def ulps32(got, true):
    return np.abs(got.astype(np.float64) - true) / np.spacing(np.abs(true).astype(np.float32)).astype(np.float64)


def ulps64(got, true):
    return np.abs(got.astype(np.longdouble) - true) / np.spacing(np.abs(true).astype(np.float64)).astype(np.longdouble)


def log_arguments(rng):
    words = rng.integers(0, 2**32, FLOAT_DRAWS, dtype=np.uint64)
    draws = (words.astype(np.float32) + np.float32(0.5)) / np.float32(4294967296.0)
    edges = np.float32([2.0**-33, 1e-7, 2.0**-24, 0.5, 0.75, 1 - 2.0**-24, 1.0])
    return np.concatenate([draws, 1.0 - draws, edges]).astype(np.float32)


def exp_arguments(rng):
    return np.concatenate([-rng.uniform(0, 1, FLOAT_DRAWS // 2), -rng.uniform(0, 110, FLOAT_DRAWS // 2),
                           [0.0, -1e-8, -87.3, -103.0, -104.5, -200.0]]).astype(np.float32)


def turn_arguments(rng):
    return np.concatenate([rng.random(FLOAT_DRAWS), [0.0, 0.125, 0.25, 0.5, 0.75, 1 - 2.0**-24, 2.0**-24]]).astype(
        np.float32)


def check_log(x, got):
    assert np.max(ulps32(got, np.log(x.astype(np.float64)))) <= 2.0


def check_exp(x, got):
    true = np.exp(x.astype(np.float64))
    normal = true >= np.finfo(np.float32).tiny
    assert np.max(ulps32(got[normal], true[normal])) <= 1.5
    assert np.max(np.abs(got[~normal].astype(np.float64) - true[~normal])) <= 2.0**-149


def check_sincos(t, s, c):
    angle = 2.0 * np.pi * t.astype(np.float64)
    for got, true in ((s, np.sin(angle)), (c, np.cos(angle))):
        assert np.max(np.abs(got.astype(np.float64) - true)) <= 1.2e-7
        away = np.abs(true) > 1e-3
        assert np.max(ulps32(got[away], true[away])) <= 2.0


def test_float_series_against_the_true_functions(oracle):
    lib = oracle.load()
    rng = np.random.default_rng(7)
    x = log_arguments(rng)
    check_log(x, np.array([lib.oracle_log_f(float(v)) for v in x], np.float32))
    x = exp_arguments(rng)
    check_exp(x, np.array([lib.oracle_exp_f(float(v)) for v in x], np.float32))
    t = turn_arguments(rng)
    s = np.empty_like(t)
    c = np.empty_like(t)
    a, b = C.c_float(), C.c_float()
    for i, v in enumerate(t):
        lib.oracle_sincos_turn_f(float(v), C.byref(a), C.byref(b))
        s[i], c[i] = a.value, b.value
    check_sincos(t, s, c)


def test_double_series_against_the_true_functions(oracle):
    lib = oracle.load()
    rng = np.random.default_rng(8)
    x = np.concatenate([rng.random(50_000), [2.0**-60, 1e-300, 0.5, 1.0]])
    got = np.array([lib.oracle_log_d(float(v)) for v in x])
    assert np.max(ulps64(got, np.log(x.astype(np.longdouble)))) <= 2.5
    x = np.concatenate([-rng.uniform(0, 100, 50_000), [0.0, -700.0]])
    got = np.array([lib.oracle_exp_d(float(v)) for v in x])
    assert np.max(ulps64(got, np.exp(x.astype(np.longdouble)))) <= 1.5
    t = rng.random(50_000)
    a, b = C.c_double(), C.c_double()
    s, c = np.empty_like(t), np.empty_like(t)
    for i, v in enumerate(t):
        lib.oracle_sincos_turn_d(float(v), C.byref(a), C.byref(b))
        s[i], c[i] = a.value, b.value
    angle = 2 * np.pi * t.astype(np.longdouble)
    assert float(np.max(np.abs(s - np.sin(angle)))) <= 5e-16
    assert float(np.max(np.abs(c - np.cos(angle)))) <= 5e-16

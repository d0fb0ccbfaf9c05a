"""The engine's device functions, run on the GPU through the C ABI.

Boundary physics against the reference's own outputs (golden vectors made by
tests/golden/make_golden.py from the reference's OptiXBoundaryPhysics.cuh)
and the reference's known-answer tests, within 1e-5 relative (the agreement
with the Geant4 formulas that is required); the device math and RNG bit for bit
against the CPU oracle.
"""
import ctypes as C
import math

import numpy as np
import pytest

from g4go_b200 import eval_fresnel, eval_lambertian, eval_math, eval_uniform

from test_oracle_boundary import GOLDEN, _fresnel_golden_check

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_device_fresnel_known_answers(precision):
    """TestOpticalBoundaryPhysics.cxx:37-69 evaluated by the transport kernel's ComputeFresnel."""
    angle_b = math.atan(1.5)
    d_b = np.array([math.sin(angle_b), 0.0, math.cos(angle_b)])
    p_b = np.cross(d_b, [0.0, 1.0, 0.0])
    p_b /= np.linalg.norm(p_b)
    angle_t = 50.0 * math.pi / 180.0
    out = eval_fresnel(
        [[0, 0, 1], d_b, [math.sin(angle_t), 0, math.cos(angle_t)]],
        [[1, 0, 0], p_b, [0, 1, 0]],
        [[0, 0, -1], [0, 0, -1], [0, 0, -1]],
        [1.0, 1.0, 1.5], [1.5, 1.5, 1.0], precision=precision,
    )
    assert out[0, 13] == 0 and abs(out[0, 12] - 0.96) <= 1e-5
    assert abs(out[0, 2] + 1) <= 1e-6 and abs(out[0, 5] - 1) <= 1e-6
    assert abs(np.dot(out[0, 0:3], out[0, 6:9])) <= 1e-6
    assert abs(out[1, 12] - 1.0) <= 1e-5
    assert out[2, 13] == 1 and abs(out[2, 12]) <= 1e-6 and out[2, 2] < 0
    assert abs(np.dot(out[2, 0:3], out[2, 6:9])) <= 1e-6


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_device_fresnel_matches_reference_golden(precision):
    golden = np.load(GOLDEN)
    out = eval_fresnel(golden["fresnel_direction"], golden["fresnel_polarization"], golden["fresnel_normal"],
                       golden["fresnel_index_from"], golden["fresnel_index_to"], precision=precision)
    _fresnel_golden_check(out, golden, tolerance=1e-5)


def test_device_fresnel_bit_equal_to_oracle(oracle):
    golden = np.load(GOLDEN)
    out = eval_fresnel(golden["fresnel_direction"], golden["fresnel_polarization"], golden["fresnel_normal"],
                       golden["fresnel_index_from"], golden["fresnel_index_to"], precision="fp32")
    lib = oracle.load()
    f3 = C.POINTER(C.c_float)
    for i in range(golden["fresnel_direction"].shape[0]):
        want = np.zeros(14, dtype=np.float32)
        args = [np.ascontiguousarray(golden[k][i]) for k in ("fresnel_direction", "fresnel_polarization", "fresnel_normal")]
        lib.oracle_fresnel_f(*(a.ctypes.data_as(f3) for a in args), float(golden["fresnel_index_from"][i]),
                             float(golden["fresnel_index_to"][i]), want.ctypes.data_as(f3))
        np.testing.assert_array_equal(out[i].astype(np.float32), want)


def test_device_lambertian_matches_reference_golden():
    golden = np.load(GOLDEN)
    out = eval_lambertian(golden["lambertian_normal"], golden["lambertian_radial"], golden["lambertian_azimuth"])
    np.testing.assert_allclose(out, golden["lambertian_out"], atol=2e-6)
    assert np.all(np.sum(out * golden["lambertian_normal"], axis=1) >= -1e-7)


def test_device_math_bit_equal_to_oracle(oracle):
    lib = oracle.load()
    rng = np.random.default_rng(5)
    u = np.concatenate([(rng.integers(0, 2**32, 20000).astype(np.float64) + 0.5) / 2**32,
                        [1e-7, 0.5, 1.0, 2.0, 1e-30, 3.0e38]]).astype(np.float32)
    got = eval_math("log", u)
    want = np.array([lib.oracle_log_f(float(x)) for x in u], dtype=np.float32)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    x = np.concatenate([-rng.random(20000) * 90.0, rng.normal(size=2000) * 10, [0.0, -104.5, 88.0]]).astype(np.float32)
    got = eval_math("exp", x)
    want = np.array([lib.oracle_exp_f(float(v)) for v in x], dtype=np.float32)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    t = np.concatenate([rng.random(20000), [0.0, 0.125, 0.25, 0.5, 0.75, 0.999999]]).astype(np.float32)
    s, c = eval_math("sincos_turn", t)
    ws = np.zeros(1, np.float32)
    wc = np.zeros(1, np.float32)
    f3 = C.POINTER(C.c_float)
    for i, v in enumerate(t):
        lib.oracle_sincos_turn_f(float(v), ws.ctypes.data_as(f3), wc.ctypes.data_as(f3))
        assert s[i].view(np.uint32) == ws[0].view(np.uint32) and c[i].view(np.uint32) == wc[0].view(np.uint32), v


def test_device_uniform_bit_equal_to_oracle(oracle):
    lib = oracle.load()
    rng = np.random.default_rng(9)
    n = 4096
    keys = rng.integers(0, 2**63, n, dtype=np.uint64)
    bounce = rng.integers(0, 4096, n).astype(np.uint32)
    process = rng.choice([0, 1, 2, 3, 4, 5, 10, 20], n).astype(np.uint32)
    draw = rng.integers(0, 2000, n).astype(np.uint32)
    seed = 0x1234_5678_9ABC_DEF0
    got = eval_uniform(seed, keys, bounce, process, draw)
    want = np.array([lib.oracle_uniform_f(seed, int(k), int(b), int(p), int(d))
                     for k, b, p, d in zip(keys, bounce, process, draw)], dtype=np.float32)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    assert np.all((got > 0) & (got <= 1))


def test_device_math_within_the_true_function_bounds():
    """The device's own log / exp / sin+cos of turns (float), evaluated on the
    GPU, against the true functions with the bounds tests/test_math_accuracy.py
    states for the oracle's series."""
    import test_math_accuracy as bounds

    rng = np.random.default_rng(17)
    x = bounds.log_arguments(rng)
    bounds.check_log(x, eval_math("log", x))
    x = bounds.exp_arguments(rng)
    bounds.check_exp(x, eval_math("exp", x))
    t = bounds.turn_arguments(rng)
    s, c = eval_math("sincos_turn", t)
    bounds.check_sincos(t, s, c)


def test_device_uniform_is_the_reference_bit_for_bit():
    """The device's counter RNG against the reference's own Uniform
    (OptiXTransportDevice.cu:254-286, compiled for the host: the fixture of
    tests/golden/make_golden_transport.py)."""
    import reference_fixture as rf

    golden = rf.load()
    for s, seed in enumerate(golden["uniform_seeds"]):
        got = eval_uniform(int(seed), golden["uniform_keys"], golden["uniform_bounce"], golden["uniform_process"],
                           golden["uniform_draw"])
        np.testing.assert_array_equal(got.view(np.uint32), golden["uniform"][s].view(np.uint32))

"""Pins the CPU oracle's boundary physics to the reference.

1. The reference's own known-answer tests (test/TestOpticalBoundaryPhysics.cxx:37-101).
2. The committed golden vectors (tests/golden/boundary_reference.npz), which
   tests/golden/make_golden.py produced by running the reference's
   OptiXBoundaryPhysics.cuh compiled from the reference tree.
3. When the reference tree is present, the compiled reference live on fresh
   random inputs.
"""
import ctypes as C
import math
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "boundary_reference.npz"
F3 = C.POINTER(C.c_float)
D3 = C.POINTER(C.c_double)

SURFACE_INTERACTION, DIRECT_TRANSMIT, ABSORB, DETECT = 3, 2, 0, 1
# The reference's SurfaceOutcome enum order (OptiXBoundaryPhysics.cuh:15-20).
REFERENCE_OUTCOME = {0: ABSORB, 1: DETECT, 2: DIRECT_TRANSMIT, 3: SURFACE_INTERACTION}


def fresnel_f(oracle, d, p, n, n1, n2):
    lib = oracle.load()
    out = np.zeros(14, dtype=np.float32)
    args = [np.ascontiguousarray(x, dtype=np.float32) for x in (d, p, n)]
    lib.oracle_fresnel_f(*(a.ctypes.data_as(F3) for a in args), float(n1), float(n2), out.ctypes.data_as(F3))
    return out


def fresnel_d(oracle, d, p, n, n1, n2):
    lib = oracle.load()
    out = np.zeros(14, dtype=np.float64)
    args = [np.ascontiguousarray(x, dtype=np.float64) for x in (d, p, n)]
    lib.oracle_fresnel_d(*(a.ctypes.data_as(D3) for a in args), float(n1), float(n2), out.ctypes.data_as(D3))
    return out


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_reference_known_answers(oracle, precision):
    """TestOpticalBoundaryPhysics.cxx:37-69 on the oracle."""
    f = fresnel_f if precision == "fp32" else fresnel_d
    out = f(oracle, [0, 0, 1], [1, 0, 0], [0, 0, -1], 1.0, 1.5)
    assert out[13] == 0
    assert abs(out[12] - 0.96) <= 1e-5
    assert abs(out[2] + 1.0) <= 1e-6
    assert abs(out[5] - 1.0) <= 1e-6
    assert abs(np.dot(out[0:3], out[6:9])) <= 1e-6

    angle = math.atan(1.5)
    d = np.array([math.sin(angle), 0.0, math.cos(angle)])
    p = np.cross(d, [0.0, 1.0, 0.0])
    p /= np.linalg.norm(p)
    out = f(oracle, d, p, [0, 0, -1], 1.0, 1.5)
    assert abs(out[12] - 1.0) <= 1e-5

    angle = 50.0 * math.pi / 180.0
    out = f(oracle, [math.sin(angle), 0, math.cos(angle)], [0, 1, 0], [0, 0, -1], 1.5, 1.0)
    assert out[13] == 1
    assert abs(out[12]) <= 1e-6
    assert out[2] < 0
    assert abs(np.dot(out[0:3], out[6:9])) <= 1e-6


def test_reference_known_answers_surface(oracle):
    """TestOpticalBoundaryPhysics.cxx:71-101 on the oracle."""
    lib = oracle.load()
    assert lib.oracle_classify_surface(0.8, 0.1, 1, 1, 0.05) == SURFACE_INTERACTION
    assert lib.oracle_classify_surface(0.8, 0.1, 1, 1, 0.75) == SURFACE_INTERACTION
    assert lib.oracle_classify_surface(0.8, 0.1, 1, 1, 0.85) == DIRECT_TRANSMIT
    assert lib.oracle_classify_surface(0.8, 0.1, 1, 1, 0.95) == ABSORB
    assert lib.oracle_classify_surface(0.0, 0.0, 0, 0, 0.5) == SURFACE_INTERACTION
    assert lib.oracle_classify_surface(0.0, 0.4, 0, 1, 0.2) == DIRECT_TRANSMIT
    assert lib.oracle_evaluate_absorption(0.3, 1, 0.2) == DETECT
    assert lib.oracle_evaluate_absorption(0.3, 1, 0.5) == ABSORB
    normal = np.array([0, 0, 1], dtype=np.float32)
    out = np.zeros(3, dtype=np.float32)
    lib.oracle_lambertian_f(normal.ctypes.data_as(F3), 0.75, 0.25, out.ctypes.data_as(F3))
    assert np.dot(out, normal) >= 0.0
    assert abs(np.dot(out, out) - 1.0) <= 1e-6


def exact_fresnel(golden):
    """Textbook polarised Fresnel in FP64 from the golden inputs: transmittance
    T = 1 - (E_s^2 r_s^2 + E_p^2 r_p^2) and the TIR flag, independent of both
    the reference and the engine."""
    d = golden["fresnel_direction"].astype(np.float64)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    n = golden["fresnel_normal"].astype(np.float64)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    p = golden["fresnel_polarization"].astype(np.float64)
    p = p - np.sum(p * d, axis=1, keepdims=True) * d
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    n1 = golden["fresnel_index_from"].astype(np.float64)
    n2 = golden["fresnel_index_to"].astype(np.float64)
    cos_i = np.clip(-np.sum(d * n, axis=1), 0, 1)
    s2 = (n1 / n2) ** 2 * (1 - cos_i**2)
    tir = s2 >= 1.0
    cos_t = np.sqrt(np.maximum(0.0, 1.0 - s2))
    s_dir = np.cross(d, n)
    s_len = np.linalg.norm(s_dir, axis=1, keepdims=True)
    normal_incidence = s_len[:, 0] < 1e-6
    s_dir = np.where(s_len > 1e-12, s_dir / np.maximum(s_len, 1e-300), 0.0)
    es = np.sum(p * s_dir, axis=1)
    ep2 = np.maximum(0.0, 1.0 - es**2)
    rs = (n1 * cos_i - n2 * cos_t) / (n1 * cos_i + n2 * cos_t)
    rp = (n2 * cos_i - n1 * cos_t) / (n2 * cos_i + n1 * cos_t)
    t = 1.0 - (es**2 * rs**2 + ep2 * rp**2)
    t = np.where(normal_incidence, 1.0 - ((n1 - n2) / (n1 + n2)) ** 2, t)
    return np.where(tir, 0.0, t), tir, s2


def _fresnel_golden_check(rows_out, golden, tolerance):
    """Away from the critical angle: vectors and transmittance match the
    reference's own outputs. Within 2e-3 rad of it, where the reference's FP32
    cos(theta_t) cancels and the engine evaluates it in FP64, the
    transmittance matches an exact FP64 evaluation to 1e-5 relative."""
    t_exact, tir_exact, s2 = exact_fresnel(golden)
    ref = golden["fresnel_out"].astype(np.float64)
    n1 = golden["fresnel_index_from"].astype(np.float64)
    n2 = golden["fresnel_index_to"].astype(np.float64)
    sin_i = np.sqrt(np.clip(s2, 0, None)) * n2 / n1
    near_critical = np.zeros(len(s2), dtype=bool)
    valid = n1 > n2
    theta = np.arcsin(np.clip(sin_i, 0, 1))
    critical = np.arcsin(np.clip(n2 / n1, 0, 1))
    near_critical[valid] = np.abs(theta[valid] - critical[valid]) <= 2e-3
    np.testing.assert_array_equal(rows_out[:, 13], tir_exact.astype(np.float64))
    np.testing.assert_allclose(rows_out[:, 12], t_exact, rtol=1e-5, atol=1e-6)
    ok = ~near_critical
    assert np.array_equal(rows_out[ok, 13], ref[ok, 13]), "TIR decisions differ away from the critical angle"
    same = ok & (rows_out[:, 13] == ref[:, 13])
    transmitted = same & (ref[:, 13] == 0)
    # Where the transmittance differs from the reference's FP32 value by more
    # than the tolerance, the reference must be the one further from exact.
    apart = same & (np.abs(rows_out[:, 12] - ref[:, 12]) > tolerance + 1e-5 * np.abs(ref[:, 12]))
    assert np.all(np.abs(ref[apart, 12] - t_exact[apart]) > np.abs(rows_out[apart, 12] - t_exact[apart])), (
        "transmittance differs from the reference where the reference is the more accurate one"
    )
    np.testing.assert_allclose(rows_out[same, 0:3], ref[same, 0:3], atol=tolerance)
    # Near Brewster's angle r_p changes sign, so the reflected polarisation's
    # p component is rounding noise there; elsewhere it must match.
    d = golden["fresnel_direction"].astype(np.float64)
    nrm = golden["fresnel_normal"].astype(np.float64)
    cos_i = np.clip(-np.sum(d * nrm, axis=1) / np.linalg.norm(d, axis=1) / np.linalg.norm(nrm, axis=1), 0, 1)
    brewster = np.arctan(n2 / n1)
    near_brewster = np.abs(np.arccos(cos_i) - brewster) < 2e-2
    # Equal indices reflect nothing: the reference's FP32 cos(theta_t) makes a
    # spurious tiny reflection at grazing incidence whose polarisation is noise.
    reflecting = same & (1.0 - ref[:, 12] > 1e-6) & ~near_brewster & (n1 != n2)
    unit_rows = (rows_out[:, 13] == 0) & (1.0 - rows_out[:, 12] > 1e-6)
    np.testing.assert_allclose(np.linalg.norm(rows_out[unit_rows, 6:9], axis=1), 1.0, atol=1e-5)
    np.testing.assert_allclose(np.sum(rows_out[unit_rows, 6:9] * rows_out[unit_rows, 0:3], axis=1), 0.0, atol=1e-5)
    np.testing.assert_allclose(rows_out[reflecting, 6:9], ref[reflecting, 6:9], atol=tolerance)
    np.testing.assert_allclose(rows_out[transmitted, 3:6], ref[transmitted, 3:6], atol=tolerance)
    transmitting = transmitted & (ref[:, 12] > 1e-6)
    np.testing.assert_allclose(rows_out[transmitting, 9:12], ref[transmitting, 9:12], atol=tolerance)
    return int(near_critical.sum())


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_oracle_fresnel_matches_reference_golden(oracle, precision):
    golden = np.load(GOLDEN)
    f = fresnel_f if precision == "fp32" else fresnel_d
    rows = np.array([
        f(oracle, golden["fresnel_direction"][i], golden["fresnel_polarization"][i], golden["fresnel_normal"][i],
          golden["fresnel_index_from"][i], golden["fresnel_index_to"][i])
        for i in range(golden["fresnel_direction"].shape[0])
    ], dtype=np.float64)
    # required agreement of the boundary unit cases with the formulas: 1e-5 relative
    _fresnel_golden_check(rows, golden, tolerance=1e-5)


def test_oracle_surface_matches_reference_golden(oracle):
    golden = np.load(GOLDEN)
    lib = oracle.load()
    for r, t, has_r, has_t, u, expected in golden["classify"]:
        got = lib.oracle_classify_surface(float(r), float(t), int(has_r), int(has_t), float(u))
        assert got == REFERENCE_OUTCOME[int(expected)], (r, t, has_r, has_t, u)
    for eff, sensor, u, expected in golden["absorb"]:
        assert lib.oracle_evaluate_absorption(float(eff), int(sensor), float(u)) == REFERENCE_OUTCOME[int(expected)]
    out = np.zeros(3, dtype=np.float32)
    for i in range(golden["lambertian_normal"].shape[0]):
        nrm = np.ascontiguousarray(golden["lambertian_normal"][i])
        lib.oracle_lambertian_f(nrm.ctypes.data_as(F3), float(golden["lambertian_radial"][i]),
                                float(golden["lambertian_azimuth"][i]), out.ctypes.data_as(F3))
        # the engine's sin/cos of 2*pi*u versus the reference's sinf/cosf(2*pi*u)
        np.testing.assert_allclose(out, golden["lambertian_out"][i], atol=2e-6)


def test_oracle_matches_live_reference(oracle):
    ref = oracle.load_reference()
    if ref is None:
        pytest.skip("reference tree not present; the committed golden vectors cover this case")
    rng = np.random.default_rng(7)
    count = 2000
    normal = rng.normal(size=(count, 3))
    normal /= np.linalg.norm(normal, axis=1, keepdims=True)
    direction = rng.normal(size=(count, 3))
    direction /= np.linalg.norm(direction, axis=1, keepdims=True)
    flip = np.sum(direction * normal, axis=1) > 0
    direction[flip] *= -1
    polarization = np.cross(direction, rng.normal(size=(count, 3)))
    polarization /= np.linalg.norm(polarization, axis=1, keepdims=True)
    indices = rng.choice([1.0, 1.41, 1.5, 1.82], size=(count, 2))
    live = {
        "fresnel_direction": direction.astype(np.float32),
        "fresnel_polarization": polarization.astype(np.float32),
        "fresnel_normal": normal.astype(np.float32),
        "fresnel_index_from": indices[:, 0].astype(np.float32),
        "fresnel_index_to": indices[:, 1].astype(np.float32),
    }
    want = np.zeros((count, 14), dtype=np.float32)
    for i in range(count):
        args = [np.ascontiguousarray(live[k][i]) for k in ("fresnel_direction", "fresnel_polarization", "fresnel_normal")]
        ref.ref_fresnel(*(a.ctypes.data_as(F3) for a in args), float(live["fresnel_index_from"][i]),
                        float(live["fresnel_index_to"][i]), want[i].ctypes.data_as(F3))
    live["fresnel_out"] = want
    rows = np.array([
        fresnel_f(oracle, live["fresnel_direction"][i], live["fresnel_polarization"][i], live["fresnel_normal"][i],
                  live["fresnel_index_from"][i], live["fresnel_index_to"][i])
        for i in range(count)
    ], dtype=np.float64)
    _fresnel_golden_check(rows, live, tolerance=1e-5)

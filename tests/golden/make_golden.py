"""Generates tests/golden/boundary_reference.npz from the reference itself.

Runs the reference's own boundary physics (src/optical/optix/OptiXBoundaryPhysics.cuh,
compiled from the reference tree by oracle/Makefile into oracle/_ref) on a
fixed, seeded set of inputs and records its outputs, so the tests can pin
both the CPU oracle and the GPU engine to the reference where the reference
tree is absent. Inputs: the known-answer cases of
test/TestOpticalBoundaryPhysics.cxx:37-101, random incidences for several
index pairs, and incidences within 1e-3 rad of the critical angle.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import binding  # noqa: E402

OUT = Path(__file__).resolve().parent / "boundary_reference.npz"


def unit(v):
    v = np.asarray(v, dtype=np.float64)
    return v / np.linalg.norm(v)


def fresnel_inputs(rng: np.random.Generator):
    rows = []
    # Known-answer cases (TestOpticalBoundaryPhysics.cxx:37-69).
    rows.append(([0, 0, 1], [1, 0, 0], [0, 0, -1], 1.0, 1.5))
    a = math.atan(1.5)
    d = [math.sin(a), 0.0, math.cos(a)]
    p = np.cross(d, [0, 1, 0])
    rows.append((d, list(unit(p)), [0, 0, -1], 1.0, 1.5))
    a = 50.0 * math.pi / 180.0
    rows.append(([math.sin(a), 0, math.cos(a)], [0, 1, 0], [0, 0, -1], 1.5, 1.0))
    # Random incidences for the detector's index pairs and a few generic ones.
    pairs = [(1.82, 1.41), (1.41, 1.82), (1.41, 1.0), (1.0, 1.41), (1.82, 1.0), (1.0, 1.5), (1.5, 1.0), (1.46, 1.57)]
    for n1, n2 in pairs:
        for _ in range(64):
            normal = unit(rng.normal(size=3))
            direction = unit(rng.normal(size=3))
            if np.dot(direction, normal) > 0:
                direction = -direction
            pol = unit(np.cross(direction, rng.normal(size=3)))
            rows.append((direction, pol, normal, n1, n2))
    # Within 1e-3 rad of the critical angle, both sides.
    for n1, n2 in [(1.82, 1.41), (1.41, 1.0), (1.5, 1.0)]:
        critical = math.asin(n2 / n1)
        for delta in np.linspace(-1e-3, 1e-3, 21):
            t = critical + delta
            for pol in ([0, 1, 0], unit([math.cos(t), 0, -math.sin(t)])):
                rows.append(([math.sin(t), 0, math.cos(t)], pol, [0, 0, -1], n1, n2))
    direction = np.array([r[0] for r in rows], dtype=np.float32)
    polarization = np.array([r[1] for r in rows], dtype=np.float32)
    normal = np.array([r[2] for r in rows], dtype=np.float32)
    n_from = np.array([r[3] for r in rows], dtype=np.float32)
    n_to = np.array([r[4] for r in rows], dtype=np.float32)
    return direction, polarization, normal, n_from, n_to


def main() -> None:
    ref = binding.load_reference()
    if ref is None:
        raise SystemExit("the reference tree is needed to generate the golden vectors")
    rng = np.random.default_rng(20251203)
    d, p, n, n1, n2 = fresnel_inputs(rng)
    f3 = C.POINTER(C.c_float)
    out = np.zeros((d.shape[0], 14), dtype=np.float32)
    for i in range(d.shape[0]):
        ref.ref_fresnel(d[i].ctypes.data_as(f3), p[i].ctypes.data_as(f3), n[i].ctypes.data_as(f3),
                        float(n1[i]), float(n2[i]), out[i].ctypes.data_as(f3))
    # Lambertian (TestOpticalBoundaryPhysics.cxx:94-101) over random normals and samples.
    lam_normal = np.array([unit(rng.normal(size=3)) for _ in range(256)], dtype=np.float32)
    lam_normal[0] = [0, 0, 1]
    lam_radial = rng.random(256).astype(np.float32)
    lam_azimuth = rng.random(256).astype(np.float32)
    lam_radial[0], lam_azimuth[0] = 0.75, 0.25
    lam_out = np.zeros((256, 3), dtype=np.float32)
    for i in range(256):
        ref.ref_lambertian(lam_normal[i].ctypes.data_as(f3), float(lam_radial[i]), float(lam_azimuth[i]),
                           lam_out[i].ctypes.data_as(f3))
    # ClassifySurface / EvaluateAbsorption on a grid (TestOpticalBoundaryPhysics.cxx:71-92).
    grid = np.linspace(0.0, 1.0, 21, dtype=np.float32)
    classify = []
    for r in grid[::4]:
        for t in grid[::4]:
            for has_r in (0, 1):
                for has_t in (0, 1):
                    for u in grid:
                        classify.append((r, t, has_r, has_t, u, ref.ref_classify_surface(r, t, has_r, has_t, u)))
    absorb = []
    for eff in grid[::2]:
        for sensor in (0, 1):
            for u in grid:
                absorb.append((eff, sensor, u, ref.ref_evaluate_absorption(eff, sensor, u)))
    np.savez_compressed(
        OUT,
        fresnel_direction=d, fresnel_polarization=p, fresnel_normal=n, fresnel_index_from=n1, fresnel_index_to=n2,
        fresnel_out=out, lambertian_normal=lam_normal, lambertian_radial=lam_radial,
        lambertian_azimuth=lam_azimuth, lambertian_out=lam_out,
        classify=np.array(classify, dtype=np.float64), absorb=np.array(absorb, dtype=np.float64),
    )
    print(f"wrote {OUT} ({d.shape[0]} Fresnel rows)")


if __name__ == "__main__":
    main()

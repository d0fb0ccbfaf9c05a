"""The boundary against the reference's own headers, compiled with g++.

The reference's record and scene types need only CLHEP's G4ThreeVector from
Geant4 (include/g4go/optical/Scene.hpp:3); tests/stubs/G4ThreeVector.hh stands
in for it, so these programs include the real
include/g4go/optical/PhotonTransport.hpp and Scene.hpp and compile the real
src/optical/Scene.cpp:

- every field of OpticalEmission, PhotonDetection,
  PhotonTransportStatistics and PhotonTransportEventStatistics sits at the
  offset and has the size of its g4b_* counterpart, and the enumerations
  (emission types, statistic fields, surface type / model / finish) have the
  same values (static_asserts: the program must compile);
- a G4GO::Optical::Scene of the benchmark detector (box meshes in local
  coordinates under axis-permuting transforms, built through the Scene's own
  Add* methods) passes through g4b::BoxScene (include/g4b_scene_adapter.hpp)
  into the boxes of g4go_b200.scenes.crystal_sipm_scene.

The reference tree is read where G4GO_REFERENCE (or the build's default
location) points; where it is absent the tests skip.
"""
import os
import subprocess
from pathlib import Path

import pytest

from g4go_b200 import build, scenes

ROOT = Path(__file__).resolve().parent.parent
STUBS = Path(__file__).resolve().parent / "stubs"


def reference_tree() -> Path | None:
    import __graft_entry__

    tree = Path(os.environ.get("G4GO_REFERENCE", str(__graft_entry__.REFERENCE_TREE)))
    return tree if (tree / "include" / "g4go" / "optical" / "Scene.hpp").is_file() else None


LAYOUT = r"""
#include <cstddef>
#include <type_traits>

#include "g4go/optical/PhotonTransport.hpp"
#include "g4b.h"

namespace R = G4GO::Optical;

#define SAME_FIELD(RT, rf, GT, gf)                                                              \
    static_assert(offsetof(RT, rf) == offsetof(GT, gf), #RT "::" #rf " offset");                \
    static_assert(sizeof(std::declval<RT>().rf) == sizeof(std::declval<GT>().gf), #RT "::" #rf " size")

SAME_FIELD(R::OpticalEmission, positionMm, g4b_optical_emission, position_mm);
SAME_FIELD(R::OpticalEmission, timeNs, g4b_optical_emission, time_ns);
SAME_FIELD(R::OpticalEmission, direction, g4b_optical_emission, direction);
SAME_FIELD(R::OpticalEmission, stepLengthMm, g4b_optical_emission, step_length_mm);
SAME_FIELD(R::OpticalEmission, stepDeltaMm, g4b_optical_emission, step_delta_mm);
SAME_FIELD(R::OpticalEmission, preVelocityMmPerNs, g4b_optical_emission, pre_velocity_mm_per_ns);
SAME_FIELD(R::OpticalEmission, polarization, g4b_optical_emission, polarization);
SAME_FIELD(R::OpticalEmission, deltaVelocityMmPerNs, g4b_optical_emission, delta_velocity_mm_per_ns);
SAME_FIELD(R::OpticalEmission, energyEv, g4b_optical_emission, energy_ev);
SAME_FIELD(R::OpticalEmission, preMeanPhotonCount, g4b_optical_emission, pre_mean_photon_count);
SAME_FIELD(R::OpticalEmission, postMeanPhotonCount, g4b_optical_emission, post_mean_photon_count);
SAME_FIELD(R::OpticalEmission, decayTimeNs, g4b_optical_emission, decay_time_ns);
SAME_FIELD(R::OpticalEmission, riseTimeNs, g4b_optical_emission, rise_time_ns);
SAME_FIELD(R::OpticalEmission, charge, g4b_optical_emission, charge);
SAME_FIELD(R::OpticalEmission, eventID, g4b_optical_emission, event_id);
SAME_FIELD(R::OpticalEmission, firstPhotonID, g4b_optical_emission, first_photon_id);
SAME_FIELD(R::OpticalEmission, photonCount, g4b_optical_emission, photon_count);
SAME_FIELD(R::OpticalEmission, volumeID, g4b_optical_emission, volume_id);
SAME_FIELD(R::OpticalEmission, materialID, g4b_optical_emission, material_id);
SAME_FIELD(R::OpticalEmission, spectrumID, g4b_optical_emission, spectrum_id);
SAME_FIELD(R::OpticalEmission, type, g4b_optical_emission, type);
static_assert(sizeof(R::OpticalEmission) == sizeof(g4b_optical_emission));
static_assert(alignof(R::OpticalEmission) == 16);

SAME_FIELD(R::PhotonDetection, positionMm, g4b_photon_detection, position_mm);
SAME_FIELD(R::PhotonDetection, timeNs, g4b_photon_detection, time_ns);
SAME_FIELD(R::PhotonDetection, direction, g4b_photon_detection, direction);
SAME_FIELD(R::PhotonDetection, energyEv, g4b_photon_detection, energy_ev);
SAME_FIELD(R::PhotonDetection, eventID, g4b_photon_detection, event_id);
SAME_FIELD(R::PhotonDetection, photonID, g4b_photon_detection, photon_id);
SAME_FIELD(R::PhotonDetection, sensorID, g4b_photon_detection, sensor_id);
static_assert(sizeof(R::PhotonDetection) == sizeof(g4b_photon_detection));

SAME_FIELD(R::PhotonTransportStatistics, validFields, g4b_statistics, valid_fields);
SAME_FIELD(R::PhotonTransportStatistics, generatedCount, g4b_statistics, generated_count);
SAME_FIELD(R::PhotonTransportStatistics, capturedCount, g4b_statistics, captured_count);
SAME_FIELD(R::PhotonTransportStatistics, detectedCount, g4b_statistics, detected_count);
SAME_FIELD(R::PhotonTransportStatistics, absorbedCount, g4b_statistics, absorbed_count);
SAME_FIELD(R::PhotonTransportStatistics, escapedCount, g4b_statistics, escaped_count);
SAME_FIELD(R::PhotonTransportStatistics, truncatedCount, g4b_statistics, truncated_count);
SAME_FIELD(R::PhotonTransportStatistics, maxBounceCount, g4b_statistics, max_bounce_count);
SAME_FIELD(R::PhotonTransportStatistics, invalidStateCount, g4b_statistics, invalid_state_count);
SAME_FIELD(R::PhotonTransportStatistics, zeroStepCount, g4b_statistics, zero_step_count);
SAME_FIELD(R::PhotonTransportStatistics, transportTimeMs, g4b_statistics, transport_time_ms);
static_assert(sizeof(R::PhotonTransportStatistics) == sizeof(g4b_statistics));
SAME_FIELD(R::PhotonTransportEventStatistics, eventID, g4b_event_statistics, event_id);
SAME_FIELD(R::PhotonTransportEventStatistics, statistics, g4b_event_statistics, statistics);
static_assert(sizeof(R::PhotonTransportEventStatistics) == sizeof(g4b_event_statistics));

static_assert(static_cast<int>(R::OpticalEmissionType::Direct) == G4B_EMISSION_DIRECT);
static_assert(static_cast<int>(R::OpticalEmissionType::Cerenkov) == G4B_EMISSION_CERENKOV);
static_assert(static_cast<int>(R::OpticalEmissionType::Scintillation) == G4B_EMISSION_SCINTILLATION);
static_assert(static_cast<int>(R::PhotonTransportStatisticField::Generated) == G4B_FIELD_GENERATED);
static_assert(static_cast<int>(R::PhotonTransportStatisticField::Captured) == G4B_FIELD_CAPTURED);
static_assert(static_cast<int>(R::PhotonTransportStatisticField::Detected) == G4B_FIELD_DETECTED);
static_assert(static_cast<int>(R::PhotonTransportStatisticField::Absorbed) == G4B_FIELD_ABSORBED);
static_assert(static_cast<int>(R::PhotonTransportStatisticField::Escaped) == G4B_FIELD_ESCAPED);
static_assert(static_cast<int>(R::PhotonTransportStatisticField::Truncated) == G4B_FIELD_TRUNCATED);
static_assert(static_cast<int>(R::PhotonTransportStatisticField::MaxBounce) == G4B_FIELD_MAX_BOUNCE);
static_assert(static_cast<int>(R::PhotonTransportStatisticField::InvalidState) == G4B_FIELD_INVALID_STATE);
static_assert(static_cast<int>(R::PhotonTransportStatisticField::ZeroStep) == G4B_FIELD_ZERO_STEP);
static_assert(static_cast<int>(R::PhotonTransportStatisticField::TransportTime) == G4B_FIELD_TRANSPORT_TIME);
static_assert(static_cast<int>(R::SurfaceType::DielectricDielectric) == G4B_SURFACE_DIELECTRIC_DIELECTRIC);
static_assert(static_cast<int>(R::SurfaceType::DielectricMetal) == G4B_SURFACE_DIELECTRIC_METAL);
static_assert(static_cast<int>(R::SurfaceModel::Glisur) == G4B_MODEL_GLISUR);
static_assert(static_cast<int>(R::SurfaceModel::Unified) == G4B_MODEL_UNIFIED);
static_assert(static_cast<int>(R::SurfaceFinish::Polished) == G4B_FINISH_POLISHED);
static_assert(static_cast<int>(R::SurfaceFinish::Ground) == G4B_FINISH_GROUND);
static_assert(R::InvalidID == G4B_INVALID_ID);

int main() { return 0; }
"""

SCENE = r"""
#include <cstdio>
#include <stdexcept>
#include <string>

#include "g4go/optical/Scene.hpp"
#include "g4b_scene_adapter.hpp"

using namespace G4GO::Optical;

// 8-vertex box mesh (12 triangles) of half sizes h in local coordinates
static Geometry BoxMesh(const char* name, double hx, double hy, double hz) {
    Geometry g{name, {}};
    for (int k = 0; k < 8; ++k) {
        g.mesh.verticesMm.push_back({(k & 1) ? hx : -hx, (k & 2) ? hy : -hy, (k & 4) ? hz : -hz});
    }
    const unsigned faces[12][3]{{0, 1, 3}, {0, 3, 2}, {4, 6, 7}, {4, 7, 5}, {0, 4, 5}, {0, 5, 1},
                                {2, 3, 7}, {2, 7, 6}, {0, 2, 6}, {0, 6, 4}, {1, 5, 7}, {1, 7, 3}};
    for (const auto& f : faces) {
        g.mesh.indices.insert(g.mesh.indices.end(), {f[0], f[1], f[2]});
    }
    g.mesh.triangleFlags.assign(12, 0);
    return g;
}

static Volume Place(const char* name, unsigned geometry, unsigned material, unsigned parent, Rotation rotation,
                    G4ThreeVector translation) {
    Volume v{};
    v.name = name;
    v.geometryID = geometry;
    v.materialID = material;
    v.parentVolumeID = parent;
    v.transform.rotation = rotation;
    v.transform.translationMm = translation;
    return v;
}

int main(int argc, char** argv) {
    if (argc < 7) {
        return 2;
    }
    const double w = std::stod(argv[1]), hx = std::stod(argv[2]), hy = std::stod(argv[3]), hz = std::stod(argv[4]);
    const double g = std::stod(argv[5]), s = std::stod(argv[6]);
    Scene scene;
    Material air{};
    air.name = "air";
    air.rindex = {{2.0F, 4.0F}, {1.0F, 1.0F}};
    Material crystal{};
    crystal.name = "crystal";
    crystal.rindex = {{2.0F, 4.0F}, {1.82F, 1.82F}};
    crystal.rindexMax = 1.82F;
    crystal.absLengthMm = {{2.0F, 4.0F}, {400.0F, 400.0F}};
    scene.AddMaterial(air);
    scene.AddMaterial(crystal);
    Surface wrapper{};
    wrapper.name = "wrapper";
    wrapper.type = SurfaceType::DielectricMetal;
    wrapper.reflectivity = {{2.0F, 4.0F}, {0.95F, 0.95F}};
    Surface cathode{};
    cathode.name = "cathode";
    cathode.type = SurfaceType::DielectricMetal;
    cathode.model = SurfaceModel::Glisur;
    cathode.finish = SurfaceFinish::Ground;
    cathode.modelValue = 0.5F;
    cathode.efficiency = {{2.0F, 3.0F, 4.0F}, {0.3F, 0.3F, 0.3F}};
    scene.AddSurface(wrapper);
    scene.AddSurface(cathode);
    scene.AddGeometry(BoxMesh("world", w, w, w));
    scene.AddGeometry(BoxMesh("crystal", hz, hx, hy));
    scene.AddGeometry(BoxMesh("grease", hx, hy, g / 2));
    scene.AddGeometry(BoxMesh("sipm", hy, hx, s / 2));
    scene.AddVolume(Place("world", 0, 0, InvalidID, Rotation{}, {0, 0, 0}));
    // world x = local y, y = local z, z = local x
    scene.AddVolume(Place("crystal", 1, 1, 0, Rotation{0, 1, 0, 0, 0, 1, 1, 0, 0}, {0, 0, 0}));
    // 180 degrees about z
    scene.AddVolume(Place("grease", 2, 1, 0, Rotation{-1, 0, 0, 0, -1, 0, 0, 0, 1}, {0, 0, hz + g / 2}));
    // x and y swapped, z flipped
    Volume sipm{Place("sipm", 3, 0, 0, Rotation{0, 1, 0, 1, 0, 0, 0, 0, -1}, {0, 0, hz + g + s / 2})};
    sipm.skinSurfaceID = 1;
    sipm.sensorID = 7;
    scene.AddVolume(sipm);
    scene.AddSurfaceBinding({1, 0, 0});
    scene.WorldVolumeID(0);
    g4b::BoxScene boxes{scene};
    const g4b_scene& out = boxes.Get();
    for (unsigned i = 0; i < out.volume_count; ++i) {
        const g4b_volume& v = out.volumes[i];
        std::printf("box %u %u %u %u %u %.9g %.9g %.9g %.9g %.9g %.9g\n", v.volume_id, v.material_id,
                    v.parent_volume_id, v.skin_surface_id, v.sensor_id, v.center_mm[0], v.center_mm[1],
                    v.center_mm[2], v.half_size_mm[0], v.half_size_mm[1], v.half_size_mm[2]);
    }
    std::printf("scene %u %u %u %u %u %u %u %g %g %u %u\n", out.material_count, out.surface_count,
                out.binding_count, out.world_volume_id, out.bindings[0].from_volume_id, out.surfaces[1].finish,
                out.surfaces[1].efficiency.count, out.surfaces[0].reflectivity.values[0],
                out.materials[1].abs_length_mm.values[1], out.materials[1].rindex.count,
                out.materials[0].abs_length_mm.count);
    return 0;
}
"""


def compile_program(tmp_path, source_text, tree, extra_sources=(), run=True, args=()):
    source = tmp_path / "program.cpp"
    source.write_text(source_text)
    exe = tmp_path / "program"
    command = ["g++", "-std=c++20", "-O1", "-I", str(STUBS), "-I", str(tree / "include"), "-I",
               str(ROOT / "include"), str(source), *map(str, extra_sources), "-o", str(exe)]
    subprocess.run(command, check=True)
    if not run:
        return []
    return subprocess.run([str(exe), *args], check=True, capture_output=True, text=True).stdout.splitlines()


def test_record_layouts_and_enumerations_are_the_reference_headers(tmp_path):
    tree = reference_tree()
    if tree is None:
        pytest.skip("the reference tree is not here")
    compile_program(tmp_path, LAYOUT, tree, run=False)


def test_the_reference_scene_type_becomes_the_benchmark_boxes(tmp_path):
    tree = reference_tree()
    if tree is None:
        pytest.skip("the reference tree is not here")
    params = scenes.DetectorParameters()
    hx, hy, hz = params.crystal_half_mm
    args = [str(v) for v in (params.world_half_mm, hx, hy, hz, params.grease_thickness_mm, params.sipm_thickness_mm)]
    lines = compile_program(tmp_path, SCENE, tree, extra_sources=[tree / "src" / "optical" / "Scene.cpp"], args=args)
    boxes = [line.split()[1:] for line in lines if line.startswith("box ")]
    benchmark = scenes.crystal_sipm_scene(params)
    assert len(boxes) == len(benchmark.volumes) == 4
    for fields, volume in zip(boxes, benchmark.volumes):
        assert int(fields[0]) == volume.volume_id
        geometry = list(map(float, fields[5:]))
        assert geometry[:3] == pytest.approx(list(volume.center_mm), abs=1e-6)
        assert geometry[3:] == pytest.approx(list(volume.half_size_mm), abs=1e-6)
    assert list(map(int, boxes[3][:5])) == [3, 0, 0, 1, 7]
    assert next(line for line in lines if line.startswith("scene ")).split()[1:] == \
        ["2", "2", "1", "0", "1", "1", "3", "0.95", "400", "2", "0"]
    assert build.PACKAGE.exists()

"""g4b::BoxScene (include/g4b_scene_adapter.hpp): the reference's exported Scene
of meshes and transforms turned into the engine's analytic boxes.

A C++ program builds a Scene with the reference's type and field names
(include/g4go/optical/Scene.hpp:30-163; a three-float vector stands in for
CLHEP's G4ThreeVector). The world, crystal, grease and SiPM of the benchmark
detector are given as 8-vertex box meshes in local coordinates, placed by
transforms that permute, flip and translate the axes. The boxes that come out
must be those of the benchmark scene (g4go_b200.scenes.crystal_sipm_scene).
The program also checks that property tables, surfaces, bindings and IDs
pass through, and that a rotated box and a non-box mesh are rejected.
"""
import subprocess

import pytest

from g4go_b200 import build, scenes

PROGRAM = r"""
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "g4b_scene_adapter.hpp"

struct Vec3 {
    double a, b, c;
    double x() const { return a; }
    double y() const { return b; }
    double z() const { return c; }
};
enum class SurfaceType : unsigned char { DielectricDielectric, DielectricMetal };
enum class SurfaceModel : unsigned char { Glisur, Unified };
enum class SurfaceFinish : unsigned char { Polished, Ground };
struct Rotation { float xx{1}, xy{}, xz{}, yx{}, yy{1}, yz{}, zx{}, zy{}, zz{1}; };
struct Transform { Rotation rotation{}; Vec3 translationMm{0, 0, 0}; };
struct PropertyTable { std::vector<float> energyEv, values; };
struct Material {
    std::string name;
    PropertyTable rindex;
    float rindexMax{1.0F};
    PropertyTable groupVelocityMmPerNs, absLengthMm;
    PropertyTable scintillationSpectrum[3];
};
struct Surface {
    std::string name;
    SurfaceType type{SurfaceType::DielectricDielectric};
    SurfaceModel model{SurfaceModel::Unified};
    SurfaceFinish finish{SurfaceFinish::Polished};
    float modelValue{1.0F};
    PropertyTable reflectivity, efficiency, transmittance, rindex, specularLobe, specularSpike, backscatter,
        surfaceRoughness;
};
struct MeshGeometry { std::string name; std::vector<Vec3> verticesMm; std::vector<unsigned> indices; };
struct Geometry { std::string name; MeshGeometry mesh; };
struct Volume {
    std::string name;
    unsigned volumeID{~0U}, physicalVolumeID{~0U}, copyNo{}, geometryID{~0U}, materialID{~0U},
        parentVolumeID{~0U}, skinSurfaceID{~0U}, sensorID{~0U}, depth{};
    bool mayHaveCoincidentBoundary{};
    Transform transform{};
};
struct SurfaceBinding { unsigned fromVolumeID{~0U}, toVolumeID{~0U}, surfaceID{~0U}; };
struct Scene {
    std::vector<Material> materials;
    std::vector<Surface> surfaces;
    std::vector<Geometry> geometries;
    std::vector<Volume> volumes;
    std::vector<SurfaceBinding> bindings;
    unsigned world{0};
    const std::vector<Material>& Materials() const { return materials; }
    const std::vector<Surface>& Surfaces() const { return surfaces; }
    const std::vector<Geometry>& Geometries() const { return geometries; }
    const std::vector<Volume>& Volumes() const { return volumes; }
    const std::vector<SurfaceBinding>& SurfaceBindings() const { return bindings; }
    unsigned WorldVolumeID() const { return world; }
};

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
    return g;
}

int main(int argc, char** argv) {
    if (argc < 7) {
        return 2;
    }
    const double w = std::stod(argv[1]), hx = std::stod(argv[2]), hy = std::stod(argv[3]), hz = std::stod(argv[4]);
    const double g = std::stod(argv[5]), s = std::stod(argv[6]);
    Scene scene;
    Material air{"air"};
    air.rindex = {{2.0F, 4.0F}, {1.0F, 1.0F}};
    Material crystal{"crystal"};
    crystal.rindex = {{2.0F, 4.0F}, {1.82F, 1.82F}};
    crystal.rindexMax = 1.82F;
    crystal.absLengthMm = {{2.0F, 4.0F}, {400.0F, 400.0F}};
    scene.materials = {air, crystal};
    Surface wrapper{"wrapper", SurfaceType::DielectricMetal, SurfaceModel::Unified, SurfaceFinish::Polished, 0.0F};
    wrapper.reflectivity = {{2.0F, 4.0F}, {0.95F, 0.95F}};
    Surface cathode{"cathode", SurfaceType::DielectricMetal, SurfaceModel::Glisur, SurfaceFinish::Ground, 0.5F};
    cathode.efficiency = {{2.0F, 3.0F, 4.0F}, {0.3F, 0.3F, 0.3F}};
    scene.surfaces = {wrapper, cathode};
    // world = R local + t; each volume's local mesh is laid out so that its
    // transform brings it onto the benchmark's box
    scene.geometries = {BoxMesh("world", w, w, w), BoxMesh("crystal", hz, hx, hy), BoxMesh("grease", hx, hy, g / 2),
                        BoxMesh("sipm", hy, hx, s / 2)};
    Volume world{"world", 0, 0, 0, 0, 0};
    Volume vcrystal{"crystal", 1, 1, 0, 1, 1, 0};
    vcrystal.transform.rotation = {0, 1, 0, 0, 0, 1, 1, 0, 0};  // world x = local y, y = local z, z = local x
    Volume grease{"grease", 2, 2, 0, 2, 1, 0};
    grease.transform.rotation = {-1, 0, 0, 0, -1, 0, 0, 0, 1};  // 180 degrees about z
    grease.transform.translationMm = {0, 0, hz + g / 2};
    Volume sipm{"sipm", 3, 3, 0, 3, 0, 0, 1, 7};
    sipm.transform.rotation = {0, 1, 0, 1, 0, 0, 0, 0, -1};  // swap x and y, flip z
    sipm.transform.translationMm = {0, 0, hz + g + s / 2};
    scene.volumes = {world, vcrystal, grease, sipm};
    scene.bindings = {{1, 0, 0}};
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
    int rejected = 0;
    Scene rotated = scene;
    rotated.volumes[1].transform.rotation = {0.70710678F, -0.70710678F, 0, 0.70710678F, 0.70710678F, 0, 0, 0, 1};
    try { g4b::BoxScene bad{rotated}; } catch (const std::invalid_argument&) { ++rejected; }
    Scene prism = scene;
    prism.geometries[2].mesh.verticesMm[7] = {0, 0, 0};  // a vertex moved inside
    try { g4b::BoxScene bad{prism}; } catch (const std::invalid_argument&) { ++rejected; }
    Scene wedge = scene;
    wedge.geometries[3].mesh.verticesMm.resize(6);  // two corners missing
    try { g4b::BoxScene bad{wedge}; } catch (const std::invalid_argument&) { ++rejected; }
    std::printf("rejected %d\n", rejected);
    return 0;
}
"""


def test_reference_scene_meshes_become_the_benchmark_boxes(tmp_path):
    params = scenes.DetectorParameters()
    box_scene = scenes.crystal_sipm_scene(params)
    hx, hy, hz = params.crystal_half_mm
    source = tmp_path / "adapter.cpp"
    source.write_text(PROGRAM)
    exe = tmp_path / "adapter"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
                    "-Wno-missing-field-initializers", "-I", str(build.PACKAGE.parent / "include"), str(source), "-o", str(exe)], check=True)
    args = [str(v) for v in (params.world_half_mm, hx, hy, hz, params.grease_thickness_mm, params.sipm_thickness_mm)]
    lines = subprocess.run([str(exe), *args], check=True, capture_output=True, text=True).stdout.splitlines()
    boxes = [line.split()[1:] for line in lines if line.startswith("box ")]
    assert len(boxes) == 4
    for fields, volume in zip(boxes, box_scene.volumes):
        ids = list(map(int, fields[:5]))
        geometry = list(map(float, fields[5:]))
        assert ids[0] == volume.volume_id
        assert geometry[:3] == pytest.approx(list(volume.center_mm), abs=1e-6)
        assert geometry[3:] == pytest.approx(list(volume.half_size_mm), abs=1e-6)
    assert list(map(int, boxes[3][:5])) == [3, 0, 0, 1, 7]  # skin surface and sensor ID pass through
    scene_line = next(line for line in lines if line.startswith("scene ")).split()[1:]
    assert scene_line == ["2", "2", "1", "0", "1", "1", "3", "0.95", "400", "2", "0"]
    assert lines[-1] == "rejected 3"

"""Transport through the reference's exported Scene, against the oracle.

A C++ program builds the benchmark detector as the reference's exporter
hands it over - a Scene of 8-vertex box meshes in local coordinates, placed
by transforms that permute, flip and translate the axes (the type and field
names of include/g4go/optical/Scene.hpp:30-163, restated here because the GPU
machine has no reference tree; tests/test_reference_headers.py runs the same
adapter on the reference's real Scene type) - and transports gensteps through
the C++ drop-in g4b::TransportHost (include/g4b_transport_host.hpp), whose
PrepareScene converts the Scene with g4b::BoxScene. The detections and
per-event counters must be those of the CPU oracle on the engine's native
boxes (g4go_b200.scenes.crystal_sipm_scene), byte for byte.
"""
import subprocess

import numpy as np
import pytest

from g4go_b200 import DETECTION_DTYPE, PhotonTransportConfig, build, scenes

pytestmark = pytest.mark.gpu

PROGRAM = r"""
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "g4b_transport_host.hpp"

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
struct Batch {
    std::vector<g4b_optical_emission> emissions;
    std::vector<std::uint32_t> eventIDs;
    std::vector<std::uint32_t> emissionEventIndices;
};

// Local half sizes and the rotation that maps local axes onto the world's:
// world axis i = sign_i * local axis perm[i].
static const int kPermutations[4][3]{{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {1, 0, 2}};
static const float kSigns[4][3]{{1, 1, 1}, {1, 1, 1}, {-1, 1, 1}, {1, -1, -1}};

static Geometry BoxMesh(const double h[3]) {
    Geometry g{"box", {}};
    for (int k = 0; k < 8; ++k) {
        g.mesh.verticesMm.push_back({(k & 1) ? h[0] : -h[0], (k & 2) ? h[1] : -h[1], (k & 4) ? h[2] : -h[2]});
    }
    const unsigned faces[12][3]{{0, 1, 3}, {0, 3, 2}, {4, 6, 7}, {4, 7, 5}, {0, 4, 5}, {0, 5, 1},
                                {2, 3, 7}, {2, 7, 6}, {0, 2, 6}, {0, 6, 4}, {1, 5, 7}, {1, 7, 3}};
    for (const auto& f : faces) {
        g.mesh.indices.insert(g.mesh.indices.end(), {f[0], f[1], f[2]});
    }
    return g;
}

static PropertyTable ReadTable(std::istringstream& in) {
    unsigned n{};
    in >> n;
    PropertyTable t;
    t.energyEv.resize(n);
    t.values.resize(n);
    for (auto& e : t.energyEv) in >> e;
    for (auto& v : t.values) in >> v;
    return t;
}

template<class T>
static std::vector<T> ReadRaw(const char* path) {
    std::ifstream f(path, std::ios::binary);
    std::vector<char> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    std::vector<T> out(bytes.size() / sizeof(T));
    std::memcpy(out.data(), bytes.data(), out.size() * sizeof(T));
    return out;
}

int main(int argc, char** argv) {
    if (argc < 8) {
        return 2;
    }
    Scene scene;
    std::ifstream spec(argv[1]);
    std::string line;
    while (std::getline(spec, line)) {
        std::istringstream in(line);
        std::string kind;
        in >> kind;
        if (kind == "material") {
            Material m;
            in >> m.name >> m.rindexMax;
            scene.materials.push_back(m);
        } else if (kind == "mprop") {
            std::string what;
            int component{};
            in >> what >> component;
            Material& m = scene.materials.back();
            PropertyTable t = ReadTable(in);
            if (what == "rindex") m.rindex = t;
            else if (what == "velocity") m.groupVelocityMmPerNs = t;
            else if (what == "abs") m.absLengthMm = t;
            else if (what == "spectrum") m.scintillationSpectrum[component] = t;
        } else if (kind == "surface") {
            Surface s;
            int type{}, model{}, finish{};
            in >> s.name >> type >> model >> finish >> s.modelValue;
            s.type = static_cast<SurfaceType>(type);
            s.model = static_cast<SurfaceModel>(model);
            s.finish = static_cast<SurfaceFinish>(finish);
            scene.surfaces.push_back(s);
        } else if (kind == "sprop") {
            std::string what;
            in >> what;
            Surface& s = scene.surfaces.back();
            PropertyTable t = ReadTable(in);
            if (what == "reflectivity") s.reflectivity = t;
            else if (what == "efficiency") s.efficiency = t;
            else if (what == "transmittance") s.transmittance = t;
        } else if (kind == "volume") {
            Volume v;
            double c[3], h[3];
            in >> v.volumeID >> v.materialID >> v.parentVolumeID >> v.skinSurfaceID >> v.sensorID >> c[0] >> c[1] >>
                c[2] >> h[0] >> h[1] >> h[2];
            const int k = static_cast<int>(scene.volumes.size() % 4);
            double local[3];
            float r[3][3]{};
            for (int i = 0; i < 3; ++i) {
                local[kPermutations[k][i]] = h[i];
                r[i][kPermutations[k][i]] = kSigns[k][i];
            }
            v.geometryID = static_cast<unsigned>(scene.geometries.size());
            scene.geometries.push_back(BoxMesh(local));
            v.transform.rotation = {r[0][0], r[0][1], r[0][2], r[1][0], r[1][1], r[1][2], r[2][0], r[2][1], r[2][2]};
            v.transform.translationMm = {c[0], c[1], c[2]};
            scene.volumes.push_back(v);
        } else if (kind == "binding") {
            SurfaceBinding b;
            in >> b.fromVolumeID >> b.toVolumeID >> b.surfaceID;
            scene.bindings.push_back(b);
        } else if (kind == "world") {
            in >> scene.world;
        }
    }
    Batch batch;
    batch.emissions = ReadRaw<g4b_optical_emission>(argv[2]);
    batch.eventIDs = ReadRaw<std::uint32_t>(argv[3]);
    batch.emissionEventIndices = ReadRaw<std::uint32_t>(argv[4]);
    g4b_config config{};
    config.seed = std::stoull(argv[5]);
    config.device = -1;
    config.ordered_detections = 1;
    g4b::TransportHost host{config};
    host.EnqueueEmissions(scene, batch);
    const g4b::TransportOutput out{host.CompleteOldestBatch()};
    std::ofstream(argv[6], std::ios::binary)
        .write(reinterpret_cast<const char*>(out.detections.data()),
               static_cast<std::streamsize>(out.detections.size() * sizeof(g4b_photon_detection)));
    std::ofstream(argv[7], std::ios::binary)
        .write(reinterpret_cast<const char*>(out.eventStatistics.data()),
               static_cast<std::streamsize>(out.eventStatistics.size() * sizeof(g4b_event_statistics)));
    std::printf("%zu detections\n", out.detections.size());
    return 0;
}
"""


def table_line(prefix, what, table, component=None):
    energy, values = (np.asarray(a, np.float32) for a in table)
    head = f"{prefix} {what}" + (f" {component}" if component is not None else (" 0" if prefix == "mprop" else ""))
    return " ".join([head, str(energy.size), *map(repr, map(float, energy)), *map(repr, map(float, values))])


def scene_spec(scene) -> str:
    lines = []
    for m in scene.materials:
        # the exporter sets rindexMax to the RINDEX table's maximum
        rindex_max = float(m.rindex_max) if m.rindex_max else (
            float(np.max(m.rindex[1])) if m.rindex is not None else 1.0)
        lines.append(f"material {m.name} {rindex_max!r}")
        if m.rindex is not None:
            lines.append(table_line("mprop", "rindex", m.rindex))
        if m.group_velocity_mm_per_ns is not None:
            lines.append(table_line("mprop", "velocity", m.group_velocity_mm_per_ns))
        if m.abs_length_mm is not None:
            lines.append(table_line("mprop", "abs", m.abs_length_mm))
        for c, spectrum in enumerate(m.scintillation_spectrum):
            if spectrum is not None:
                lines.append(table_line("mprop", "spectrum", spectrum, c))
    for s in scene.surfaces:
        lines.append(f"surface {s.name} {s.type} {s.model} {s.finish} {float(s.model_value)!r}")
        for what in ("reflectivity", "efficiency", "transmittance"):
            if getattr(s, what) is not None:
                lines.append(table_line("sprop", what, getattr(s, what)))
    for v in scene.volumes:
        numbers = [v.volume_id, v.material_id, v.parent_volume_id, v.skin_surface_id, v.sensor_id,
                   *map(float, v.center_mm), *map(float, v.half_size_mm)]
        lines.append("volume " + " ".join(map(repr, numbers)))
    for b in scene.surface_bindings:
        lines.append(f"binding {b.from_volume_id} {b.to_volume_id} {b.surface_id}")
    lines.append(f"world {scene.world_volume_id}")
    return "\n".join(lines) + "\n"


def test_exported_scene_transports_like_the_native_boxes(tmp_path, oracle):
    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload("batched", event_count=30, seed=21)
    (tmp_path / "scene.txt").write_text(scene_spec(scene))
    batch.emissions.tofile(tmp_path / "emissions.bin")
    batch.event_ids.tofile(tmp_path / "events.bin")
    batch.emission_event_indices.tofile(tmp_path / "indices.bin")
    source = tmp_path / "drop_in.cpp"
    source.write_text(PROGRAM)
    exe = tmp_path / "drop_in"
    library = build.build()
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(build.PACKAGE.parent / "include"), str(source),
                    str(library), f"-Wl,-rpath,{library.parent}", "-o", str(exe)], check=True)
    seed = 31337
    subprocess.run([str(exe), *(str(tmp_path / n) for n in ("scene.txt", "emissions.bin", "events.bin",
                                                            "indices.bin")), str(seed),
                    str(tmp_path / "detections.bin"), str(tmp_path / "events_out.bin")], check=True)
    detections = np.fromfile(tmp_path / "detections.bin", dtype=DETECTION_DTYPE)
    reference = oracle.transport(scene, batch, PhotonTransportConfig(seed=seed, precision="fp32"))
    assert detections.shape[0] == reference.detections.shape[0] > 0
    assert detections.tobytes() == reference.detections.tobytes()
    from g4go_b200 import _abi

    records = np.fromfile(tmp_path / "events_out.bin", dtype=np.dtype(_abi.EventStatistics))
    for record, (event_id, stats) in zip(records, reference.event_statistics):
        assert int(record["event_id"]) == event_id
        for key in ("detected_count", "absorbed_count", "escaped_count", "truncated_count", "max_bounce_count"):
            assert int(record["statistics"][key]) == stats[key], (event_id, key)

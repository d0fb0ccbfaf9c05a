// ref_transport_shim.cpp - the reference's own device program
// (src/optical/optix/OptiXTransportDevice.cu) compiled unmodified for the
// host, with C entry points that run it on a box scene. TEST INFRASTRUCTURE
// ONLY: it pins the CPU oracle's restatement of the counter RNG, the property
// and spectrum sampling, photon generation and the bounce loop to the
// reference's code (tests/golden/make_golden_transport.py writes its outputs
// as fixtures; tests/test_oracle_reference_transport.py compares).
//
// What is the shim's own, not the reference's:
//   - the OptiX device API (oracle/ref_stub/optix_device.h): optixTrace tests
//     the ray against every triangle of every box in double precision
//     (Moller-Trumbore, t rounded to float) and calls the program's
//     __closesthit__ch / __anyhit__ah / __miss__ms as a pipeline with
//     OPTIX_RAY_FLAG_DISABLE_ANYHIT or ENFORCE_ANYHIT|DISABLE_CLOSESTHIT would;
//   - the scene: g4b_scene boxes become 12-triangle meshes in world
//     coordinates (identity instance transforms), touching faces set to one
//     plane and flagged coincident with the rules of
//     src/optical/geant4/Geant4SceneExporter.cpp:379-487 (siblings with
//     opposite normals, parent and child either way) - the same planes the
//     engine and the oracle use;
//   - the host-side packing that OptiXTransportHost.cpp does before a launch,
//     restated: property tables (:357-372, constant flag Scene.cpp:18-22), the
//     trapezoid spectrum CDF (:374-410), dense volume indices and sorted
//     border bindings (:1217-1282), genstep volume IDs mapped to dense indices
//     and the u32 photon offsets (:643-666).
// CUDA's logf/expf/sinf/cosf/rsqrtf become the host's (cuda_on_host.h), so
// results carrying them agree with the device's to a few ulp, not bit for bit.
#include "OptiXTransportDevice.cu"

#include <algorithm>
#include <array>
#include <atomic>
#include <bit>
#include <limits>
#include <string>
#include <thread>
#include <vector>

#include "../include/g4b.h"

namespace Ref = G4GO::Optical;

namespace {

thread_local std::string gRefError;

// --- the OptiX device API over a brute-force triangle scene ----------------

struct Mesh {
    std::vector<Ref::DeviceVector3> vertices;
    std::vector<std::uint32_t> indices;
    std::vector<Ref::DeviceVector3> normals;
    std::vector<std::uint8_t> flags;
};

struct TraceState {
    unsigned int* payload[6]{};
    unsigned int instance{};
    unsigned int primitive{};
    float tmax{};
    bool ignored{};
    uint3 launch{};
};

thread_local TraceState gTrace;
const std::vector<Mesh>* gMeshes{nullptr};  // set while a call runs; read-only for its threads

// Ray-triangle distance in double precision (Moller-Trumbore), or NaN.
double Intersect(const float3& o, const float3& d, const Ref::DeviceVector3& a, const Ref::DeviceVector3& b,
                 const Ref::DeviceVector3& c) {
    const double e1[3]{double(b[0]) - a[0], double(b[1]) - a[1], double(b[2]) - a[2]};
    const double e2[3]{double(c[0]) - a[0], double(c[1]) - a[1], double(c[2]) - a[2]};
    const double dir[3]{d.x, d.y, d.z};
    const double p[3]{dir[1] * e2[2] - dir[2] * e2[1], dir[2] * e2[0] - dir[0] * e2[2], dir[0] * e2[1] - dir[1] * e2[0]};
    const double det{e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2]};
    if (!(std::fabs(det) > 1e-300)) {
        return NAN;
    }
    const double inv{1.0 / det};
    const double s[3]{double(o.x) - a[0], double(o.y) - a[1], double(o.z) - a[2]};
    const double u{(s[0] * p[0] + s[1] * p[1] + s[2] * p[2]) * inv};
    if (u < 0.0 || u > 1.0) {
        return NAN;
    }
    const double q[3]{s[1] * e1[2] - s[2] * e1[1], s[2] * e1[0] - s[0] * e1[2], s[0] * e1[1] - s[1] * e1[0]};
    const double v{(dir[0] * q[0] + dir[1] * q[1] + dir[2] * q[2]) * inv};
    if (v < 0.0 || u + v > 1.0) {
        return NAN;
    }
    return (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) * inv;
}

struct Candidate {
    float t;
    unsigned int instance, primitive;
};

}  // namespace

uint3 optixGetLaunchIndex() { return gTrace.launch; }
unsigned int optixGetInstanceId() { return gTrace.instance; }
unsigned int optixGetPrimitiveIndex() { return gTrace.primitive; }
float optixGetRayTmax() { return gTrace.tmax; }
void optixIgnoreIntersection() { gTrace.ignored = true; }
float3 optixTransformNormalFromObjectToWorldSpace(float3 normal) { return normal; }  // identity instances
unsigned int optixGetPayload_0() { return *gTrace.payload[0]; }
unsigned int optixGetPayload_1() { return *gTrace.payload[1]; }
unsigned int optixGetPayload_2() { return *gTrace.payload[2]; }
unsigned int optixGetPayload_3() { return *gTrace.payload[3]; }
unsigned int optixGetPayload_4() { return *gTrace.payload[4]; }
unsigned int optixGetPayload_5() { return *gTrace.payload[5]; }
void optixSetPayload_0(unsigned int value) { *gTrace.payload[0] = value; }
void optixSetPayload_1(unsigned int value) { *gTrace.payload[1] = value; }
void optixSetPayload_2(unsigned int value) { *gTrace.payload[2] = value; }
void optixSetPayload_3(unsigned int value) { *gTrace.payload[3] = value; }
void optixSetPayload_4(unsigned int value) { *gTrace.payload[4] = value; }
void optixSetPayload_5(unsigned int value) { *gTrace.payload[5] = value; }

void optixTrace(OptixTraversableHandle, float3 origin, float3 direction, float tmin, float tmax, float,
                OptixVisibilityMask, unsigned int rayFlags, unsigned int, unsigned int, unsigned int,
                unsigned int& p0, unsigned int& p1, unsigned int& p2, unsigned int& p3, unsigned int& p4,
                unsigned int& p5) {
    gTrace.payload[0] = &p0;
    gTrace.payload[1] = &p1;
    gTrace.payload[2] = &p2;
    gTrace.payload[3] = &p3;
    gTrace.payload[4] = &p4;
    gTrace.payload[5] = &p5;
    std::vector<Candidate> hits;
    const auto& meshes{*gMeshes};
    for (unsigned int instance{}; instance < meshes.size(); ++instance) {
        const auto& mesh{meshes[instance]};
        for (unsigned int tri{}; tri < mesh.indices.size() / 3U; ++tri) {
            const double t{Intersect(origin, direction, mesh.vertices[mesh.indices[3 * tri]],
                                     mesh.vertices[mesh.indices[3 * tri + 1]], mesh.vertices[mesh.indices[3 * tri + 2]])};
            if (!std::isfinite(t)) {
                continue;
            }
            const auto tf{static_cast<float>(t)};
            if (tf >= tmin && tf <= tmax) {
                hits.push_back({tf, instance, tri});
            }
        }
    }
    // candidates in order of distance, then of instance and triangle
    std::sort(hits.begin(), hits.end(), [](const Candidate& a, const Candidate& b) {
        return a.t != b.t ? a.t < b.t : (a.instance != b.instance ? a.instance < b.instance : a.primitive < b.primitive);
    });
    const bool anyHit{(rayFlags & OPTIX_RAY_FLAG_DISABLE_ANYHIT) == 0U};
    const Candidate* accepted{nullptr};
    for (const auto& hit : hits) {
        if (accepted != nullptr && hit.t > accepted->t) {
            break;
        }
        gTrace.instance = hit.instance;
        gTrace.primitive = hit.primitive;
        gTrace.tmax = hit.t;
        gTrace.ignored = false;
        if (anyHit) {
            Ref::__anyhit__ah();
        }
        if (!gTrace.ignored && accepted == nullptr) {
            accepted = &hit;
            if (!anyHit) {
                break;  // closest hit only: the first at the smallest distance
            }
        }
    }
    if (accepted != nullptr) {
        if ((rayFlags & OPTIX_RAY_FLAG_DISABLE_CLOSESTHIT) == 0U) {
            gTrace.instance = accepted->instance;
            gTrace.primitive = accepted->primitive;
            gTrace.tmax = accepted->t;
            Ref::__closesthit__ch();
        }
    } else {
        Ref::__miss__ms();
    }
}

namespace {

// --- host-side packing ----------------------------------------------------

struct RefScene {
    std::vector<std::vector<float>> storage;  // property arrays the device views point into
    std::vector<Ref::DeviceMaterial> materials;
    std::vector<Ref::DeviceSurface> surfaces;
    std::vector<Mesh> meshes;
    std::vector<Ref::DeviceGeometry> geometries;
    std::vector<Ref::DeviceVolume> volumes;
    std::vector<Ref::DeviceSurfaceBinding> bindings;
    std::vector<std::uint32_t> ids;  // public volume ID of each dense index
    Ref::DeviceScene device{};

    const float* Keep(const float* data, std::uint32_t count) {
        storage.emplace_back(data, data + count);
        return storage.back().data();
    }

    // UploadProperty (OptiXTransportHost.cpp:357-372) with PropertyTable::Constant (Scene.cpp:18-22).
    Ref::DeviceProperty Property(const g4b_property& p) {
        if (p.count == 0 || p.energy_ev == nullptr || p.values == nullptr) {
            return {};
        }
        bool constant{true};
        for (std::uint32_t i{1}; i < p.count; ++i) {
            constant = constant && p.values[i] == p.values[0];
        }
        return {Keep(p.energy_ev, p.count), Keep(p.values, p.count), p.count, constant ? 1U : 0U};
    }

    // UploadSpectrumProperty (OptiXTransportHost.cpp:374-410): normalised trapezoid CDF, last entry 1.
    Ref::DeviceProperty Spectrum(const g4b_property& p) {
        if (p.count == 0 || p.energy_ev == nullptr || p.values == nullptr) {
            return {};
        }
        if (p.count == 1) {
            const float one{1.0F};
            return {Keep(p.energy_ev, 1), Keep(&one, 1), 1U, 0U};
        }
        std::vector<float> cdf(p.count, 0.0F);
        for (std::uint32_t i{1}; i < p.count; ++i) {
            const float width{p.energy_ev[i] - p.energy_ev[i - 1]};
            const float v0{std::max(p.values[i - 1], 0.0F)};
            const float v1{std::max(p.values[i], 0.0F)};
            if (!(width >= 0.0F) || !std::isfinite(width) || !std::isfinite(v0) || !std::isfinite(v1)) {
                return {};
            }
            cdf[i] = cdf[i - 1] + 0.5F * width * (v0 + v1);
        }
        const float integral{cdf.back()};
        if (!(integral > 0.0F) || !std::isfinite(integral)) {
            return {};
        }
        for (auto& value : cdf) {
            value /= integral;
        }
        cdf.back() = 1.0F;
        return {Keep(p.energy_ev, p.count), Keep(cdf.data(), p.count), p.count, 0U};
    }

    std::uint32_t Dense(std::uint32_t id) const {
        if (id == G4B_INVALID_ID) {
            return G4B_INVALID_ID;
        }
        for (std::uint32_t i{}; i < ids.size(); ++i) {
            if (ids[i] == id) {
                return i;
            }
        }
        return G4B_INVALID_ID - 1U;
    }

    bool Build(const g4b_scene& s) {
        if (s.volume_count == 0 || s.volumes == nullptr) {
            gRefError = "empty scene";
            return false;
        }
        storage.reserve(64 + 32 * (s.material_count + s.surface_count));
        for (std::uint32_t m{}; m < s.material_count; ++m) {
            const auto& sm{s.materials[m]};
            Ref::DeviceMaterial material{};
            material.rindex = Property(sm.rindex);
            material.rindexMax = sm.rindex_max;
            if (material.rindexMax == 0.0F) {
                material.rindexMax = 1.0F;
                if (sm.rindex.count != 0) {
                    material.rindexMax = *std::max_element(sm.rindex.values, sm.rindex.values + sm.rindex.count);
                }
            }
            material.groupVelocityMmPerNs = Property(sm.group_velocity_mm_per_ns);
            material.absLengthMm = Property(sm.abs_length_mm);
            if (sm.rayleigh_length_mm.count != 0) {
                gRefError = "the reference's device program has no Rayleigh scattering";
                return false;
            }
            for (int c{}; c < 3; ++c) {
                material.scintillationSpectrum[static_cast<std::size_t>(c)] = Spectrum(sm.scintillation_spectrum[c]);
            }
            materials.push_back(material);
        }
        for (std::uint32_t k{}; k < s.surface_count; ++k) {
            const auto& ss{s.surfaces[k]};
            Ref::DeviceSurface surface{};
            surface.type = ss.type;
            surface.model = ss.model;
            surface.finish = ss.finish;
            surface.modelValue = ss.model_value;
            surface.reflectivity = Property(ss.reflectivity);
            surface.efficiency = Property(ss.efficiency);
            surface.transmittance = Property(ss.transmittance);
            surface.rindex = Property(ss.rindex);
            surface.specularLobe = Property(ss.specular_lobe);
            surface.specularSpike = Property(ss.specular_spike);
            surface.backscatter = Property(ss.backscatter);
            surface.surfaceRoughness = Property(ss.surface_roughness);
            surfaces.push_back(surface);
        }
        const std::uint32_t n{s.volume_count};
        for (std::uint32_t i{}; i < n; ++i) {
            ids.push_back(s.volumes[i].volume_id);
        }
        std::vector<std::array<float, 3>> lo(n), hi(n);
        std::vector<std::uint32_t> parent(n);
        for (std::uint32_t i{}; i < n; ++i) {
            const auto& v{s.volumes[i]};
            parent[i] = Dense(v.parent_volume_id);
            if (parent[i] == G4B_INVALID_ID - 1U || v.material_id >= s.material_count) {
                gRefError = "volume with an unknown parent or material";
                return false;
            }
            for (int a{}; a < 3; ++a) {
                lo[i][a] = static_cast<float>(double(v.center_mm[a]) - double(v.half_size_mm[a]));
                hi[i][a] = static_cast<float>(double(v.center_mm[a]) + double(v.half_size_mm[a]));
            }
        }
        // touching faces: one plane, flagged coincident
        std::vector<std::uint32_t> faceFlags(n, 0U);
        std::vector<bool> mayCoincide(n, false);
        constexpr double tolerance{1.0e-5};
        for (std::uint32_t i{}; i < n; ++i) {
            for (std::uint32_t j{i + 1}; j < n; ++j) {
                const bool sameParent{parent[i] != G4B_INVALID_ID && parent[i] == parent[j]};
                const bool parentChild{parent[i] == j || parent[j] == i};
                if (!sameParent && !parentChild) {
                    continue;
                }
                for (int a{}; a < 3; ++a) {
                    const int u{(a + 1) % 3};
                    const int v{(a + 2) % 3};
                    const double overlapU{std::min<double>(hi[i][u], hi[j][u]) - std::max<double>(lo[i][u], lo[j][u])};
                    const double overlapV{std::min<double>(hi[i][v], hi[j][v]) - std::max<double>(lo[i][v], lo[j][v])};
                    if (!(overlapU > 0.0 && overlapV > 0.0 && overlapU * overlapV > tolerance * tolerance)) {
                        continue;
                    }
                    for (int si{}; si < 2; ++si) {
                        for (int sj{}; sj < 2; ++sj) {
                            if (!parentChild && si == sj) {
                                continue;
                            }
                            const double pi{si == 0 ? lo[i][a] : hi[i][a]};
                            const double pj{sj == 0 ? lo[j][a] : hi[j][a]};
                            if (std::fabs(pi - pj) <= tolerance) {
                                (sj == 0 ? lo[j][a] : hi[j][a]) = static_cast<float>(pi);
                                faceFlags[i] |= 1U << (2 * a + si);
                                faceFlags[j] |= 1U << (2 * a + sj);
                                mayCoincide[i] = mayCoincide[j] = true;
                            }
                        }
                    }
                }
            }
        }
        meshes.resize(n);
        geometries.resize(n);
        for (std::uint32_t i{}; i < n; ++i) {
            auto& mesh{meshes[i]};
            for (int c{}; c < 8; ++c) {  // corner c: bit a set -> hi on axis a
                mesh.vertices.push_back({(c & 1) ? hi[i][0] : lo[i][0], (c & 2) ? hi[i][1] : lo[i][1],
                                         (c & 4) ? hi[i][2] : lo[i][2]});
            }
            for (int a{}; a < 3; ++a) {
                const int u{(a + 1) % 3};
                const int v{(a + 2) % 3};
                for (int side{}; side < 2; ++side) {
                    const auto corner{[&](int bu, int bv) {
                        return static_cast<std::uint32_t>((side << a) | (bu << u) | (bv << v));
                    }};
                    // outward winding: (u, v, a) is right-handed, so u -> v faces +a
                    const std::array<std::uint32_t, 4> quad{corner(0, 0), corner(1, 0), corner(1, 1), corner(0, 1)};
                    const std::array<std::uint32_t, 6> tris{side == 1 ? std::array<std::uint32_t, 6>{
                                                                            quad[0], quad[1], quad[2], quad[0], quad[2], quad[3]}
                                                                      : std::array<std::uint32_t, 6>{
                                                                            quad[0], quad[2], quad[1], quad[0], quad[3], quad[2]}};
                    for (int t{}; t < 2; ++t) {
                        const auto& p0{mesh.vertices[tris[3 * t]]};
                        const auto& p1{mesh.vertices[tris[3 * t + 1]]};
                        const auto& p2{mesh.vertices[tris[3 * t + 2]]};
                        // CreateTriangleNormals (OptiXTransportHost.cpp:1102-1115): unit cross product in double
                        const double e1[3]{double(p1[0]) - p0[0], double(p1[1]) - p0[1], double(p1[2]) - p0[2]};
                        const double e2[3]{double(p2[0]) - p0[0], double(p2[1]) - p0[1], double(p2[2]) - p0[2]};
                        const double c[3]{e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                                          e1[0] * e2[1] - e1[1] * e2[0]};
                        const double length{std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2])};
                        if (!(length > 0.0)) {
                            gRefError = "degenerate box face";
                            return false;
                        }
                        mesh.normals.push_back({static_cast<float>(c[0] / length), static_cast<float>(c[1] / length),
                                                static_cast<float>(c[2] / length)});
                        for (int k{}; k < 3; ++k) {
                            mesh.indices.push_back(tris[3 * t + k]);
                        }
                        mesh.flags.push_back(((faceFlags[i] >> (2 * a + side)) & 1U) != 0U ? 1U : 0U);
                    }
                }
            }
            geometries[i].mesh = {mesh.vertices.data(), mesh.indices.data(), mesh.normals.data(), mesh.flags.data(),
                                  static_cast<std::uint32_t>(mesh.vertices.size()),
                                  static_cast<std::uint32_t>(mesh.indices.size() / 3)};
            const auto& v{s.volumes[i]};
            Ref::DeviceVolume volume{};
            volume.volumeID = i;
            volume.geometryID = i;
            volume.materialID = v.material_id;
            volume.parentVolumeID = parent[i];
            volume.skinSurfaceID = v.skin_surface_id;
            volume.sensorID = v.sensor_id;
            volume.mayHaveCoincidentBoundary = mayCoincide[i] ? 1U : 0U;
            volumes.push_back(volume);
        }
        for (std::uint32_t b{}; b < s.binding_count; ++b) {
            const auto from{Dense(s.bindings[b].from_volume_id)};
            const auto to{Dense(s.bindings[b].to_volume_id)};
            if (from >= G4B_INVALID_ID - 1U || to >= G4B_INVALID_ID - 1U) {
                gRefError = "binding with an unknown volume";
                return false;
            }
            bindings.push_back({from, to, s.bindings[b].surface_id});
        }
        std::sort(bindings.begin(), bindings.end(), [](const auto& a, const auto& b) {
            return a.fromVolumeID != b.fromVolumeID ? a.fromVolumeID < b.fromVolumeID : a.toVolumeID < b.toVolumeID;
        });
        const auto world{Dense(s.world_volume_id)};
        if (world >= G4B_INVALID_ID - 1U) {
            gRefError = "no world volume";
            return false;
        }
        device = {materials.data(), static_cast<std::uint32_t>(materials.size()), surfaces.data(),
                  static_cast<std::uint32_t>(surfaces.size()), geometries.data(),
                  static_cast<std::uint32_t>(geometries.size()), volumes.data(),
                  static_cast<std::uint32_t>(volumes.size()), bindings.data(),
                  static_cast<std::uint32_t>(bindings.size()), world};
        return true;
    }
};

// Genstep as the device record, volume ID mapped to its dense index.
bool ToDevice(const RefScene& scene, const g4b_optical_emission& in, Ref::DeviceOpticalEmission& out) {
    static_assert(sizeof(g4b_optical_emission) == sizeof(Ref::DeviceOpticalEmission));
    out = std::bit_cast<Ref::DeviceOpticalEmission>(in);
    out.volumeID = scene.Dense(in.volume_id);
    if (out.volumeID >= G4B_INVALID_ID - 1U) {
        gRefError = "genstep in an unknown volume";
        return false;
    }
    return true;
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return gRefError.c_str(); }

// Uniform (OptiXTransportDevice.cu:254-286).
float ref_uniform(uint64_t seed, uint64_t photonKey, uint32_t bounce, uint32_t process, uint32_t draw) {
    return Ref::Uniform(seed, photonKey, bounce, process, draw);
}

// SampleProperty (:198-216) on a caller's table.
float ref_sample_property(const float* energy, const float* values, uint32_t count, uint32_t constant, float x,
                          float defaultValue) {
    const Ref::DeviceProperty property{energy, values, count, constant};
    return Ref::SampleProperty(property, x, defaultValue);
}

// SampleSpectrum (:322-344) on a caller's CDF.
float ref_sample_spectrum(const float* energy, const float* cdf, uint32_t count, float u) {
    const Ref::DeviceProperty spectrum{energy, cdf, count, 0U};
    return Ref::SampleSpectrum(spectrum, u);
}

// The spectrum CDF as the shim packs it (trapezoid, normalised, last = 1); 0 if rejected.
uint32_t ref_spectrum_cdf(const float* energy, const float* values, uint32_t count, float* cdfOut) {
    RefScene scene;
    const auto packed{scene.Spectrum(g4b_property{energy, values, count, 0U})};
    if (packed.count == 0) {
        return 0U;
    }
    std::memcpy(cdfOut, packed.values, sizeof(float) * packed.count);
    return packed.count;
}

// GeneratePhoton (:346-481) for photon `local[i]` of genstep `emissionIndex[i]`.
// Each output row: position[3], direction[3], polarization[3], energy; time
// separately (the reference keeps it in float).
int ref_generate(const g4b_scene* sceneDesc, uint64_t seed, const g4b_optical_emission* emissions,
                 uint32_t emissionCount, const uint32_t* emissionIndex, const uint32_t* local, uint32_t n,
                 float* out, double* timeOut) {
    RefScene scene;
    if (sceneDesc == nullptr || !scene.Build(*sceneDesc)) {
        return -1;
    }
    gMeshes = &scene.meshes;
    Ref::gLaunchParams = {};
    Ref::gLaunchParams.scene = scene.device;
    Ref::gLaunchParams.seed = seed;
    for (uint32_t i{}; i < n; ++i) {
        if (emissionIndex[i] >= emissionCount) {
            gRefError = "emission index out of range";
            return -1;
        }
        Ref::DeviceOpticalEmission emission{};
        if (!ToDevice(scene, emissions[emissionIndex[i]], emission)) {
            return -1;
        }
        const auto photon{Ref::GeneratePhoton(emission, emission.firstPhotonID + local[i], local[i], 0U)};
        const float row[10]{photon.positionMm[0], photon.positionMm[1], photon.positionMm[2],
                            photon.direction[0], photon.direction[1], photon.direction[2],
                            photon.polarization[0], photon.polarization[1], photon.polarization[2],
                            photon.energyEv};
        std::memcpy(out + 10ULL * i, row, sizeof(row));
        timeOut[i] = photon.timeNs;
    }
    gMeshes = nullptr;
    return 0;
}

typedef struct ref_result {
    uint32_t* fate;          /* [photon_end - photon_begin]: outcome | bounces << 3 (1 det, 2 abs, 3 esc, 4 trunc, 5 inv) */
    uint32_t* zero_steps;    /* [photon_end - photon_begin] */
    g4b_photon_detection* detections; /* [photon_end - photon_begin] capacity; flattened order */
    uint64_t detection_count;
    g4b_event_statistics* event_statistics; /* [event_count] */
    g4b_statistics statistics;
    uint64_t total_bounce_count;
    uint64_t coincident_candidate_trace_count;
    uint64_t coincident_candidate_hit_count;
} ref_result;

// __raygen__rg (:660-941) once per photon of [photonBegin, photonEnd) of the
// batch, on `threads` host threads, each photon with its own cleared run
// counters so its fate can be read from them.
int ref_transport(const g4b_scene* sceneDesc, const g4b_config* config, const g4b_optical_emission* emissions,
                  uint32_t emissionCount, const uint32_t* eventIDs, uint32_t eventCount,
                  const uint32_t* emissionEventIndices, uint32_t threads, uint64_t photonBegin, uint64_t photonEnd,
                  ref_result* result) {
    RefScene scene;
    if (sceneDesc == nullptr || config == nullptr || result == nullptr || !scene.Build(*sceneDesc)) {
        if (sceneDesc == nullptr || config == nullptr || result == nullptr) {
            gRefError = "null argument";
        }
        return -1;
    }
    std::vector<Ref::DeviceOpticalEmission> device(emissionCount);
    std::vector<std::uint32_t> offsets(emissionCount + 1U, 0U);
    std::uint64_t total{};
    for (uint32_t e{}; e < emissionCount; ++e) {
        if (!ToDevice(scene, emissions[e], device[e])) {
            return -1;
        }
        if (emissionEventIndices[e] >= eventCount || emissions[e].event_id != eventIDs[emissionEventIndices[e]]) {
            gRefError = "emission event index does not match event ID";
            return -1;
        }
        total += emissions[e].photon_count;
        if (total > std::numeric_limits<std::uint32_t>::max()) {
            gRefError = "more than 2^32 photons";
            return -1;
        }
        offsets[e + 1U] = static_cast<std::uint32_t>(total);
    }
    if (photonEnd == 0 || photonEnd > total) {
        photonEnd = total;
    }
    if (photonBegin > photonEnd) {
        photonBegin = photonEnd;
    }
    std::vector<Ref::DevicePhotonHit> hits(total);
    std::vector<std::uint32_t> hitFlags(total, 0U);
    threads = std::max<uint32_t>(threads == 0 ? std::thread::hardware_concurrency() : threads, 1U);
    std::vector<std::vector<Ref::DeviceEventTransportStats>> eventStats(
        threads, std::vector<Ref::DeviceEventTransportStats>(eventCount));
    std::vector<Ref::DeviceTransportStats> runStats(threads);
    std::atomic<uint64_t> next{photonBegin};
    gMeshes = &scene.meshes;
    const auto worker{[&](uint32_t t) {
        Ref::gLaunchParams = {};
        auto& p{Ref::gLaunchParams};
        p.emissions = device.data();
        p.emissionEventIndices = emissionEventIndices;
        p.emissionOffsets = offsets.data();
        p.hits = hits.data();
        p.hitFlags = hitFlags.data();
        p.eventStats = eventStats[t].data();
        p.scene = scene.device;
        p.seed = config->seed;
        p.maxBounceCount = config->max_bounces_per_photon == 0 ? 4096U : config->max_bounces_per_photon;
        p.emissionCount = emissionCount;
        p.eventCount = eventCount;
        p.photonCount = static_cast<std::uint32_t>(total);
        p.enablePerformanceDiagnostics = 1U;
        p.boundaryEpsilonMm = config->boundary_tolerance_mm > 0.0F ? config->boundary_tolerance_mm : 1.0e-4F;
        Ref::DeviceTransportStats photon{};
        p.stats = &photon;
        for (;;) {
            const uint64_t slot{next.fetch_add(1)};
            if (slot >= photonEnd) {
                break;
            }
            photon = {};
            gTrace.launch = uint3{static_cast<unsigned int>(slot), 0U, 0U};
            Ref::__raygen__rg();
            const uint32_t outcome{photon.detectedCount != 0 ? 1U : photon.absorbedCount != 0 ? 2U
                                   : photon.escapedCount != 0 ? 3U : photon.truncatedCount != 0 ? 4U : 5U};
            const uint64_t i{slot - photonBegin};
            if (result->fate != nullptr) {
                result->fate[i] = outcome | static_cast<uint32_t>(photon.totalBounceCount << 3U);
            }
            if (result->zero_steps != nullptr) {
                result->zero_steps[i] = static_cast<uint32_t>(photon.zeroStepCount);
            }
            auto& run{runStats[t]};
            run.detectedCount += photon.detectedCount;
            run.absorbedCount += photon.absorbedCount;
            run.escapedCount += photon.escapedCount;
            run.truncatedCount += photon.truncatedCount;
            run.maxBounceCount = std::max(run.maxBounceCount, photon.maxBounceCount);
            run.invalidStateCount += photon.invalidStateCount;
            run.zeroStepCount += photon.zeroStepCount;
            run.totalBounceCount += photon.totalBounceCount;
            run.coincidentCandidateTraceCount += photon.coincidentCandidateTraceCount;
            run.coincidentCandidateHitCount += photon.coincidentCandidateHitCount;
        }
    }};
    std::vector<std::thread> pool;
    for (uint32_t t{1}; t < threads; ++t) {
        pool.emplace_back(worker, t);
    }
    worker(0);
    for (auto& thread : pool) {
        thread.join();
    }
    gMeshes = nullptr;
    // CompleteOldestBatch's conversion of the flagged hits (OptiXTransportHost.cpp:862-874), in slot order
    result->detection_count = 0;
    for (uint64_t slot{photonBegin}; slot < photonEnd; ++slot) {
        if (hitFlags[slot] == 0U) {
            continue;
        }
        const auto& hit{hits[slot]};
        g4b_photon_detection record{};
        for (int k{}; k < 3; ++k) {
            record.position_mm[k] = hit.positionMm[static_cast<std::size_t>(k)];
            record.direction[k] = hit.direction[static_cast<std::size_t>(k)];
        }
        record.time_ns = hit.timeNs;
        record.energy_ev = hit.energyEv;
        record.event_id = hit.eventID;
        record.photon_id = hit.photonID;
        record.sensor_id = hit.sensorID;
        if (result->detections != nullptr) {
            result->detections[result->detection_count] = record;
        }
        ++result->detection_count;
    }
    g4b_statistics run{};
    result->total_bounce_count = 0;
    result->coincident_candidate_trace_count = 0;
    result->coincident_candidate_hit_count = 0;
    for (uint32_t t{}; t < threads; ++t) {
        run.detected_count += runStats[t].detectedCount;
        run.absorbed_count += runStats[t].absorbedCount;
        run.escaped_count += runStats[t].escapedCount;
        run.truncated_count += runStats[t].truncatedCount;
        run.max_bounce_count = std::max<uint64_t>(run.max_bounce_count, runStats[t].maxBounceCount);
        run.invalid_state_count += runStats[t].invalidStateCount;
        run.zero_step_count += runStats[t].zeroStepCount;
        result->total_bounce_count += runStats[t].totalBounceCount;
        result->coincident_candidate_trace_count += runStats[t].coincidentCandidateTraceCount;
        result->coincident_candidate_hit_count += runStats[t].coincidentCandidateHitCount;
    }
    run.captured_count = total;
    result->statistics = run;
    if (result->event_statistics != nullptr) {
        for (uint32_t ev{}; ev < eventCount; ++ev) {
            g4b_event_statistics out{};
            out.event_id = eventIDs[ev];
            for (uint32_t t{}; t < threads; ++t) {
                const auto& c{eventStats[t][ev]};
                out.statistics.detected_count += c.detectedCount;
                out.statistics.absorbed_count += c.absorbedCount;
                out.statistics.escaped_count += c.escapedCount;
                out.statistics.truncated_count += c.truncatedCount;
                out.statistics.max_bounce_count = std::max<uint64_t>(out.statistics.max_bounce_count, c.maxBounceCount);
                out.statistics.invalid_state_count += c.invalidStateCount;
                out.statistics.zero_step_count += c.zeroStepCount;
            }
            result->event_statistics[ev] = out;
        }
        for (uint32_t e{}; e < emissionCount; ++e) {
            result->event_statistics[emissionEventIndices[e]].statistics.captured_count += emissions[e].photon_count;
        }
    }
    return 0;
}

}  // extern "C"

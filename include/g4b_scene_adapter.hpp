// g4b_scene_adapter.hpp - the reference's exported Scene as an analytic box scene.
//
// G4GO's Geant4SceneExporter turns the Geant4 world into a Scene of triangle
// meshes with per-volume transforms (include/g4go/optical/Scene.hpp:94-163,
// src/optical/geant4/Geant4SceneExporter.cpp:192-254). B200 has no RT cores and
// the engine intersects axis-aligned boxes analytically, so this header
// recognises each volume's mesh as a box: the vertices, taken to world
// coordinates by the volume's transform, must sit on the eight corners of
// their bounding box, and the transform must be a signed axis permutation.
// Anything else (rotated or non-box solids) is rejected with
// std::invalid_argument, as the exporter rejects solids it cannot mesh
// (Geant4SceneExporter.cpp:501-503). Materials, surfaces, skin surfaces,
// sensors and border bindings map field by field; property tables are
// borrowed from the Scene (g4b_set_scene copies them), so the Scene must
// outlive the g4b_scene until it has been set.
//
// Header-only and generic: any type with the reference Scene's accessors
// (Materials(), Surfaces(), Geometries(), Volumes(), SurfaceBindings(),
// WorldVolumeID()) and field names works, so the reference's own Scene passes
// through without Geant4 or CLHEP headers here.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "g4b.h"

namespace g4b {

class BoxScene final {
public:
    template<class Scene>
    explicit BoxScene(const Scene& scene) {
        for (const auto& material : scene.Materials()) {
            g4b_material m{};
            m.rindex = Property(material.rindex);
            m.rindex_max = material.rindexMax;
            m.group_velocity_mm_per_ns = Property(material.groupVelocityMmPerNs);
            m.abs_length_mm = Property(material.absLengthMm);
            for (std::size_t k{}; k < 3; ++k) {
                m.scintillation_spectrum[k] = Property(material.scintillationSpectrum[k]);
            }
            fMaterials.push_back(m);
        }
        for (const auto& surface : scene.Surfaces()) {
            g4b_surface s{};
            s.type = static_cast<std::uint8_t>(surface.type);
            s.model = static_cast<std::uint8_t>(surface.model);
            s.finish = static_cast<std::uint8_t>(surface.finish);
            s.model_value = surface.modelValue;
            s.reflectivity = Property(surface.reflectivity);
            s.efficiency = Property(surface.efficiency);
            s.transmittance = Property(surface.transmittance);
            s.rindex = Property(surface.rindex);
            s.specular_lobe = Property(surface.specularLobe);
            s.specular_spike = Property(surface.specularSpike);
            s.backscatter = Property(surface.backscatter);
            s.surface_roughness = Property(surface.surfaceRoughness);
            fSurfaces.push_back(s);
        }
        const auto& geometries{scene.Geometries()};
        for (const auto& volume : scene.Volumes()) {
            if (volume.geometryID >= geometries.size()) {
                throw std::invalid_argument("volume " + volume.name + " has no geometry");
            }
            g4b_volume v{};
            v.volume_id = volume.volumeID;
            v.material_id = volume.materialID;
            v.parent_volume_id = volume.parentVolumeID;
            v.skin_surface_id = volume.skinSurfaceID;
            v.sensor_id = volume.sensorID;
            Box(volume.name, geometries[volume.geometryID].mesh.verticesMm, volume.transform, v);
            fVolumes.push_back(v);
        }
        for (const auto& binding : scene.SurfaceBindings()) {
            fBindings.push_back({binding.fromVolumeID, binding.toVolumeID, binding.surfaceID});
        }
        fScene.materials = fMaterials.data();
        fScene.material_count = static_cast<std::uint32_t>(fMaterials.size());
        fScene.surfaces = fSurfaces.data();
        fScene.surface_count = static_cast<std::uint32_t>(fSurfaces.size());
        fScene.volumes = fVolumes.data();
        fScene.volume_count = static_cast<std::uint32_t>(fVolumes.size());
        fScene.bindings = fBindings.data();
        fScene.binding_count = static_cast<std::uint32_t>(fBindings.size());
        fScene.world_volume_id = scene.WorldVolumeID();
    }

    BoxScene(const BoxScene&) = delete;
    BoxScene& operator=(const BoxScene&) = delete;

    const g4b_scene& Get() const { return fScene; }
    const std::vector<g4b_volume>& Volumes() const { return fVolumes; }

private:
    template<class Table>
    static g4b_property Property(const Table& table) {
        g4b_property p{};
        if (table.energyEv.size() != table.values.size()) {
            throw std::invalid_argument("property table with mismatched energy and value counts");
        }
        p.energy_ev = table.energyEv.data();
        p.values = table.values.data();
        p.count = static_cast<std::uint32_t>(table.energyEv.size());
        return p;
    }

    // World-space axis-aligned box of a mesh, or std::invalid_argument.
    template<class Vertices, class Transform>
    static void Box(const std::string& name, const Vertices& vertices, const Transform& transform, g4b_volume& out) {
        const auto& r{transform.rotation};
        const double m[3][3]{{r.xx, r.xy, r.xz}, {r.yx, r.yy, r.yz}, {r.zx, r.zy, r.zz}};
        constexpr double kUnit{1.0e-6};
        for (int i{}; i < 3; ++i) {
            int rowOnes{0};
            int columnOnes{0};
            for (int j{}; j < 3; ++j) {
                const bool rowUnit{std::fabs(std::fabs(m[i][j]) - 1.0) <= kUnit};
                const bool rowZero{std::fabs(m[i][j]) <= kUnit};
                const bool columnUnit{std::fabs(std::fabs(m[j][i]) - 1.0) <= kUnit};
                if (!rowUnit && !rowZero) {
                    throw std::invalid_argument("volume " + name + " is rotated off the axes; only axis-aligned boxes "
                                                "are supported");
                }
                rowOnes += rowUnit ? 1 : 0;
                columnOnes += columnUnit ? 1 : 0;
            }
            if (rowOnes != 1 || columnOnes != 1) {
                throw std::invalid_argument("volume " + name + " has a transform that is not an axis permutation");
            }
        }
        if (vertices.size() < 8U) {
            throw std::invalid_argument("volume " + name + " is not a box (fewer than 8 vertices)");
        }
        const double t[3]{static_cast<double>(transform.translationMm.x()),
                          static_cast<double>(transform.translationMm.y()),
                          static_cast<double>(transform.translationMm.z())};
        std::vector<std::array<double, 3>> world;
        world.reserve(vertices.size());
        std::array<double, 3> lo{HUGE_VAL, HUGE_VAL, HUGE_VAL};
        std::array<double, 3> hi{-HUGE_VAL, -HUGE_VAL, -HUGE_VAL};
        for (const auto& vertex : vertices) {
            const double p[3]{static_cast<double>(vertex.x()), static_cast<double>(vertex.y()),
                              static_cast<double>(vertex.z())};
            std::array<double, 3> w{};
            for (int i{}; i < 3; ++i) {
                w[i] = m[i][0] * p[0] + m[i][1] * p[1] + m[i][2] * p[2] + t[i];
                lo[i] = std::min(lo[i], w[i]);
                hi[i] = std::max(hi[i], w[i]);
            }
            world.push_back(w);
        }
        // every vertex on a corner of the bounding box, and every corner used
        unsigned corners{0U};
        for (const auto& w : world) {
            unsigned corner{0U};
            for (int i{}; i < 3; ++i) {
                const double tolerance{1.0e-6 * std::max(1.0, std::fabs(hi[i]) + std::fabs(lo[i]))};
                if (std::fabs(w[i] - hi[i]) <= tolerance) {
                    corner |= 1U << i;
                } else if (std::fabs(w[i] - lo[i]) > tolerance) {
                    throw std::invalid_argument("volume " + name + " is not a box (a vertex inside its bounds)");
                }
            }
            corners |= 1U << corner;
        }
        if (corners != 0xffU) {
            throw std::invalid_argument("volume " + name + " is not a box (a corner is missing)");
        }
        for (int i{}; i < 3; ++i) {
            if (!(hi[i] > lo[i])) {
                throw std::invalid_argument("volume " + name + " has a flat box");
            }
            out.center_mm[i] = static_cast<float>(0.5 * (lo[i] + hi[i]));
            out.half_size_mm[i] = static_cast<float>(0.5 * (hi[i] - lo[i]));
        }
    }

    std::vector<g4b_material> fMaterials;
    std::vector<g4b_surface> fSurfaces;
    std::vector<g4b_volume> fVolumes;
    std::vector<g4b_surface_binding> fBindings;
    g4b_scene fScene{};
};

}  // namespace g4b

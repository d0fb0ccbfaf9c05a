// ref_boundary_shim.cpp - C entry points over the reference's own boundary
// physics, compiled from the reference tree where it lies
// (src/optical/optix/OptiXBoundaryPhysics.cuh, included through -I; see
// oracle/Makefile). TEST INFRASTRUCTURE ONLY: it pins the CPU oracle's
// restatement of ComputeFresnel, ClassifySurface, EvaluateAbsorption and
// SampleLambertian to the reference's code.
#include "OptiXBoundaryPhysics.cuh"

namespace Physics = G4GO::Optical::BoundaryPhysics;
using G4GO::Optical::DeviceVector3;

extern "C" {

void ref_fresnel(const float d[3], const float p[3], const float n[3], float indexFrom, float indexTo, float out[14]) {
    const auto r{Physics::ComputeFresnel(DeviceVector3{d[0], d[1], d[2]}, DeviceVector3{p[0], p[1], p[2]},
                                         DeviceVector3{n[0], n[1], n[2]}, indexFrom, indexTo)};
    const DeviceVector3* vectors[4]{&r.reflectedDirection, &r.transmittedDirection, &r.reflectedPolarization,
                                    &r.transmittedPolarization};
    for (int k = 0; k < 4; ++k) {
        for (int c = 0; c < 3; ++c) {
            out[3 * k + c] = vectors[k]->at(c);
        }
    }
    out[12] = r.transmittance;
    out[13] = r.totalInternalReflection ? 1.0F : 0.0F;
}

int ref_classify_surface(float reflectivity, float transmittance, int hasR, int hasT, float sample) {
    return static_cast<int>(Physics::ClassifySurface(reflectivity, transmittance, hasR != 0, hasT != 0, sample));
}

int ref_evaluate_absorption(float efficiency, int sensor, float sample) {
    return static_cast<int>(Physics::EvaluateAbsorption(efficiency, sensor != 0, sample));
}

void ref_lambertian(const float n[3], float radial, float azimuth, float out[3]) {
    const auto v{Physics::SampleLambertian(DeviceVector3{n[0], n[1], n[2]}, radial, azimuth)};
    out[0] = v.at(0);
    out[1] = v.at(1);
    out[2] = v.at(2);
}

}  // extern "C"

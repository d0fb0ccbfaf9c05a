// optix_device.h stand-in: the dozen OptiX device-API names that the
// reference's device program (src/optical/optix/OptiXTransportDevice.cu)
// calls, declared for a host build. TEST INFRASTRUCTURE ONLY.
//
// The definitions live in oracle/ref_transport_shim.cpp: optixTrace
// intersects the ray with every triangle of every instance of the scene the
// shim built (no acceleration structure: the scenes are a few boxes), and
// calls the program's own __closesthit__ch, __anyhit__ah and __miss__ms the
// way an OptiX pipeline would; the getters and setters read and write that
// trace's hit and payload. The ray-flag values are this file's own; only
// their names matter to the program.
#ifndef G4B_REF_OPTIX_DEVICE_H
#define G4B_REF_OPTIX_DEVICE_H

using OptixTraversableHandle = unsigned long long;
using OptixVisibilityMask = unsigned int;

enum OptixRayFlags : unsigned int {
    OPTIX_RAY_FLAG_NONE = 0U,
    OPTIX_RAY_FLAG_DISABLE_ANYHIT = 1U << 0U,
    OPTIX_RAY_FLAG_ENFORCE_ANYHIT = 1U << 1U,
    OPTIX_RAY_FLAG_DISABLE_CLOSESTHIT = 1U << 2U,
};

uint3 optixGetLaunchIndex();
unsigned int optixGetInstanceId();
unsigned int optixGetPrimitiveIndex();
float optixGetRayTmax();
void optixIgnoreIntersection();
float3 optixTransformNormalFromObjectToWorldSpace(float3 normal);

unsigned int optixGetPayload_0();
unsigned int optixGetPayload_1();
unsigned int optixGetPayload_2();
unsigned int optixGetPayload_3();
unsigned int optixGetPayload_4();
unsigned int optixGetPayload_5();
void optixSetPayload_0(unsigned int value);
void optixSetPayload_1(unsigned int value);
void optixSetPayload_2(unsigned int value);
void optixSetPayload_3(unsigned int value);
void optixSetPayload_4(unsigned int value);
void optixSetPayload_5(unsigned int value);

void optixTrace(OptixTraversableHandle handle, float3 origin, float3 direction, float tmin, float tmax,
                float rayTime, OptixVisibilityMask visibilityMask, unsigned int rayFlags, unsigned int sbtOffset,
                unsigned int sbtStride, unsigned int missSbtIndex, unsigned int& payload0, unsigned int& payload1,
                unsigned int& payload2, unsigned int& payload3, unsigned int& payload4, unsigned int& payload5);

#endif

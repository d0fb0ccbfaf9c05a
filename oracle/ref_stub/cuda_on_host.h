// cuda_on_host.h - the CUDA language pieces that the reference's device
// program uses, given host meanings so that g++ can compile it unmodified.
// TEST INFRASTRUCTURE ONLY (force-included by oracle/Makefile when it builds
// oracle/_ref/libref_transport.so).
//
//   - __device__, __global__, __host__ and __forceinline__ become ordinary
//     (inline) functions;
//   - __constant__ becomes thread_local: the one constant-memory object, the
//     launch parameters, is then per host thread, so threads can run photons
//     with launch parameters (statistics buffers) of their own;
//   - float3 / uint3 / make_float3, the bit casts and the 64-bit atomics are
//     written here from their documented meaning;
//   - rsqrtf is 1/sqrtf (the device's is an approximation within 2 ulp).
#ifndef G4B_REF_CUDA_ON_HOST_H
#define G4B_REF_CUDA_ON_HOST_H

#include <math.h>

#include <cmath>
#include <cstdint>
#include <cstring>

#define __device__
#define __global__
#define __host__
#define __forceinline__ inline
#define __constant__ thread_local

struct float3 {
    float x, y, z;
};

struct uint3 {
    unsigned int x, y, z;
};

inline float3 make_float3(float x, float y, float z) { return float3{x, y, z}; }

inline unsigned int __float_as_uint(float value) {
    unsigned int bits;
    std::memcpy(&bits, &value, sizeof(bits));
    return bits;
}

inline float __uint_as_float(unsigned int bits) {
    float value;
    std::memcpy(&value, &bits, sizeof(value));
    return value;
}

inline float rsqrtf(float value) { return 1.0F / sqrtf(value); }

inline unsigned long long atomicAdd(unsigned long long* address, unsigned long long value) {
    return __atomic_fetch_add(address, value, __ATOMIC_RELAXED);
}

inline unsigned long long atomicMax(unsigned long long* address, unsigned long long value) {
    unsigned long long seen{__atomic_load_n(address, __ATOMIC_RELAXED)};
    while (seen < value &&
           !__atomic_compare_exchange_n(address, &seen, value, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
    }
    return seen;
}

#endif

// kernels.h - host-side entry points into the engine's CUDA kernels.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "engine_layout.h"

namespace g4b {

enum KernelPrecision : int { kFP32 = 0, kFP64 = 1 };
enum KernelForm : int { kBatched = 0, kPlain = 1, kWithDiagnostics = 2, kPregenerated = 4, kParkedQueue = 8 };

// The transport kernel for (precision, form), as a function pointer usable in
// cudaLaunchKernel and in graph kernel nodes. `form` may carry
// kWithDiagnostics (the variant that also counts coincident-face retraces)
// and, for the batched FP32 form, kPregenerated (photons read from the
// photon store instead of generated in the loop), with kParkedQueue too
// (photons read from the wave's queue of parked photons).
const void* TransportKernel(int precision, int form);
const void* GenerateKernel();
const void* ZeroCountersKernel();

// Raises the dynamic shared-memory limit of every transport kernel.
cudaError_t ConfigureTransportKernels(std::size_t sharedBytes);

cudaError_t TransportOccupancy(int precision, int form, int blockSize, std::size_t sharedBytes, int* blocksPerSM);

cudaError_t LaunchZeroCounters(EventCounters* events, std::uint32_t eventCount, RunCounters* run, cudaStream_t stream);

cudaError_t LaunchTransport(const LaunchParams& params, int precision, int form, unsigned grid, unsigned block,
                            std::size_t sharedBytes, cudaStream_t stream);

// Generation pass of the batched FP32 form: fills params.store with the
// photons [photonBegin, photonEnd) (256-thread blocks, the scene in shared
// memory).
cudaError_t LaunchGenerate(const LaunchParams& params, unsigned grid, std::size_t sharedBytes, cudaStream_t stream);

// Ordered compaction: orders `count` hits by their flattened-photon slot
// (the order cub::DeviceSelect::Flagged gives the reference,
// src/optical/optix/OptiXHitCompaction.cu:23-30) and writes 48-byte
// detection records. bitmap: ceil(photons/32) words; prefix: one word per
// bitmap word; blockSums: ceil(words/1024) + 1 words.
cudaError_t LaunchOrderHits(const HitColumns& hits, unsigned long long count, std::uint32_t photonCount,
                            std::uint32_t* bitmap, std::uint32_t* prefix, std::uint32_t* blockSums,
                            void* detectionsOut, bool ordered, cudaStream_t stream);

// Ordering of one wave's hits, after its transport: the wave's hits are rows
// [0, *count) of `region` (its own region of the hit buffer; a count above
// region.capacity means the region overflowed and only its rows are read),
// its slots lie in [slotBegin, slotEnd) (slotBegin a multiple of 32). The
// wave's records go to detectionsOut from row outRows[0] on, in slot order
// within the wave; outRows[1] = outRows[0] + the rows written, and run gets
// the wave's count added to hitCount and folded into maxWaveHits. Calls for
// consecutive waves must run in wave order (they share blockSums and chain
// outRows). Six launches when ordered (after a bitmap-range clear), two
// otherwise.
cudaError_t LaunchOrderWaveHits(const HitColumns& region, const unsigned long long* count,
                                unsigned long long* outRows, RunCounters* run, std::uint32_t slotBegin,
                                std::uint32_t slotEnd, std::uint32_t* bitmap, std::uint32_t* prefix,
                                std::uint32_t* blockSums, void* detectionsOut, bool ordered, unsigned grid,
                                cudaStream_t stream);

// Ordering of caller-owned detection records by a unique slot key below
// slotLimit (at most kStaticOrderMaxSlots) with all scratch in one array
// compiled into the library. StaticOrderScratch gives that array's address on
// the current device. LaunchOrderRecordsStatic enqueues the ranking on
// `stream`, copies the count of rejected keys (out of range or repeated) to
// *statusHost and waits for the stream. Calls that overlap in time on one
// device share the array and race.
constexpr std::uint32_t kStaticOrderMaxSlots{1U << 24};
cudaError_t StaticOrderScratch(std::uint32_t** scratch);
cudaError_t LaunchOrderRecordsStatic(const void* records, const std::uint32_t* keys, unsigned long long count,
                                     std::uint32_t slotLimit, std::uint32_t* scratch, void* out,
                                     std::uint32_t* statusHost, cudaStream_t stream);

// Gradient replay over the photons [photonBegin, photonEnd) of the last
// transport: each one is regenerated and re-transported from its RNG counters
// with dual numbers, alternate branches of its Fresnel choices and of its
// exits near box edges (within edgeBand mm, or the distance a fast edge moves
// over +-edgeIndexWindow in n; edgeBand 0: no edge term) transported when an
// index target is set, and its derivative terms summed into `sums`.
cudaError_t LaunchGradientReplay(const LaunchParams& params, int precision, std::uint32_t indexMaterial,
                                 std::uint32_t absMaterial, std::uint32_t reflectivitySurface, float edgeBand,
                                 float edgeIndexWindow, unsigned grid, std::size_t sharedBytes, GradientSums* sums,
                                 cudaStream_t stream);

cudaError_t LaunchEvalFresnel(int precision, std::uint32_t n, const double* in, double* out, cudaStream_t stream);
cudaError_t LaunchEvalLambertian(int precision, std::uint32_t n, const double* in, double* out, cudaStream_t stream);
cudaError_t LaunchEvalMath(std::uint32_t kind, std::uint32_t n, const float* in, float* out, cudaStream_t stream);
cudaError_t LaunchEvalUniform(std::uint32_t n, unsigned long long seed, const unsigned long long* keys,
                              const std::uint32_t* counters, float* out, cudaStream_t stream);

}  // namespace g4b

// transport_kernels.cu - the engine's CUDA kernels for sm_100a.
//
// TransportBatched: one persistent launch per batch. Every warp pulls chunks
// of flattened photon indices from a device work queue (one atomic ticket per
// chunk), generates them 32 at a time into a shared-memory photon queue, and
// refills any idle lane from that queue in every iteration, so warps stay full
// while histories of a few to thousands of bounces finish at different times. Gensteps are read as 8 x 16-byte loads; the scene lives in shared
// memory; detections are compacted with one atomic per warp into a
// structure-of-arrays hit buffer; event counters accumulate per lane and are
// flushed once per event change.
//
// TransportPlain: one thread per photon over one event's photons, the launch
// layout of the reference's __raygen__rg (OptiXTransportDevice.cu:660-941).
//
// Both share the same generation and bounce code (g4b_device.cuh).

#include <cstdint>

#include <cuda_runtime.h>

#include "engine_layout.h"
#include "g4b_device.cuh"
#include "kernels.h"

namespace g4b {

using namespace dev;

namespace {

constexpr unsigned kFullMask = 0xffffffffU;

extern __shared__ __align__(16) unsigned char gShared[];

__device__ __forceinline__ void LoadScene(const LaunchParams& p) {
    const uint4* source{reinterpret_cast<const uint4*>(p.scene)};
    uint4* destination{reinterpret_cast<uint4*>(gShared)};
    const std::uint32_t words{p.sceneBytes / 16U};
    for (std::uint32_t i = threadIdx.x; i < words; i += blockDim.x) {
        destination[i] = source[i];
    }
    __syncthreads();
}

// Event counters of the event a lane is currently working on; flushed with
// global atomics when the lane moves to another event and at the end.
struct LaneCounters {
    std::uint32_t eventIndex;
    std::uint32_t detected, absorbed, escaped, truncated, invalid, zeroStep, maxBounce;

    __device__ __forceinline__ void Reset() {
        detected = absorbed = escaped = truncated = invalid = zeroStep = maxBounce = 0U;
    }
    __device__ __forceinline__ void Flush(EventCounters* events) {
        if (eventIndex == kInvalidID) {
            return;
        }
        EventCounters* e{events + eventIndex};
        if (detected != 0U) atomicAdd(&e->detected, static_cast<unsigned long long>(detected));
        if (absorbed != 0U) atomicAdd(&e->absorbed, static_cast<unsigned long long>(absorbed));
        if (escaped != 0U) atomicAdd(&e->escaped, static_cast<unsigned long long>(escaped));
        if (truncated != 0U) atomicAdd(&e->truncated, static_cast<unsigned long long>(truncated));
        if (invalid != 0U) atomicAdd(&e->invalid, static_cast<unsigned long long>(invalid));
        if (zeroStep != 0U) atomicAdd(&e->zeroStep, static_cast<unsigned long long>(zeroStep));
        if (maxBounce != 0U) atomicMax(&e->maxBounce, static_cast<unsigned long long>(maxBounce));
        Reset();
    }
    __device__ __forceinline__ void Switch(std::uint32_t newEvent, EventCounters* events) {
        if (newEvent != eventIndex) {
            Flush(events);
            eventIndex = newEvent;
        }
    }
    __device__ __forceinline__ void Finish(std::uint32_t result, std::uint32_t bounces) {
        switch (result) {
        case kDetected: ++detected; break;
        case kAbsorbed: ++absorbed; break;
        case kEscaped: ++escaped; break;
        case kTruncated: ++truncated; break;
        default: ++invalid; break;
        }
        maxBounce = max(maxBounce, bounces);
    }
};

// A thread's event counters and bounce total in the batched form, in shared
// memory: they change once per photon, and keeping them out of registers
// leaves more of the register budget to the step loop.
struct LaneTally {
    LaneCounters counters;
    unsigned long long bounces;
};
static_assert(sizeof(LaneTally) == kLaneTallyBytes, "tally layout");

// Largest emission e in [begin, end) with offsets[e] <= slot (FindEmissionIndex, :304-320).
__device__ __forceinline__ std::uint32_t FindEmission(const std::uint32_t* __restrict__ offsets, std::uint32_t begin,
                                                      std::uint32_t end, std::uint32_t slot) {
    std::uint32_t lo{begin};
    std::uint32_t hi{end};
    while (hi - lo > 1U) {
        const std::uint32_t mid{(lo + hi) >> 1U};
        if (__ldg(offsets + mid) <= slot) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// Warp-aggregated hit write: one atomic per warp reserves rows for every lane
// that detected in this iteration; lanes then write their columns at
// consecutive rows (coalesced). Must be reached by all 32 lanes.
template<class R>
__device__ __forceinline__ void WriteHits(bool write, const Photon<R>& photon, std::uint32_t sensorID,
                                          const LaunchParams& p, unsigned lane) {
    const unsigned mask{__ballot_sync(kFullMask, write)};
    if (mask == 0U) {
        return;
    }
    const int leader{__ffs(static_cast<int>(mask)) - 1};
    unsigned long long base{};
    if (static_cast<int>(lane) == leader) {
        base = atomicAdd(p.hitCounter, static_cast<unsigned long long>(__popc(mask)));
    }
    base = __shfl_sync(kFullMask, base, leader);
    if (write) {
        const unsigned long long row{base + static_cast<unsigned>(__popc(mask & ((1U << lane) - 1U)))};
        if (row < p.hits.capacity) {
            p.hits.positionX[row] = static_cast<float>(photon.position.x);
            p.hits.positionY[row] = static_cast<float>(photon.position.y);
            p.hits.positionZ[row] = static_cast<float>(photon.position.z);
            p.hits.time[row] = static_cast<float>(photon.time);
            p.hits.directionX[row] = static_cast<float>(photon.direction.x);
            p.hits.directionY[row] = static_cast<float>(photon.direction.y);
            p.hits.directionZ[row] = static_cast<float>(photon.direction.z);
            p.hits.energy[row] = static_cast<float>(photon.energy);
            p.hits.eventID[row] = photon.eventID;
            p.hits.photonID[row] = photon.photonID;
            p.hits.sensorID[row] = sensorID;
            p.hits.slot[row] = photon.slot;
        }
    }
}

__device__ __forceinline__ void FlushRunCounters(const LaunchParams& p, unsigned long long bounces,
                                                 std::uint32_t coincidentTraces, std::uint32_t coincidentHits,
                                                 unsigned lane) {
#pragma unroll
    for (int offset = 16; offset > 0; offset >>= 1) {
        bounces += __shfl_down_sync(kFullMask, bounces, offset);
    }
    const unsigned traces{__reduce_add_sync(kFullMask, coincidentTraces)};
    const unsigned hits{__reduce_add_sync(kFullMask, coincidentHits)};
    if (lane == 0U) {
        if (bounces != 0ULL) atomicAdd(&p.run->totalBounces, bounces);
        if (traces != 0U) atomicAdd(&p.run->coincidentTraces, static_cast<unsigned long long>(traces));
        if (hits != 0U) atomicAdd(&p.run->coincidentHits, static_cast<unsigned long long>(hits));
    }
}

// Turns a freshly generated photon into a live one, applying the validity
// test and the initial normalisation of __raygen__rg (:693-703).
template<class R>
__device__ __forceinline__ bool StartPhoton(Photon<R>& photon) {
    const R lengthSquared{Dot(photon.direction, photon.direction)};
    if (!(photon.energy > R(0)) || !IsFinite(photon.energy) || !(lengthSquared > R(0)) || !IsFinite(lengthSquared)) {
        return false;
    }
    photon.direction = NormalizeChecked(photon.direction);
    photon.polarization = ProjectPolarization(photon.polarization, photon.direction);
    return true;
}

__device__ __forceinline__ void RecordFate(const LaunchParams& p, std::uint32_t slot, std::uint32_t result,
                                           std::uint32_t bounces, double time) {
    if (p.photonFate != nullptr) {
        p.photonFate[slot] = result | (bounces << 3U);
    }
    if (p.photonTime != nullptr) {
        p.photonTime[slot] = time;
    }
}

// Row i of the photon store: a generated, valid FP32 photon.
__device__ __forceinline__ void StorePhoton(const PhotonStore& store, std::uint32_t i, const Photon<float>& photon) {
    store.position[0][i] = photon.position.x;
    store.position[1][i] = photon.position.y;
    store.position[2][i] = photon.position.z;
    store.direction[0][i] = photon.direction.x;
    store.direction[1][i] = photon.direction.y;
    store.direction[2][i] = photon.direction.z;
    store.polarization[0][i] = photon.polarization.x;
    store.polarization[1][i] = photon.polarization.y;
    store.polarization[2][i] = photon.polarization.z;
    store.energy[i] = photon.energy;
    store.time[i] = photon.time;
    store.eventID[i] = photon.eventID;
    store.photonID[i] = photon.photonID;
    store.volume[i] = photon.volume;
    store.eventIndex[i] = photon.eventIndex;
}

// Reads row i back; false for a photon that failed the validity test.
__device__ __forceinline__ bool LoadStoredPhoton(const PhotonStore& store, std::uint32_t i, std::uint32_t slot,
                                                 Photon<float>& photon) {
    photon.eventIndex = __ldcs(store.eventIndex + i);
    if (photon.eventIndex == kInvalidID) {
        return false;
    }
    photon.position = {__ldcs(store.position[0] + i), __ldcs(store.position[1] + i), __ldcs(store.position[2] + i)};
    photon.direction = {__ldcs(store.direction[0] + i), __ldcs(store.direction[1] + i),
                        __ldcs(store.direction[2] + i)};
    photon.polarization = {__ldcs(store.polarization[0] + i), __ldcs(store.polarization[1] + i),
                           __ldcs(store.polarization[2] + i)};
    photon.energy = __ldcs(store.energy + i);
    photon.time = __ldcs(store.time + i);
    photon.eventID = __ldcs(store.eventID + i);
    photon.photonID = __ldcs(store.photonID + i);
    photon.volume = __ldcs(store.volume + i);
    photon.slot = slot;
    photon.bounce = 0U;
    return true;
}

// Parks a photon (it left its volume, or its history reached kDeferBounces)
// in the wave's queue, which a second launch of the pass kernel transports;
// false (the photon stays in its lane) when the queue is full.
__device__ __forceinline__ bool DeferPhoton(const DeferredQueue& queue, const Photon<float>& photon) {
    const unsigned int i{atomicAdd(queue.count, 1U)};
    if (i >= queue.capacity) {
        return false;
    }
    DeferredPhoton& parked{queue.photons[i]};
    parked.position[0] = photon.position.x;
    parked.position[1] = photon.position.y;
    parked.position[2] = photon.position.z;
    parked.direction[0] = photon.direction.x;
    parked.direction[1] = photon.direction.y;
    parked.direction[2] = photon.direction.z;
    parked.polarization[0] = photon.polarization.x;
    parked.polarization[1] = photon.polarization.y;
    parked.polarization[2] = photon.polarization.z;
    parked.energy = photon.energy;
    parked.time = photon.time;
    parked.volume = photon.volume;
    parked.bounce = photon.bounce;
    parked.eventID = photon.eventID;
    parked.photonID = photon.photonID;
    parked.eventIndex = photon.eventIndex;
    parked.slot = photon.slot;
    return true;
}

// Parked photon i back into a lane.
__device__ __forceinline__ void LoadDeferredPhoton(const DeferredQueue& queue, std::uint32_t i, Photon<float>& photon) {
    const DeferredPhoton& source{queue.photons[i]};
    photon.position = {source.position[0], source.position[1], source.position[2]};
    photon.direction = {source.direction[0], source.direction[1], source.direction[2]};
    photon.polarization = {source.polarization[0], source.polarization[1], source.polarization[2]};
    photon.energy = source.energy;
    photon.time = source.time;
    photon.volume = source.volume;
    photon.bounce = source.bounce;
    photon.eventID = source.eventID;
    photon.photonID = source.photonID;
    photon.eventIndex = source.eventIndex;
    photon.slot = source.slot;
}

// Generation pass of the batched FP32 form: every photon of the wave
// [photonBegin, photonEnd) made from its genstep and RNG counters as the
// transport kernel would make it, validity-tested (invalid ones counted and
// recorded here) and written to the store. A warp takes 32 consecutive slots:
// one binary search for the first, a forward scan per lane.
__global__ void __launch_bounds__(256) GeneratePhotons(const LaunchParams p) {
    LoadScene(p);
    const PackedScene& scene{*reinterpret_cast<const PackedScene*>(gShared)};
    const float* pool{PoolOf(scene)};
    const unsigned lane{threadIdx.x & 31U};
    const std::uint32_t warps{gridDim.x * (blockDim.x >> 5U)};
    const std::uint32_t warp{blockIdx.x * (blockDim.x >> 5U) + (threadIdx.x >> 5U)};
    for (std::uint32_t base{p.photonBegin + warp * 32U}; base < p.photonEnd; base += warps * 32U) {
        const std::uint32_t slot{base + lane};
        if (slot >= p.photonEnd) {
            continue;
        }
        std::uint32_t e{FindEmission(p.emissionOffsets, p.emissionBegin, p.emissionEnd, base)};
        while (__ldg(p.emissionOffsets + e + 1U) <= slot) {
            ++e;
        }
        Emission emission;
        LoadEmission(p.emissions, e, emission);
        const std::uint32_t local{slot - __ldg(p.emissionOffsets + e)};
        const std::uint32_t eventIndex{__ldg(p.emissionEventIndices + e)};
        Photon<float> photon{};
        GeneratePhoton<float>(scene, pool, emission, emission.FirstPhotonID() + local, p.seed, NoGradient(), photon);
        photon.eventIndex = eventIndex;
        photon.slot = slot;
        const std::uint32_t row{slot - p.photonBegin};
        if (StartPhoton(photon)) {
            StorePhoton(p.store, row, photon);
        } else {
            atomicAdd(&p.events[eventIndex].invalid, 1ULL);
            RecordFate(p, slot, kInvalid, 0U, photon.time);
            p.store.eventIndex[row] = kInvalidID;
        }
    }
}

// The shared-memory photon queue of one warp (layout sizes kQueueBytesFP32/64).
template<class R>
struct WarpQueue {
    R positionX[32], positionY[32], positionZ[32];
    R directionX[32], directionY[32], directionZ[32];
    R polarizationX[32], polarizationY[32], polarizationZ[32];
    R energy[32];
    double time[32];
    std::uint32_t eventID[32], photonID[32], volume[32], eventIndex[32], slot[32];

    __device__ __forceinline__ void Put(unsigned k, const Photon<R>& photon) {
        positionX[k] = photon.position.x;
        positionY[k] = photon.position.y;
        positionZ[k] = photon.position.z;
        directionX[k] = photon.direction.x;
        directionY[k] = photon.direction.y;
        directionZ[k] = photon.direction.z;
        polarizationX[k] = photon.polarization.x;
        polarizationY[k] = photon.polarization.y;
        polarizationZ[k] = photon.polarization.z;
        energy[k] = photon.energy;
        time[k] = photon.time;
        eventID[k] = photon.eventID;
        photonID[k] = photon.photonID;
        volume[k] = photon.volume;
        eventIndex[k] = photon.eventIndex;
        slot[k] = photon.slot;
    }
    __device__ __forceinline__ void Take(unsigned k, Photon<R>& photon) const {
        photon.position = {positionX[k], positionY[k], positionZ[k]};
        photon.direction = {directionX[k], directionY[k], directionZ[k]};
        photon.polarization = {polarizationX[k], polarizationY[k], polarizationZ[k]};
        photon.energy = energy[k];
        photon.time = time[k];
        photon.eventID = eventID[k];
        photon.photonID = photonID[k];
        photon.volume = volume[k];
        photon.eventIndex = eventIndex[k];
        photon.slot = slot[k];
        photon.bounce = 0U;
    }
};
static_assert(sizeof(WarpQueue<float>) == kQueueBytesFP32, "queue layout");
static_assert(sizeof(WarpQueue<double>) == kQueueBytesFP64, "queue layout");

// The shared-memory Fresnel ring of one warp. Steps that stop at a boundary
// without a surface park here as pending jobs; once 32 are pending the whole
// warp completes them together (one job per lane) and they stay in place as
// ready photons, which idle lanes take before fresh ones. Entries are used in
// ring order: [readyHead, pendingHead) ready, [pendingHead, pendingEnd) pending.
template<class R, std::uint32_t kRingEntries = kFresnelRingEntries>
struct FresnelRing {
    static constexpr std::uint32_t kEntries = kRingEntries;
    R positionX[kEntries], positionY[kEntries], positionZ[kEntries];  // the boundary point while pending
    R directionX[kEntries], directionY[kEntries], directionZ[kEntries];
    R polarizationX[kEntries], polarizationY[kEntries], polarizationZ[kEntries];
    R energy[kEntries], indexFrom[kEntries], indexTo[kEntries];
    double time[kEntries];
    std::uint32_t eventID[kEntries], photonID[kEntries], volume[kEntries], eventIndex[kEntries], slot[kEntries],
        bounce[kEntries];
    // pending: next volume | normal axis << 8 | sign bits of the normal << 10; ready: the step result
    std::uint32_t link[kEntries];

    __device__ __forceinline__ void PutPhoton(unsigned k, const Photon<R>& photon) {
        directionX[k] = photon.direction.x;
        directionY[k] = photon.direction.y;
        directionZ[k] = photon.direction.z;
        polarizationX[k] = photon.polarization.x;
        polarizationY[k] = photon.polarization.y;
        polarizationZ[k] = photon.polarization.z;
        energy[k] = photon.energy;
        time[k] = photon.time;
        eventID[k] = photon.eventID;
        photonID[k] = photon.photonID;
        volume[k] = photon.volume;
        eventIndex[k] = photon.eventIndex;
        slot[k] = photon.slot;
        bounce[k] = photon.bounce;
    }
    __device__ __forceinline__ void TakePhoton(unsigned k, Photon<R>& photon) const {
        photon.position = {positionX[k], positionY[k], positionZ[k]};
        photon.direction = {directionX[k], directionY[k], directionZ[k]};
        photon.polarization = {polarizationX[k], polarizationY[k], polarizationZ[k]};
        photon.energy = energy[k];
        photon.time = time[k];
        photon.eventID = eventID[k];
        photon.photonID = photonID[k];
        photon.volume = volume[k];
        photon.eventIndex = eventIndex[k];
        photon.slot = slot[k];
        photon.bounce = bounce[k];
    }
    __device__ __forceinline__ void PutJob(unsigned k, const Photon<R>& photon, const FresnelJob<R>& job) {
        PutPhoton(k, photon);
        positionX[k] = job.boundary.x;
        positionY[k] = job.boundary.y;
        positionZ[k] = job.boundary.z;
        indexFrom[k] = job.indexFrom;
        indexTo[k] = job.indexTo;
        // the boundary normal is a unit axis of a box face; the signs of all
        // three components are kept, zeros included, so the completed step
        // is bit-identical to one finished in place
        const std::uint32_t axis{job.normal.x != R(0) ? 0U : (job.normal.y != R(0) ? 1U : 2U)};
        link[k] = job.next | (axis << 8U) | (static_cast<std::uint32_t>(signbit(job.normal.x)) << 10U) |
                  (static_cast<std::uint32_t>(signbit(job.normal.y)) << 11U) |
                  (static_cast<std::uint32_t>(signbit(job.normal.z)) << 12U);
    }
    __device__ __forceinline__ void TakeJob(unsigned k, Photon<R>& photon, FresnelJob<R>& job) const {
        TakePhoton(k, photon);
        job.boundary = photon.position;
        job.indexFrom = indexFrom[k];
        job.indexTo = indexTo[k];
        const std::uint32_t code{link[k]};
        job.next = code & 0xffU;
        const std::uint32_t axis{(code >> 8U) & 3U};
        const R x{axis == 0U ? R(1) : R(0)}, y{axis == 1U ? R(1) : R(0)}, z{axis == 2U ? R(1) : R(0)};
        job.normal = {((code >> 10U) & 1U) != 0U ? -x : x, ((code >> 11U) & 1U) != 0U ? -y : y,
                      ((code >> 12U) & 1U) != 0U ? -z : z};
    }
    __device__ __forceinline__ void PutReady(unsigned k, const Photon<R>& photon, std::uint32_t result) {
        PutPhoton(k, photon);
        positionX[k] = photon.position.x;
        positionY[k] = photon.position.y;
        positionZ[k] = photon.position.z;
        link[k] = result;
    }
};
static_assert(sizeof(FresnelRing<float>) == kRingBytesFP32, "ring layout");
static_assert(sizeof(FresnelRing<double>) == kRingBytesFP64, "ring layout");
static_assert(sizeof(FresnelRing<float, kFresnelRingEntriesPass>) == kRingBytesFP32Pass, "ring layout");


// A Fresnel step completed in the lane that reached it, when the ring is full.
template<class R>
G4B_COLD std::uint32_t FinishFresnelHere(Photon<R>& photon, const FresnelJob<R>& job, unsigned long long seed,
                                         std::uint32_t maxBounce, R epsilon) {
    return FinishFresnel(photon, job.boundary, job.normal, job.indexFrom, job.indexTo, job.next, seed, maxBounce,
                         epsilon);
}

// Completes `count` (<= 32) pending Fresnel jobs from pendingHead, one per
// lane, leaving them in place as ready photons.
template<class R, class Ring>
__device__ __forceinline__ void ResolvePending(Ring& ring, std::uint32_t& pendingHead, std::uint32_t count,
                                               unsigned lane, const LaunchParams& p, R epsilon) {
    if (lane < count) {
        const unsigned k{(pendingHead + lane) % Ring::kEntries};
        Photon<R> photon{};
        FresnelJob<R> job;
        ring.TakeJob(k, photon, job);
        const std::uint32_t result{FinishFresnel(photon, job.boundary, job.normal, job.indexFrom, job.indexTo, job.next,
                                                 p.seed, p.maxBounce, epsilon)};
        ring.PutReady(k, photon, result);
    }
    pendingHead += count;
    __syncwarp();
}

// Persistent transport. Each warp owns a 32-entry photon queue in shared
// memory. When the queue is empty and a lane needs a photon, the whole warp
// takes the next 32 flattened photon indices of its chunk (one atomic on the
// device work queue per chunk) and generates them together, so generation
// runs with every lane busy; idle lanes then refill from the queue in every
// iteration at the cost of a few shared-memory loads.
// Resident 256-thread blocks per SM the compiler must allow: for FP32 three
// (at most 85 registers), which measured faster than the unconstrained
// allocation despite a few spills; FP64 keeps the compiler's choice.
template<class R>
struct BatchedMinBlocks {
    static constexpr int value = 3;
};
template<>
struct BatchedMinBlocks<double> {
    static constexpr int value = 1;
};

// kDiagnostics: count coincident-face retraces and hits, which the reference
// does only with enablePerformanceDiagnostics (OptiXTransportDevice.cu:752-775);
// without it the counting is compiled out, which frees registers in the loop.
// kPregenerated (FP32 only): the wave's photons come from the photon store
// that GeneratePhotons filled, and the loop carries no generation code.
// kParked (with kPregenerated): the photons come from the wave's queue of
// parked photons instead, and each step completes its Fresnel boundary in
// place: what the queue holds is few photons with long histories, whose
// steps should each take one loop iteration, not the three that parking in
// the ring costs a lone photon.
template<class R, bool kDiagnostics, bool kPregenerated = false, bool kParked = false>
__global__ void __launch_bounds__(256, BatchedMinBlocks<R>::value) TransportBatched(const LaunchParams p) {
    LoadScene(p);
    const PackedScene& scene{*reinterpret_cast<const PackedScene*>(gShared)};
    const float* pool{PoolOf(scene)};
    const unsigned lane{threadIdx.x & 31U};
    const unsigned lanesBelow{(1U << lane) - 1U};
    const R epsilon{R(p.epsilon)};
    static_assert(!kParked || kPregenerated, "the parked-photon form reads the pass form's queue");
    // whether this lane may still park photons in the wave's queue (the
    // parked form parks none itself)
    bool parkOpen{kPregenerated && !kParked && p.deferred.photons != nullptr};
    const std::uint32_t totalPhotons{kParked ? min(*p.deferred.count, p.deferred.capacity)
                                             : p.photonEnd - p.photonBegin};
    const std::uint32_t sceneEnd{(p.sceneBytes + 15U) & ~15U};
    // shared memory: scene, then one photon queue per warp (not with
    // kPregenerated: lanes take photons straight from the store), one Fresnel
    // ring per warp, one tally per lane
    const std::uint32_t warps{blockDim.x >> 5U};
    constexpr std::uint32_t kQueueBytes{kPregenerated ? 0U : static_cast<std::uint32_t>(sizeof(WarpQueue<R>))};
    WarpQueue<R>& queue{*reinterpret_cast<WarpQueue<R>*>(gShared + sceneEnd + (threadIdx.x >> 5U) * kQueueBytes)};
    using Ring = FresnelRing<R, kPregenerated ? kFresnelRingEntriesPass : kFresnelRingEntries>;
    Ring& ring{*reinterpret_cast<Ring*>(gShared + sceneEnd + warps * kQueueBytes + (threadIdx.x >> 5U) * sizeof(Ring))};
    LaneTally& tally{*reinterpret_cast<LaneTally*>(gShared + sceneEnd + warps * (kQueueBytes + sizeof(Ring)) +
                                                   threadIdx.x * sizeof(LaneTally))};
    constexpr std::uint32_t kRing{Ring::kEntries};
    std::uint32_t readyHead{0U};
    std::uint32_t pendingHead{0U};
    std::uint32_t pendingEnd{0U};

    std::uint32_t chunkNext{0U};
    std::uint32_t chunkEnd{0U};
    std::uint32_t cursor{0U};
    std::uint32_t queueHead{0U};
    std::uint32_t queueCount{0U};
    bool workDone{false};
    bool alive{false};
    Photon<R> photon{};
    LaneCounters& counters{tally.counters};
    counters.eventIndex = kInvalidID;
    counters.Reset();
    tally.bounces = 0ULL;
    std::uint32_t coincidentTraces{0U};
    std::uint32_t coincidentHits{0U};

    for (;;) {
        unsigned need{__ballot_sync(kFullMask, !alive)};
        // Photons done with their Fresnel boundary go first.
        if (need != 0U && pendingHead != readyHead) {
            const std::uint32_t ready{pendingHead - readyHead};
            const std::uint32_t rank{static_cast<std::uint32_t>(__popc(need & lanesBelow))};
            if (!alive && rank < ready) {
                const unsigned k{(readyHead + rank) % kRing};
                ring.TakePhoton(k, photon);
                const std::uint32_t status{ring.link[k]};
                counters.Switch(photon.eventIndex, p.events);
                if (status == kContinue) {
                    alive = true;
                } else {  // truncated by the Fresnel step's bounce
                    counters.Finish(status, photon.bounce);
                    tally.bounces += photon.bounce;
                    RecordFate(p, photon.slot, status, photon.bounce, photon.time);
                }
            }
            readyHead += min(static_cast<std::uint32_t>(__popc(need)), ready);
            if (readyHead >= kRing) {
                // keep the three positions small; subtracting the ring size
                // leaves every entry index (position mod kRing) unchanged
                readyHead -= kRing;
                pendingHead -= kRing;
                pendingEnd -= kRing;
            }
            __syncwarp();
            need = __ballot_sync(kFullMask, !alive);
        }
        if constexpr (kPregenerated) {
            // Lanes that need a photon take the next slots of the warp's chunk
            // straight from the store; a photon that failed the validity test
            // leaves its lane needing one.
            while (need != 0U) {
                if (chunkNext >= chunkEnd) {
                    if (workDone) {
                        break;
                    }
                    std::uint32_t start{0U};
                    if (lane == 0U) {
                        start = atomicAdd(p.workTicket, p.chunk);
                    }
                    start = __shfl_sync(kFullMask, start, 0);
                    if (start >= totalPhotons) {
                        workDone = true;
                        break;
                    }
                    chunkNext = p.photonBegin + start;
                    chunkEnd = p.photonBegin + min(start + p.chunk, totalPhotons);
                }
                const std::uint32_t available{chunkEnd - chunkNext};
                const std::uint32_t rank{static_cast<std::uint32_t>(__popc(need & lanesBelow))};
                if (((need >> lane) & 1U) != 0U && rank < available) {
                    const std::uint32_t slot{chunkNext + rank};
                    if constexpr (kParked) {
                        LoadDeferredPhoton(p.deferred, slot - p.photonBegin, photon);
                        counters.Switch(photon.eventIndex, p.events);
                        alive = true;
                    } else if (LoadStoredPhoton(p.store, slot - p.photonBegin, slot, photon)) {
                        counters.Switch(photon.eventIndex, p.events);
                        alive = true;
                    }
                }
                chunkNext += min(static_cast<std::uint32_t>(__popc(need)), available);
                need = __ballot_sync(kFullMask, !alive);
            }
        }
        if constexpr (!kPregenerated) {
        while (need != 0U) {
            if (queueHead == queueCount) {
                if (workDone) {
                    break;
                }
                // Refill the queue: the warp generates its next 32 photons.
                if (chunkNext >= chunkEnd) {
                    std::uint32_t start{0U};
                    if (lane == 0U) {
                        start = atomicAdd(p.workTicket, p.chunk);
                    }
                    start = __shfl_sync(kFullMask, start, 0);
                    if (start >= totalPhotons) {
                        workDone = true;
                        break;
                    }
                    chunkNext = p.photonBegin + start;
                    chunkEnd = p.photonBegin + min(start + p.chunk, totalPhotons);
                    cursor = FindEmission(p.emissionOffsets, p.emissionBegin, p.emissionEnd, chunkNext);
                }
                const std::uint32_t available{chunkEnd - chunkNext};
                const bool has{lane < available};
                std::uint32_t e{cursor};
                bool valid{false};
                Photon<R> fresh{};
                if (has) {
                    const std::uint32_t slot{chunkNext + lane};
                    while (__ldg(p.emissionOffsets + e + 1U) <= slot) {
                        ++e;
                    }
                    Emission emission;
                    LoadEmission(p.emissions, e, emission);
                    const std::uint32_t local{slot - __ldg(p.emissionOffsets + e)};
                    const std::uint32_t eventIndex{__ldg(p.emissionEventIndices + e)};
                    GeneratePhoton<R>(scene, pool, emission, emission.FirstPhotonID() + local, p.seed, NoGradient(),
                                      fresh);
                    fresh.eventIndex = eventIndex;
                    fresh.slot = (p.slotBase != nullptr) ? __ldg(p.slotBase + e) + local : slot;
                    valid = StartPhoton(fresh);
                    if (!valid) {
                        atomicAdd(&p.events[eventIndex].invalid, 1ULL);
                        RecordFate(p, fresh.slot, kInvalid, 0U, fresh.time);
                    }
                }
                const unsigned hasMask{__ballot_sync(kFullMask, has)};
                cursor = __shfl_sync(kFullMask, e, 31 - __clz(static_cast<int>(hasMask)));
                chunkNext += min(available, 32U);
                const unsigned validMask{__ballot_sync(kFullMask, valid)};
                if (valid) {
                    queue.Put(static_cast<unsigned>(__popc(validMask & lanesBelow)), fresh);
                }
                __syncwarp();
                queueHead = 0U;
                queueCount = static_cast<std::uint32_t>(__popc(validMask));
                continue;
            }
            const std::uint32_t available{queueCount - queueHead};
            const std::uint32_t rank{static_cast<std::uint32_t>(__popc(need & lanesBelow))};
            const bool take{((need >> lane) & 1U) != 0U && rank < available};
            if (take) {
                queue.Take(queueHead + rank, photon);
                counters.Switch(photon.eventIndex, p.events);
                alive = true;
            }
            queueHead += min(static_cast<std::uint32_t>(__popc(need)), available);
            need = __ballot_sync(kFullMask, !alive);
        }
        }
        // no photon to step and no fresh work left: complete what is pending,
        // even if fewer than 32, at the one completion site below
        bool draining{false};
        if (__ballot_sync(kFullMask, alive) == 0U) {
            if (pendingEnd == pendingHead) {
                if (pendingHead != readyHead) {
                    continue;
                }
                break;
            }
            draining = true;
        }

        std::uint32_t result{kContinue};
        StepExtras extras{0U, 0U, 0U, 0U};
        FresnelJob<R> job;
        if (alive) {
            if constexpr (kParked) {
                result = StepPhoton<R>(scene, pool, photon, p.seed, p.maxBounce, epsilon, extras, NoGradient());
            } else {
                // the pass form parks photons that leave their volume in the
                // wave's queue, for the queue's own launch, until the lane
                // finds the queue full
                result = StepPhoton<R, true>(scene, pool, photon, p.seed, p.maxBounce, epsilon, extras, NoGradient(),
                                             &job, parkOpen);
            }
        }
        if (result == kFresnelPendingLost) {
            if constexpr (kRing >= 2U * 32U - 1U) {
                result = kFresnelPending;  // the pass form parks such photons before they get here
            } else {
                // a photon that left its volume the way the reference lets it
                // often reflects totally at every step for thousands of steps:
                // in the ring it would advance one step per completion of 32
                result = FinishFresnelHere(photon, job, p.seed, p.maxBounce, epsilon);
            }
        }
        // a photon that left its volume is untouched by the step: parked below
        bool leftVolume{false};
        if constexpr (kPregenerated && !kParked) {
            leftVolume = alive && result == kLeftVolume;
            if (leftVolume) {
                result = kContinue;
            }
        }
        const bool parking{alive && result == kFresnelPending};
        const unsigned parkMask{__ballot_sync(kFullMask, parking)};
        if constexpr (kRing >= 2U * 32U - 1U) {
            // The ring cannot be full. Between steps at most 31 entries are
            // ready or pending: pending ones stay below 32 (32 are completed
            // whenever 32 wait), and the lanes that parked in one step take
            // ready entries first in the next, as many as they are, which is
            // at least as many as a completion of 32 added beyond the 32
            // that parked. So up to 32 parking photons always fit, and the
            // live photon never has its address taken by a fallback.
            if (parking) {
                ring.PutJob((pendingEnd + static_cast<std::uint32_t>(__popc(parkMask & lanesBelow))) % kRing, photon,
                            job);
            }
            pendingEnd += static_cast<std::uint32_t>(__popc(parkMask));
        } else if (parkMask != 0U) {
            const std::uint32_t room{kRing - (pendingEnd - readyHead)};
            if (parking) {
                const std::uint32_t rank{static_cast<std::uint32_t>(__popc(parkMask & lanesBelow))};
                if (rank < room) {
                    ring.PutJob((pendingEnd + rank) % kRing, photon, job);
                } else {
                    result = FinishFresnelHere(photon, job, p.seed, p.maxBounce, epsilon);
                }
            }
            pendingEnd += min(static_cast<std::uint32_t>(__popc(parkMask)), room);
        }
        WriteHits(alive && result == kDetected, photon, extras.sensorID, p, lane);
        if (alive) {
            if (extras.zeroSteps != 0U) {
                counters.zeroStep += extras.zeroSteps;
            }
            if constexpr (kDiagnostics) {
                coincidentTraces += extras.coincidentTraces;
                coincidentHits += extras.coincidentHits;
            }
            if (result == kFresnelPending) {
                alive = false;
            } else if (result != kContinue) {
                const std::uint32_t bounces{result == kTruncated ? photon.bounce : photon.bounce + 1U};
                counters.Finish(result, bounces);
                tally.bounces += bounces;
                RecordFate(p, photon.slot, result, bounces, photon.time);
                alive = false;
            }
        }
        if constexpr (kPregenerated && !kParked) {
            // a photon that left its volume or whose history grew long goes
            // to the wave's queue launch, and the lane takes fresh work
            // (identical results: the step is the same); with the queue full
            // it stays, and steps in place from now on
            if (alive && (leftVolume || photon.bounce >= kDeferBounces) && parkOpen) {
                if (DeferPhoton(p.deferred, photon)) {
                    alive = false;
                } else {
                    parkOpen = false;
                }
            }
        }
        __syncwarp();
        const std::uint32_t pending{pendingEnd - pendingHead};
        if (pending >= 32U || (draining && pending != 0U)) {
            ResolvePending(ring, pendingHead, min(pending, 32U), lane, p, epsilon);
        }
    }
    counters.Flush(p.events);
    FlushRunCounters(p, tally.bounces, coincidentTraces, coincidentHits, lane);
}

// Two resident 256-thread blocks per SM (at most 128 registers): for the
// FP64 form this measured 6 % faster than the compiler's unconstrained
// allocation of 173 registers, despite a few spills.
template<class R, bool kDiagnostics>
__global__ void __launch_bounds__(256, 2) TransportPlain(const LaunchParams p) {
    LoadScene(p);
    const PackedScene& scene{*reinterpret_cast<const PackedScene*>(gShared)};
    const float* pool{PoolOf(scene)};
    const unsigned lane{threadIdx.x & 31U};
    const R epsilon{R(p.epsilon)};
    const std::uint32_t slot{p.photonBegin + blockIdx.x * blockDim.x + threadIdx.x};

    LaneCounters counters{};
    counters.eventIndex = kInvalidID;
    counters.Reset();
    unsigned long long laneBounces{0ULL};
    std::uint32_t coincidentTraces{0U};
    std::uint32_t coincidentHits{0U};
    Photon<R> photon{};
    bool alive{false};
    if (slot < p.photonEnd) {
        const std::uint32_t e{FindEmission(p.emissionOffsets, p.emissionBegin, p.emissionEnd, slot)};
        Emission emission;
        LoadEmission(p.emissions, e, emission);
        const std::uint32_t local{slot - __ldg(p.emissionOffsets + e)};
        const std::uint32_t eventIndex{__ldg(p.emissionEventIndices + e)};
        counters.eventIndex = eventIndex;
        GeneratePhoton<R>(scene, pool, emission, emission.FirstPhotonID() + local, p.seed, NoGradient(), photon);
        photon.eventIndex = eventIndex;
        photon.slot = (p.slotBase != nullptr) ? __ldg(p.slotBase + e) + local : slot;
        alive = StartPhoton(photon);
        if (!alive) {
            ++counters.invalid;
            RecordFate(p, photon.slot, kInvalid, 0U, photon.time);
        }
    }
    while (__ballot_sync(kFullMask, alive) != 0U) {
        std::uint32_t result{kContinue};
        StepExtras extras{0U, 0U, 0U, 0U};
        if (alive) {
            result = StepPhoton<R>(scene, pool, photon, p.seed, p.maxBounce, epsilon, extras, NoGradient());
        }
        WriteHits(alive && result == kDetected, photon, extras.sensorID, p, lane);
        if (alive) {
            counters.zeroStep += extras.zeroSteps;
            if constexpr (kDiagnostics) {
                coincidentTraces += extras.coincidentTraces;
                coincidentHits += extras.coincidentHits;
            }
            if (result != kContinue) {
                const std::uint32_t bounces{result == kTruncated ? photon.bounce : photon.bounce + 1U};
                counters.Finish(result, bounces);
                laneBounces += bounces;
                RecordFate(p, photon.slot, result, bounces, photon.time);
                alive = false;
            }
        }
    }
    counters.Flush(p.events);
    FlushRunCounters(p, laneBounces, coincidentTraces, coincidentHits, lane);
}

// Seed of the draws of an alternate branch spawned at the step that ended
// with bounce number `bounce`: independent of the photon's own draws.
__device__ __forceinline__ unsigned long long AlternateSeed(unsigned long long seed, std::uint32_t bounce) {
    return seed ^ (0x9E3779B97F4A7C15ULL * (static_cast<unsigned long long>(bounce) + 1ULL));
}

// Transports `branch` to its end with the draws of `seed`. Returns whether it
// was detected and its arrival time.
template<class R>
__device__ bool RunBranch(const PackedScene& scene, const float* pool, const LaunchParams& p, Photon<R>& branch,
                          unsigned long long seed, double* time) {
    if (branch.bounce >= p.maxBounce) {
        return false;
    }
    const R epsilon{R(p.epsilon)};
    StepExtras extras{0U, 0U, 0U, 0U};
    std::uint32_t result;
    do {
        result = StepPhoton<R>(scene, pool, branch, seed, p.maxBounce, epsilon, extras, NoGradient());
    } while (result == kContinue);
    *time = branch.time;
    return result == kDetected;
}

// Transports the branch a replayed photon did not take at its last Fresnel
// choice to its end in plain arithmetic. Returns whether it was detected and
// its arrival time.
template<class R>
__device__ bool RunAlternate(const PackedScene& scene, const float* pool, const LaunchParams& p,
                             const Photon<Dual<R>>& taken, double* time) {
    Photon<R> branch{};
    branch.position = taken.tangents.alternatePosition;
    branch.direction = taken.tangents.alternateDirection;
    branch.polarization = taken.tangents.alternatePolarization;
    branch.volume = taken.tangents.alternateVolume;
    branch.time = taken.time;
    branch.energy = taken.energy.v;
    branch.bounce = taken.bounce;
    branch.eventID = taken.eventID;
    branch.photonID = taken.photonID;
    return RunBranch(scene, pool, p, branch, AlternateSeed(p.seed, taken.bounce), time);
}

// Transports the state a replayed photon's last step left for its edge term
// (the same step, its ray leaving through the face beyond the edge) to its
// end in plain arithmetic, with the photon's own draws.
template<class R>
__device__ bool RunEdgeBranch(const PackedScene& scene, const float* pool, const LaunchParams& p,
                              const Photon<Dual<R>>& taken, double* time) {
    Photon<R> branch{};
    branch.position = taken.tangents.edgePosition;
    branch.direction = taken.tangents.edgeDirection;
    branch.polarization = taken.tangents.edgePolarization;
    branch.volume = taken.tangents.edgeVolume;
    branch.time = taken.tangents.edgeTime;
    branch.energy = taken.energy.v;
    branch.bounce = taken.tangents.edgeBounce;
    branch.eventID = taken.eventID;
    branch.photonID = taken.photonID;
    return RunBranch(scene, pool, p, branch, p.seed, time);
}

// Gradient replay: every photon of the batch is regenerated from its RNG
// counters and re-transported with dual numbers (pathwise derivatives), its
// score terms accumulating; with a refractive-index target each Fresnel choice
// at a boundary without a surface spawns its alternate branch instead of a
// score (measure-valued derivative, bounded where the score dT/T is not),
// and each step that leaves its box near an edge the branch through the face
// beyond it (SpawnEdgeBranch: the boundary term of the moving edge).
// Per photon, with f its detection and t its arrival time:
//   dN     += f (S + W) - sum_k w_k f_k
//   d(tN)  += f (t (S + W) + dt) - sum_k w_k f_k t_k
// where S is the score, w_k = +-dT/dn of Fresnel choice k or the weight of
// edge term k, W = sum w_k and f_k, t_k the outcome of its branch.
// Grid-stride over the photons, FP64 sums reduced per warp at the end.
template<class R>
__global__ void __launch_bounds__(128) GradientReplay(const LaunchParams p, GradientTargets targets,
                                                      GradientSums* sums) {
    using D = Dual<R>;
    LoadScene(p);
    const PackedScene& scene{*reinterpret_cast<const PackedScene*>(gShared)};
    const float* pool{PoolOf(scene)};
    double values[10]{};
    for (std::uint32_t slot = p.photonBegin + blockIdx.x * blockDim.x + threadIdx.x; slot < p.photonEnd;
         slot += gridDim.x * blockDim.x) {
        const std::uint32_t e{FindEmission(p.emissionOffsets, 0U, p.emissionCount, slot)};
        Emission emission;
        LoadEmission(p.emissions, e, emission);
        const std::uint32_t local{slot - __ldg(p.emissionOffsets + e)};
        Photon<D> photon{};
        photon.tangents.alternates = targets.indexMaterial != kInvalidID;
        GeneratePhoton<D>(scene, pool, emission, emission.FirstPhotonID() + local, p.seed, targets, photon);
        photon.slot = slot;
        std::uint32_t result{kInvalid};
        StepExtras extras{0U, 0U, 0U, 0U};
        double weights{0.0};
        double alternateDetected{0.0};
        double alternateTime{0.0};
        if (StartPhoton(photon)) {
            const D epsilon{p.epsilon};
            do {
                result = StepPhoton<D>(scene, pool, photon, p.seed, p.maxBounce, epsilon, extras, targets);
                if (photon.tangents.alternatePending) {
                    photon.tangents.alternatePending = false;
                    const double w{photon.tangents.alternateWeight};
                    double time{0.0};
                    weights += w;
                    if (RunAlternate(scene, pool, p, photon, &time)) {
                        alternateDetected += w;
                        alternateTime += w * time;
                    }
                }
                if (photon.tangents.edgePending) {
                    photon.tangents.edgePending = false;
                    const double w{photon.tangents.edgeWeight};
                    double time{0.0};
                    weights += w;
                    if (RunEdgeBranch(scene, pool, p, photon, &time)) {
                        alternateDetected += w;
                        alternateTime += w * time;
                    }
                }
            } while (result == kContinue);
        }
        values[2] -= alternateDetected;
        values[6] -= alternateTime;
        if (result == kDetected) {
            const double t{photon.time};
            const double score[4]{photon.tangents.scoreIndex + weights, photon.tangents.scoreAbsLength,
                                  photon.tangents.scoreReflectivity, 0.0};
            const double dt[4]{photon.tangents.dTimeDIndex, 0.0, 0.0, photon.tangents.dTimeDDecay};
            values[0] += 1.0;
            values[1] += t;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                values[2 + j] += score[j];
                values[6 + j] += t * score[j] + dt[j];
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 10; ++k) {
#pragma unroll
        for (int offset = 16; offset > 0; offset >>= 1) {
            values[k] += __shfl_down_sync(kFullMask, values[k], offset);
        }
    }
    if ((threadIdx.x & 31U) == 0U) {
        atomicAdd(&sums->detected, values[0]);
        atomicAdd(&sums->time, values[1]);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            atomicAdd(&sums->score[j], values[2 + j]);
            atomicAdd(&sums->timeScore[j], values[6 + j]);
        }
    }
}

__global__ void ZeroCounters(EventCounters* events, std::uint32_t eventCount, RunCounters* run) {
    const std::uint32_t i{blockIdx.x * blockDim.x + threadIdx.x};
    const std::uint32_t words{eventCount * static_cast<std::uint32_t>(sizeof(EventCounters) / 16U)};
    uint4* destination{reinterpret_cast<uint4*>(events)};
    for (std::uint32_t w = i; w < words; w += gridDim.x * blockDim.x) {
        destination[w] = make_uint4(0U, 0U, 0U, 0U);
    }
    if (i < sizeof(RunCounters) / 8U) {
        reinterpret_cast<unsigned long long*>(run)[i] = 0ULL;
    }
}

// --- ordered compaction (bitmap of detected slots + exclusive prefix) -----

__global__ void MarkSlots(const std::uint32_t* __restrict__ slots, unsigned long long count,
                          std::uint32_t* __restrict__ bitmap) {
    for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        const std::uint32_t slot{slots[i]};
        atomicOr(bitmap + (slot >> 5U), 1U << (slot & 31U));
    }
}

// Block b sums the population counts of words [1024 b, 1024 b + 1024).
__global__ void __launch_bounds__(256) BlockPopcount(const std::uint32_t* __restrict__ bitmap, std::uint32_t words,
                                                     std::uint32_t* __restrict__ blockSums) {
    __shared__ std::uint32_t warpSums[8];
    const std::uint32_t base{blockIdx.x * 1024U};
    std::uint32_t sum{0U};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const std::uint32_t w{base + threadIdx.x * 4U + static_cast<std::uint32_t>(k)};
        if (w < words) {
            sum += static_cast<std::uint32_t>(__popc(bitmap[w]));
        }
    }
    sum = __reduce_add_sync(kFullMask, sum);
    if ((threadIdx.x & 31U) == 0U) {
        warpSums[threadIdx.x >> 5U] = sum;
    }
    __syncthreads();
    if (threadIdx.x == 0U) {
        std::uint32_t total{0U};
        for (int w = 0; w < 8; ++w) {
            total += warpSums[w];
        }
        blockSums[blockIdx.x] = total;
    }
}

// Exclusive scan of the block sums in place, one CTA of 1024 threads.
__global__ void __launch_bounds__(1024) ScanBlockSums(std::uint32_t* sums, std::uint32_t count) {
    __shared__ std::uint32_t warpTotals[32];
    __shared__ std::uint32_t carry;
    if (threadIdx.x == 0U) {
        carry = 0U;
    }
    __syncthreads();
    const unsigned lane{threadIdx.x & 31U};
    const unsigned warp{threadIdx.x >> 5U};
    for (std::uint32_t base = 0; base < count; base += 1024U) {
        const std::uint32_t i{base + threadIdx.x};
        const std::uint32_t value{i < count ? sums[i] : 0U};
        std::uint32_t inclusive{value};
#pragma unroll
        for (int offset = 1; offset < 32; offset <<= 1) {
            const std::uint32_t other{__shfl_up_sync(kFullMask, inclusive, offset)};
            if (lane >= static_cast<unsigned>(offset)) {
                inclusive += other;
            }
        }
        if (lane == 31U) {
            warpTotals[warp] = inclusive;
        }
        __syncthreads();
        if (warp == 0U) {
            std::uint32_t t{warpTotals[lane]};
#pragma unroll
            for (int offset = 1; offset < 32; offset <<= 1) {
                const std::uint32_t other{__shfl_up_sync(kFullMask, t, offset)};
                if (lane >= static_cast<unsigned>(offset)) {
                    t += other;
                }
            }
            warpTotals[lane] = t;
        }
        __syncthreads();
        const std::uint32_t warpPrefix{warp == 0U ? 0U : warpTotals[warp - 1U]};
        if (i < count) {
            sums[i] = carry + warpPrefix + inclusive - value;
        }
        __syncthreads();
        if (threadIdx.x == 1023U) {
            carry += warpPrefix + inclusive;
        }
        __syncthreads();
    }
}

// prefix[w] = number of set bits in words [0, w).
__global__ void __launch_bounds__(256) WordPrefix(const std::uint32_t* __restrict__ bitmap, std::uint32_t words,
                                                  const std::uint32_t* __restrict__ blockSums,
                                                  std::uint32_t* __restrict__ prefix) {
    __shared__ std::uint32_t warpTotals[8];
    const std::uint32_t base{blockIdx.x * 1024U + threadIdx.x * 4U};
    std::uint32_t counts[4];
    std::uint32_t local{0U};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const std::uint32_t w{base + static_cast<std::uint32_t>(k)};
        counts[k] = w < words ? static_cast<std::uint32_t>(__popc(bitmap[w])) : 0U;
        local += counts[k];
    }
    const unsigned lane{threadIdx.x & 31U};
    const unsigned warp{threadIdx.x >> 5U};
    std::uint32_t inclusive{local};
#pragma unroll
    for (int offset = 1; offset < 32; offset <<= 1) {
        const std::uint32_t other{__shfl_up_sync(kFullMask, inclusive, offset)};
        if (lane >= static_cast<unsigned>(offset)) {
            inclusive += other;
        }
    }
    if (lane == 31U) {
        warpTotals[warp] = inclusive;
    }
    __syncthreads();
    std::uint32_t warpPrefix{0U};
    for (unsigned w = 0; w < warp; ++w) {
        warpPrefix += warpTotals[w];
    }
    std::uint32_t running{blockSums[blockIdx.x] + warpPrefix + inclusive - local};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const std::uint32_t w{base + static_cast<std::uint32_t>(k)};
        if (w < words) {
            prefix[w] = running;
        }
        running += counts[k];
    }
}

// Writes each hit as a 48-byte detection record (PhotonDetection,
// PhotonTransport.hpp:71-81) at its rank among detected slots, or at its
// device row when `ordered` is false.
__global__ void ScatterDetections(const HitColumns hits, unsigned long long count,
                                  const std::uint32_t* __restrict__ bitmap, const std::uint32_t* __restrict__ prefix,
                                  bool ordered, float4* __restrict__ out) {
    for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        unsigned long long row{i};
        if (ordered) {
            const std::uint32_t slot{hits.slot[i]};
            const std::uint32_t word{slot >> 5U};
            const std::uint32_t below{bitmap[word] & ((1U << (slot & 31U)) - 1U)};
            row = prefix[word] + static_cast<std::uint32_t>(__popc(below));
        }
        float4* record{out + row * 3ULL};
        record[0] = make_float4(hits.positionX[i], hits.positionY[i], hits.positionZ[i], hits.time[i]);
        record[1] = make_float4(hits.directionX[i], hits.directionY[i], hits.directionZ[i], hits.energy[i]);
        record[2] = make_float4(__uint_as_float(hits.eventID[i]), __uint_as_float(hits.photonID[i]),
                                __uint_as_float(hits.sensorID[i]), 0.0F);
    }
}

// --- ordering into a fixed scratch array ---------------------------------
//
// The same bitmap / block-sum / word-prefix ranking as above, for callers that
// cannot allocate device memory: the three scratch arrays and a status word
// live in one array compiled into the library, sized for kStaticOrderMaxSlots
// slot keys (2 MiB bitmap + 2 MiB prefix + 2 KiB block sums).

constexpr std::uint32_t kStaticOrderWords{kStaticOrderMaxSlots / 32U};
constexpr std::uint32_t kStaticOrderBlocks{kStaticOrderWords / 1024U};
constexpr std::uint32_t kStaticPrefixOffset{kStaticOrderWords};
constexpr std::uint32_t kStaticSumsOffset{2U * kStaticOrderWords};
constexpr std::uint32_t kStaticStatusOffset{kStaticSumsOffset + kStaticOrderBlocks + 64U};
constexpr std::uint32_t kStaticScratchWords{kStaticStatusOffset + 64U};

static __device__ __align__(256) std::uint32_t gStaticOrderScratch[kStaticScratchWords];

// Per-wave ordering. Each wave of the generation pass writes its hits to its
// own region of the hit buffer, rows [0, count) of the region (count is the
// wave's row counter, clamped to the region's rows: a larger count means the
// region overflowed and the batch reruns). The waves' records go to the
// detection buffer one after another, in wave order: wave k's start row is
// the sum of the earlier waves' counts, which AdvanceWaveRows computes on the
// device once wave k's transport has finished, and the records are ranked by
// slot within the wave.
__global__ void AdvanceWaveRows(const unsigned long long* __restrict__ count, unsigned long long* __restrict__ outRows,
                                unsigned long long regionRows, RunCounters* __restrict__ run) {
    if (blockIdx.x == 0U && threadIdx.x == 0U) {
        const unsigned long long c{*count};
        outRows[1] = outRows[0] + min(c, regionRows);
        run->hitCount += c;
        run->maxWaveHits = max(run->maxWaveHits, c);
    }
}

__global__ void MarkWaveSlots(const std::uint32_t* __restrict__ slots, const unsigned long long* __restrict__ count,
                              unsigned long long regionRows, std::uint32_t* __restrict__ bitmap) {
    const unsigned long long end{min(*count, regionRows)};
    for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < end;
         i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        const std::uint32_t slot{slots[i]};
        atomicOr(bitmap + (slot >> 5U), 1U << (slot & 31U));
    }
}

__global__ void ScatterWaveDetections(const HitColumns hits, const unsigned long long* __restrict__ count,
                                      unsigned long long regionRows, const unsigned long long* __restrict__ outRows,
                                      const std::uint32_t* __restrict__ bitmap,
                                      const std::uint32_t* __restrict__ prefix, bool ordered,
                                      float4* __restrict__ out) {
    const unsigned long long end{min(*count, regionRows)};
    const unsigned long long first{outRows[0]};
    for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < end;
         i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        unsigned long long row{first + i};
        if (ordered) {
            const std::uint32_t slot{hits.slot[i]};
            const std::uint32_t word{slot >> 5U};
            const std::uint32_t below{bitmap[word] & ((1U << (slot & 31U)) - 1U)};
            row = first + prefix[word] + static_cast<std::uint32_t>(__popc(below));
        }
        float4* record{out + row * 3ULL};
        record[0] = make_float4(hits.positionX[i], hits.positionY[i], hits.positionZ[i], hits.time[i]);
        record[1] = make_float4(hits.directionX[i], hits.directionY[i], hits.directionZ[i], hits.energy[i]);
        record[2] = make_float4(__uint_as_float(hits.eventID[i]), __uint_as_float(hits.photonID[i]),
                                __uint_as_float(hits.sensorID[i]), 0.0F);
    }
}

// Marks each record's slot key in the bitmap. A key at or above slotLimit,
// or one already marked, touches nothing and adds one to *status.
__global__ void MarkKeysChecked(const std::uint32_t* __restrict__ keys, unsigned long long count,
                                std::uint32_t slotLimit, std::uint32_t* __restrict__ bitmap,
                                std::uint32_t* __restrict__ status) {
    for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        const std::uint32_t key{keys[i]};
        if (key >= slotLimit) {
            atomicAdd(status, 1U);
            continue;
        }
        const std::uint32_t bit{1U << (key & 31U)};
        if ((atomicOr(bitmap + (key >> 5U), bit) & bit) != 0U) {
            atomicAdd(status, 1U);
        }
    }
}

// Copies each 48-byte record to the rank of its key among the marked keys.
// Ranks stay below the number of marked keys, which is at most `count`, so
// every store lands inside `out` even when keys were rejected above.
__global__ void ScatterRecords(const float4* __restrict__ in, const std::uint32_t* __restrict__ keys,
                               unsigned long long count, std::uint32_t slotLimit,
                               const std::uint32_t* __restrict__ bitmap, const std::uint32_t* __restrict__ prefix,
                               float4* __restrict__ out) {
    for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        const std::uint32_t key{keys[i]};
        if (key >= slotLimit) {
            continue;
        }
        const std::uint32_t word{key >> 5U};
        const std::uint32_t below{bitmap[word] & ((1U << (key & 31U)) - 1U)};
        const unsigned long long row{prefix[word] + static_cast<std::uint32_t>(__popc(below))};
        const float4* source{in + i * 3ULL};
        float4* target{out + row * 3ULL};
        target[0] = source[0];
        target[1] = source[1];
        target[2] = source[2];
    }
}

// --- device evaluation of single functions ------------------------------

template<class R>
__global__ void EvalFresnel(std::uint32_t n, const double* __restrict__ in, double* __restrict__ out) {
    const std::uint32_t i{blockIdx.x * blockDim.x + threadIdx.x};
    if (i >= n) {
        return;
    }
    const double* row{in + static_cast<std::size_t>(i) * 11U};
    const V3<R> d{R(row[0]), R(row[1]), R(row[2])};
    const V3<R> pol{R(row[3]), R(row[4]), R(row[5])};
    const V3<R> nrm{R(row[6]), R(row[7]), R(row[8])};
    const FresnelOutput<R> f{ComputeFresnel(d, pol, nrm, R(row[9]), R(row[10]))};
    double* o{out + static_cast<std::size_t>(i) * 14U};
    const V3<R> vs[4]{f.reflectedDirection, f.transmittedDirection, f.reflectedPolarization, f.transmittedPolarization};
    for (int k = 0; k < 4; ++k) {
        o[3 * k] = static_cast<double>(vs[k].x);
        o[3 * k + 1] = static_cast<double>(vs[k].y);
        o[3 * k + 2] = static_cast<double>(vs[k].z);
    }
    o[12] = static_cast<double>(f.transmittance);
    o[13] = f.tir ? 1.0 : 0.0;
}

template<class R>
__global__ void EvalLambertian(std::uint32_t n, const double* __restrict__ in, double* __restrict__ out) {
    const std::uint32_t i{blockIdx.x * blockDim.x + threadIdx.x};
    if (i >= n) {
        return;
    }
    const double* row{in + static_cast<std::size_t>(i) * 5U};
    const V3<R> v{SampleLambertian(V3<R>{R(row[0]), R(row[1]), R(row[2])}, R(row[3]), R(row[4]))};
    out[3 * i] = static_cast<double>(v.x);
    out[3 * i + 1] = static_cast<double>(v.y);
    out[3 * i + 2] = static_cast<double>(v.z);
}

__global__ void EvalMath(std::uint32_t kind, std::uint32_t n, const float* __restrict__ in, float* __restrict__ out) {
    const std::uint32_t i{blockIdx.x * blockDim.x + threadIdx.x};
    if (i >= n) {
        return;
    }
    const float x{in[i]};
    if (kind == 0U) {
        out[i] = LogF(x);
    } else if (kind == 1U) {
        out[i] = ExpF(x);
    } else {
        float s, c;
        SinCosTurnF(x, &s, &c);
        out[i] = s;
        out[n + i] = c;
    }
}

__global__ void EvalUniform(std::uint32_t n, unsigned long long seed, const unsigned long long* __restrict__ keys,
                            const std::uint32_t* __restrict__ counters, float* __restrict__ out) {
    const std::uint32_t i{blockIdx.x * blockDim.x + threadIdx.x};
    if (i >= n) {
        return;
    }
    out[i] = Uniform<float>(seed, keys[i], counters[3 * i], counters[3 * i + 1], counters[3 * i + 2]);
}

unsigned BlocksFor(unsigned long long n, unsigned block) {
    const unsigned long long blocks{(n + block - 1ULL) / block};
    return static_cast<unsigned>(blocks == 0ULL ? 1ULL : (blocks > 1048576ULL ? 1048576ULL : blocks));
}

}  // namespace

const void* TransportKernel(int precision, int form) {
    const bool diagnostics{(form & kWithDiagnostics) != 0};
    if ((form & ~kWithDiagnostics) == kPlain) {
        if (precision == kFP64) {
            return diagnostics ? reinterpret_cast<const void*>(&TransportPlain<double, true>)
                               : reinterpret_cast<const void*>(&TransportPlain<double, false>);
        }
        return diagnostics ? reinterpret_cast<const void*>(&TransportPlain<float, true>)
                           : reinterpret_cast<const void*>(&TransportPlain<float, false>);
    }
    if (precision == kFP64) {
        return diagnostics ? reinterpret_cast<const void*>(&TransportBatched<double, true>)
                           : reinterpret_cast<const void*>(&TransportBatched<double, false>);
    }
    if ((form & kParkedQueue) != 0) {
        return diagnostics ? reinterpret_cast<const void*>(&TransportBatched<float, true, true, true>)
                           : reinterpret_cast<const void*>(&TransportBatched<float, false, true, true>);
    }
    if ((form & kPregenerated) != 0) {
        return diagnostics ? reinterpret_cast<const void*>(&TransportBatched<float, true, true>)
                           : reinterpret_cast<const void*>(&TransportBatched<float, false, true>);
    }
    return diagnostics ? reinterpret_cast<const void*>(&TransportBatched<float, true>)
                       : reinterpret_cast<const void*>(&TransportBatched<float, false>);
}

const void* GenerateKernel() { return reinterpret_cast<const void*>(&GeneratePhotons); }

const void* ZeroCountersKernel() { return reinterpret_cast<const void*>(&ZeroCounters); }

cudaError_t ConfigureTransportKernels(std::size_t sharedBytes) {
    for (int precision = 0; precision < 2; ++precision) {
        // kBatched, kPlain, each with and without kWithDiagnostics, and the
        // pregenerated and parked-photon batched kernels (FP32)
        constexpr int kForms[]{0, 1, 2, 3, 4, 6, 12, 14};
        for (const int form : kForms) {
            const cudaError_t error{cudaFuncSetAttribute(TransportKernel(precision, form),
                                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                         static_cast<int>(sharedBytes))};
            if (error != cudaSuccess) {
                return error;
            }
        }
    }
    return cudaFuncSetAttribute(GenerateKernel(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(sharedBytes));
}

cudaError_t TransportOccupancy(int precision, int form, int blockSize, std::size_t sharedBytes, int* blocksPerSM) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocksPerSM, TransportKernel(precision, form), blockSize,
                                                         sharedBytes);
}

cudaError_t LaunchZeroCounters(EventCounters* events, std::uint32_t eventCount, RunCounters* run,
                               cudaStream_t stream) {
    const unsigned long long words{static_cast<unsigned long long>(eventCount) * (sizeof(EventCounters) / 16U)};
    ZeroCounters<<<BlocksFor(words < 32ULL ? 32ULL : words, 256U), 256, 0, stream>>>(events, eventCount, run);
    return cudaGetLastError();
}

cudaError_t LaunchGenerate(const LaunchParams& params, unsigned grid, std::size_t sharedBytes, cudaStream_t stream) {
    GeneratePhotons<<<grid, 256, sharedBytes, stream>>>(params);
    return cudaGetLastError();
}

cudaError_t LaunchTransport(const LaunchParams& params, int precision, int form, unsigned grid, unsigned block,
                            std::size_t sharedBytes, cudaStream_t stream) {
    void* arguments[]{const_cast<LaunchParams*>(&params)};
    return cudaLaunchKernel(TransportKernel(precision, form), dim3(grid), dim3(block), arguments, sharedBytes,
                            stream);
}

cudaError_t LaunchOrderHits(const HitColumns& hits, unsigned long long count, std::uint32_t photonCount,
                            std::uint32_t* bitmap, std::uint32_t* prefix, std::uint32_t* blockSums,
                            void* detectionsOut, bool ordered, cudaStream_t stream) {
    if (count == 0ULL) {
        return cudaSuccess;
    }
    if (ordered) {
        const std::uint32_t words{(photonCount + 31U) / 32U};
        const std::uint32_t blocks{(words + 1023U) / 1024U};
        cudaError_t error{cudaMemsetAsync(bitmap, 0, static_cast<std::size_t>(words) * 4U, stream)};
        if (error != cudaSuccess) {
            return error;
        }
        MarkSlots<<<BlocksFor(count, 256U), 256, 0, stream>>>(hits.slot, count, bitmap);
        BlockPopcount<<<blocks, 256, 0, stream>>>(bitmap, words, blockSums);
        ScanBlockSums<<<1, 1024, 0, stream>>>(blockSums, blocks);
        WordPrefix<<<blocks, 256, 0, stream>>>(bitmap, words, blockSums, prefix);
    }
    ScatterDetections<<<BlocksFor(count, 256U), 256, 0, stream>>>(hits, count, bitmap, prefix, ordered,
                                                                  static_cast<float4*>(detectionsOut));
    return cudaGetLastError();
}

cudaError_t LaunchOrderWaveHits(const HitColumns& region, const unsigned long long* count,
                                unsigned long long* outRows, RunCounters* run, std::uint32_t slotBegin,
                                std::uint32_t slotEnd, std::uint32_t* bitmap, std::uint32_t* prefix,
                                std::uint32_t* blockSums, void* detectionsOut, bool ordered, unsigned grid,
                                cudaStream_t stream) {
    AdvanceWaveRows<<<1, 32, 0, stream>>>(count, outRows, region.capacity, run);
    if (ordered) {
        const std::uint32_t wordBegin{slotBegin / 32U};
        const std::uint32_t words{(slotEnd - slotBegin + 31U) / 32U};
        const std::uint32_t blocks{(words + 1023U) / 1024U};
        cudaError_t error{cudaMemsetAsync(bitmap + wordBegin, 0, static_cast<std::size_t>(words) * 4U, stream)};
        if (error != cudaSuccess) {
            return error;
        }
        MarkWaveSlots<<<grid, 256, 0, stream>>>(region.slot, count, region.capacity, bitmap);
        BlockPopcount<<<blocks, 256, 0, stream>>>(bitmap + wordBegin, words, blockSums);
        ScanBlockSums<<<1, 1024, 0, stream>>>(blockSums, blocks);
        WordPrefix<<<blocks, 256, 0, stream>>>(bitmap + wordBegin, words, blockSums, prefix + wordBegin);
    }
    ScatterWaveDetections<<<grid, 256, 0, stream>>>(region, count, region.capacity, outRows, bitmap, prefix, ordered,
                                                    static_cast<float4*>(detectionsOut));
    return cudaGetLastError();
}

cudaError_t StaticOrderScratch(std::uint32_t** scratch) {
    return cudaGetSymbolAddress(reinterpret_cast<void**>(scratch), gStaticOrderScratch);
}

cudaError_t LaunchOrderRecordsStatic(const void* records, const std::uint32_t* keys, unsigned long long count,
                                     std::uint32_t slotLimit, std::uint32_t* scratch, void* out,
                                     std::uint32_t* statusHost, cudaStream_t stream) {
    std::uint32_t* bitmap{scratch};
    std::uint32_t* prefix{scratch + kStaticPrefixOffset};
    std::uint32_t* blockSums{scratch + kStaticSumsOffset};
    std::uint32_t* status{scratch + kStaticStatusOffset};
    const std::uint32_t words{(slotLimit + 31U) / 32U};
    const std::uint32_t blocks{(words + 1023U) / 1024U};
    // the bitmap and the status word must start at zero; prefix and block
    // sums are fully rewritten below
    cudaError_t error{cudaMemsetAsync(bitmap, 0, static_cast<std::size_t>(words) * 4U, stream)};
    if (error == cudaSuccess) {
        error = cudaMemsetAsync(status, 0, sizeof(std::uint32_t), stream);
    }
    if (error != cudaSuccess) {
        return error;
    }
    MarkKeysChecked<<<BlocksFor(count, 256U), 256, 0, stream>>>(keys, count, slotLimit, bitmap, status);
    BlockPopcount<<<blocks, 256, 0, stream>>>(bitmap, words, blockSums);
    ScanBlockSums<<<1, 1024, 0, stream>>>(blockSums, blocks);
    WordPrefix<<<blocks, 256, 0, stream>>>(bitmap, words, blockSums, prefix);
    ScatterRecords<<<BlocksFor(count, 256U), 256, 0, stream>>>(static_cast<const float4*>(records), keys, count,
                                                               slotLimit, bitmap, prefix, static_cast<float4*>(out));
    error = cudaGetLastError();
    if (error == cudaSuccess) {
        error = cudaMemcpyAsync(statusHost, status, sizeof(std::uint32_t), cudaMemcpyDeviceToHost, stream);
    }
    if (error == cudaSuccess) {
        error = cudaStreamSynchronize(stream);
    }
    return error;
}

cudaError_t LaunchGradientReplay(const LaunchParams& params, int precision, std::uint32_t indexMaterial,
                                 std::uint32_t absMaterial, std::uint32_t reflectivitySurface, float edgeBand,
                                 float edgeIndexWindow, unsigned grid, std::size_t sharedBytes, GradientSums* sums,
                                 cudaStream_t stream) {
    const GradientTargets targets{indexMaterial, absMaterial, reflectivitySurface, edgeBand, edgeIndexWindow};
    const void* kernel{precision == kFP64 ? reinterpret_cast<const void*>(&GradientReplay<double>)
                                          : reinterpret_cast<const void*>(&GradientReplay<float>)};
    cudaError_t error{cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(sharedBytes))};
    if (error != cudaSuccess) {
        return error;
    }
    if (params.photonEnd <= params.photonBegin) {
        return cudaSuccess;
    }
    if (precision == kFP64) {
        GradientReplay<double><<<grid, 128, sharedBytes, stream>>>(params, targets, sums);
    } else {
        GradientReplay<float><<<grid, 128, sharedBytes, stream>>>(params, targets, sums);
    }
    return cudaGetLastError();
}

cudaError_t LaunchEvalFresnel(int precision, std::uint32_t n, const double* in, double* out, cudaStream_t stream) {
    if (precision == kFP64) {
        EvalFresnel<double><<<BlocksFor(n, 128U), 128, 0, stream>>>(n, in, out);
    } else {
        EvalFresnel<float><<<BlocksFor(n, 128U), 128, 0, stream>>>(n, in, out);
    }
    return cudaGetLastError();
}

cudaError_t LaunchEvalLambertian(int precision, std::uint32_t n, const double* in, double* out,
                                 cudaStream_t stream) {
    if (precision == kFP64) {
        EvalLambertian<double><<<BlocksFor(n, 128U), 128, 0, stream>>>(n, in, out);
    } else {
        EvalLambertian<float><<<BlocksFor(n, 128U), 128, 0, stream>>>(n, in, out);
    }
    return cudaGetLastError();
}

cudaError_t LaunchEvalMath(std::uint32_t kind, std::uint32_t n, const float* in, float* out, cudaStream_t stream) {
    EvalMath<<<BlocksFor(n, 256U), 256, 0, stream>>>(kind, n, in, out);
    return cudaGetLastError();
}

cudaError_t LaunchEvalUniform(std::uint32_t n, unsigned long long seed, const unsigned long long* keys,
                              const std::uint32_t* counters, float* out, cudaStream_t stream) {
    EvalUniform<<<BlocksFor(n, 256U), 256, 0, stream>>>(n, seed, keys, counters, out);
    return cudaGetLastError();
}

}  // namespace g4b

// count_ops.cpp - the oracle's FP32 photon step instantiated with a counting
// number type: every floating-point operation the restated algorithm performs
// is counted, per photon-step (one bounce-loop iteration, the reference's
// totalBounceCount unit, OptiXTransportDevice.cu:707-709,935-937). TEST AND
// MEASUREMENT INFRASTRUCTURE ONLY: it gives the algorithmic operations per
// step for the instruction-issue roofline (oracle/count_ops.py writes them to
// profiles/). Built into its own library (oracle/Makefile); the oracle itself
// is cpu_transport.cpp unchanged (its one hook, G4B_COUNT_FP64, is empty there).
//
// Counted: FP32 add/subtract/negate, multiply, divide, fused multiply-add,
// square root, compare, min/max/abs, and the float<->double conversions; the
// FP64 operations of the time accumulation (one add per conversion into the
// global time) and of the total-internal-reflection test (hook); calls of
// log, exp and sin/cos (weighted by the script as one special-function
// operation plus its range reduction); uniform draws (the script charges one
// Philox-4x32-10 block per four draws, the minimal use of the generator).
// Integer indexing, table searches and control flow are not counted.
#include <cstdint>
#include <cmath>
#include <limits>

struct OpCounts {
    std::uint64_t add, mul, div, fma, sqrt, cmp, minmax, cvt, fp64, log, exp, sincos, uniform;
};
thread_local OpCounts gOps{};

struct Counted {
    float v;
    Counted() = default;
    constexpr Counted(float x) : v(x) {}                         // NOLINT: implicit, as the oracle's R(x)
    constexpr Counted(double x) : v(static_cast<float>(x)) {}    // NOLINT
    constexpr Counted(int x) : v(static_cast<float>(x)) {}       // NOLINT
    explicit operator float() const { return v; }
    explicit operator double() const {
        ++gOps.cvt;
        ++gOps.fp64;  // the conversion feeds one FP64 accumulation
        return static_cast<double>(v);
    }
    Counted& operator+=(Counted o) { ++gOps.add; v += o.v; return *this; }
    Counted& operator-=(Counted o) { ++gOps.add; v -= o.v; return *this; }
    Counted& operator*=(Counted o) { ++gOps.mul; v *= o.v; return *this; }
    Counted& operator/=(Counted o) { ++gOps.div; v /= o.v; return *this; }
};
inline Counted operator+(Counted a, Counted b) { ++gOps.add; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { ++gOps.add; return Counted(a.v - b.v); }
inline Counted operator-(Counted a) { ++gOps.add; return Counted(-a.v); }
inline Counted operator*(Counted a, Counted b) { ++gOps.mul; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { ++gOps.div; return Counted(a.v / b.v); }
inline bool operator<(Counted a, Counted b) { ++gOps.cmp; return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { ++gOps.cmp; return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { ++gOps.cmp; return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { ++gOps.cmp; return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { ++gOps.cmp; return a.v == b.v; }
inline bool operator!=(Counted a, Counted b) { ++gOps.cmp; return a.v != b.v; }

namespace std {
template<>
class numeric_limits<Counted> {
public:
    static constexpr bool is_specialized{true};
    static constexpr Counted infinity() { return Counted(numeric_limits<float>::infinity()); }
    static constexpr Counted quiet_NaN() { return Counted(numeric_limits<float>::quiet_NaN()); }
    static constexpr Counted max() { return Counted(numeric_limits<float>::max()); }
    static constexpr Counted lowest() { return Counted(numeric_limits<float>::lowest()); }
    static constexpr Counted epsilon() { return Counted(numeric_limits<float>::epsilon()); }
};
inline Counted sqrt(Counted a) { ++gOps.sqrt; return Counted(std::sqrt(a.v)); }
inline Counted fabs(Counted a) { ++gOps.minmax; return Counted(std::fabs(a.v)); }
inline Counted fmin(Counted a, Counted b) { ++gOps.minmax; return Counted(std::fmin(a.v, b.v)); }
inline Counted fmax(Counted a, Counted b) { ++gOps.minmax; return Counted(std::fmax(a.v, b.v)); }
inline Counted fma(Counted a, Counted b, Counted c) { ++gOps.fma; return Counted(std::fma(a.v, b.v, c.v)); }
inline bool isfinite(Counted a) { ++gOps.cmp; return std::isfinite(a.v); }
inline bool isnan(Counted a) { ++gOps.cmp; return std::isnan(a.v); }
}  // namespace std

#define G4B_COUNT_FP64(n) gOps.fp64 += (n);
#include "cpu_transport.cpp"

Counted Log(Counted x);
Counted Exp(Counted x);
void SinCosTurn(Counted t, Counted* s, Counted* c);

namespace {
template<>
Counted Uniform<Counted>(std::uint64_t seed, std::uint64_t key, std::uint32_t bounce, std::uint32_t process,
                         std::uint32_t draw) {
    ++gOps.uniform;
    return Counted(Uniform<float>(seed, key, bounce, process, draw));
}
}  // namespace

Counted Log(Counted x) { ++gOps.log; return Counted(LogF(x.v)); }
Counted Exp(Counted x) { ++gOps.exp; return Counted(ExpF(x.v)); }
void SinCosTurn(Counted t, Counted* s, Counted* c) {
    ++gOps.sincos;
    float a, b;
    SinCosTurnF(t.v, &a, &b);
    *s = Counted(a);
    *c = Counted(b);
}

extern "C" {

// Transports photons [photonBegin, photonEnd) of the batch with the counting
// FP32 step on one thread and writes the operation counts (13 numbers, in
// OpCounts order) and the photon-steps taken. Returns 0 or a negative status.
int oracle_count_ops(const g4b_scene* sceneDesc, const g4b_config* config, const g4b_optical_emission* emissions,
                     uint32_t emissionCount, const uint32_t* emissionEventIndices, uint32_t eventCount,
                     uint64_t photonBegin, uint64_t photonEnd, uint64_t* counts, uint64_t* steps) {
    Scene scene{};
    if (sceneDesc == nullptr || config == nullptr || !BuildScene(*sceneDesc, scene)) {
        return G4B_ERR_INVALID_ARGUMENT;
    }
    std::vector<uint64_t> offsets(emissionCount + 1U, 0);
    for (uint32_t i{}; i < emissionCount; ++i) {
        offsets[i + 1] = offsets[i] + emissions[i].photon_count;
    }
    photonEnd = std::min<uint64_t>(photonEnd, offsets[emissionCount]);
    ThreadState state{};
    state.events.assign(eventCount, EventCounters{});
    gOps = OpCounts{};
    uint32_t e{0};
    for (uint64_t slot{photonBegin}; slot < photonEnd; ++slot) {
        while (slot >= offsets[e + 1]) {
            ++e;
        }
        TransportPhoton<Counted>(scene, *config, emissions[e], static_cast<uint32_t>(slot - offsets[e]),
                                 emissionEventIndices[e], slot, state, nullptr, nullptr);
    }
    const uint64_t values[13]{gOps.add, gOps.mul, gOps.div, gOps.fma, gOps.sqrt, gOps.cmp, gOps.minmax,
                              gOps.cvt, gOps.fp64, gOps.log, gOps.exp, gOps.sincos, gOps.uniform};
    std::copy(values, values + 13, counts);
    *steps = state.totalBounces;
    return G4B_OK;
}

}  // extern "C"

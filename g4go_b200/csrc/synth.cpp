// synth.cpp - seeded synthetic genstep source (include/g4b_synth.h).
//
// Stand-in for the Geant4 host side: an electron crosses the crystal in
// straight steps; each step emits one scintillation genstep and, above the
// Cerenkov threshold, one Cerenkov genstep, with the fields that
// Geant4EventAdapter::CaptureCerenkov / CaptureScintillation fill
// (src/optical/geant4/Geant4EventAdapter.cpp:282-388).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/g4b_synth.h"

struct g4b_synth_batch {
    std::vector<g4b_optical_emission> emissions;
    std::vector<std::uint32_t> eventIDs;
    std::vector<std::uint32_t> emissionEventIndices;
    std::uint64_t photons{0};
};

namespace {

thread_local std::string gSynthError;

constexpr double kElectronMassMeV = 0.51099895;
constexpr double kSpeedOfLightMmPerNs = 299.792458;
constexpr double kHcEvNm = 1239.84198;
constexpr double kPi = 3.14159265358979323846;

// splitmix64 stream, one per event.
struct Random {
    std::uint64_t state;
    explicit Random(std::uint64_t seed) : state(seed) {}
    std::uint64_t Next() {
        std::uint64_t z{(state += 0x9E3779B97F4A7C15ULL)};
        z = (z ^ (z >> 30U)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27U)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31U);
    }
    double Uniform() { return (static_cast<double>(Next() >> 11U) + 0.5) * (1.0 / 9007199254740992.0); }
    double Gauss() {
        const double u1{Uniform()};
        const double u2{Uniform()};
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
    }
    // Poisson: multiplication method below a mean of 30, normal approximation above.
    std::uint32_t Poisson(double mean) {
        if (!(mean > 0.0)) {
            return 0;
        }
        if (mean < 30.0) {
            const double limit{std::exp(-mean)};
            double product{Uniform()};
            std::uint32_t count{0};
            while (product > limit) {
                product *= Uniform();
                ++count;
            }
            return count;
        }
        const double value{mean + std::sqrt(mean) * Gauss() + 0.5};
        return value > 0.0 ? static_cast<std::uint32_t>(value) : 0U;
    }
};

double Beta(double kineticMeV) {
    const double gamma{1.0 + kineticMeV / kElectronMassMeV};
    return std::sqrt(std::max(0.0, 1.0 - 1.0 / (gamma * gamma)));
}

// Continuous-slowing-down stopping power (MeV/mm): the minimum-ionising
// mass stopping power of a CsI-like crystal, 1.24 MeV cm^2/g, scaled by
// 1/beta^2 with a slow logarithmic rise. A stand-in for Geant4's e- physics.
double StoppingPower(double kineticMeV, double density) {
    const double beta{std::max(Beta(kineticMeV), 0.05)};
    const double gamma{1.0 + kineticMeV / kElectronMassMeV};
    return 1.24 * density * 0.1 * (1.0 + 0.08 * std::log(gamma)) / (beta * beta);
}

// Scintillation photon count (G4GOQuasiScintillation.cpp:146-160).
std::uint32_t ScintillationCount(Random& random, double mean, double resolution) {
    if (mean <= 10.0) {
        return random.Poisson(mean);
    }
    const double sigma{resolution * std::sqrt(mean)};
    const double sampled{mean + sigma * random.Gauss() + 0.5};
    return sampled > 0.0 ? static_cast<std::uint32_t>(sampled) : 0U;
}

// Frank-Tamm mean photons per mm for unit charge and a constant index over
// [emin, emax] eV: 369.81 / (eV cm) * (emax - emin) * (1 - 1 / (beta n)^2).
double CerenkovPerMm(double beta, double n, double emin, double emax) {
    const double bn{beta * n};
    if (!(bn > 1.0)) {
        return 0.0;
    }
    return 36.981 * (emax - emin) * (1.0 - 1.0 / (bn * bn));
}

void SetVector(float out[3], double x, double y, double z) {
    out[0] = static_cast<float>(x);
    out[1] = static_cast<float>(y);
    out[2] = static_cast<float>(z);
}

struct EventResult {
    std::vector<g4b_optical_emission> emissions;
};

void GenerateElectronEvent(const g4b_synth_params& p, std::uint32_t eventIndex, EventResult& out) {
    Random random{p.seed * 0xD1342543DE82EF95ULL + 0x632BE59BD9B4E019ULL * (static_cast<std::uint64_t>(eventIndex) + 1U)};
    const double step{p.step_mm > 0.0 ? p.step_mm : 0.1};
    const double density{p.density_g_cm3 > 0.0 ? p.density_g_cm3 : 7.1};
    const double resolution{p.resolution_scale > 0.0 ? p.resolution_scale : 1.0};
    double kinetic{p.energy_min_mev};
    if (p.energy_mode == G4B_SYNTH_ENERGY_UNIFORM) {
        kinetic = p.energy_min_mev + (p.energy_max_mev - p.energy_min_mev) * random.Uniform();
    } else if (p.energy_mode == G4B_SYNTH_ENERGY_LOG_UNIFORM) {
        kinetic = p.energy_min_mev * std::exp(std::log(p.energy_max_mev / p.energy_min_mev) * random.Uniform());
    }
    const double cx{p.crystal_center_mm[0]}, cy{p.crystal_center_mm[1]}, cz{p.crystal_center_mm[2]};
    const double hx{p.crystal_half_size_mm[0]}, hy{p.crystal_half_size_mm[1]}, hz{p.crystal_half_size_mm[2]};
    double x{cx}, y{cy};
    if (p.entry_mode == G4B_SYNTH_ENTRY_UNIFORM_ON_FACE) {
        x = cx + hx * (2.0 * random.Uniform() - 1.0);
        y = cy + hy * (2.0 * random.Uniform() - 1.0);
    }
    double z{cz - hz};
    const double theta{p.max_incidence_deg * kPi / 180.0 * random.Uniform()};
    const double phi{2.0 * kPi * random.Uniform()};
    const double dx{std::sin(theta) * std::cos(phi)};
    const double dy{std::sin(theta) * std::sin(phi)};
    const double dz{std::cos(theta)};
    double time{0.0};
    std::uint32_t nextPhotonID{0};
    const std::uint32_t eventID{p.first_event_id + eventIndex};

    const auto inside{[&](double px, double py, double pz) {
        return std::fabs(px - cx) <= hx && std::fabs(py - cy) <= hy && pz >= cz - hz && pz <= cz + hz;
    }};
    while (kinetic > 0.0 && inside(x, y, z)) {
        const double betaPre{Beta(kinetic)};
        double deposit{StoppingPower(kinetic, density) * step};
        double length{step};
        if (deposit >= kinetic || kinetic - deposit < 0.01) {
            // last step: stop over the fraction of the step the energy allows
            length = step * std::min(1.0, kinetic / std::max(deposit, 1e-12));
            deposit = kinetic;
        }
        const double kineticPost{kinetic - deposit};
        const double betaPost{Beta(kineticPost)};
        const double velocityPre{betaPre * kSpeedOfLightMmPerNs};
        const double velocityPost{betaPost * kSpeedOfLightMmPerNs};

        g4b_optical_emission base{};
        SetVector(base.position_mm, x, y, z);
        base.time_ns = static_cast<float>(time);
        SetVector(base.direction, dx, dy, dz);
        base.step_length_mm = static_cast<float>(length);
        SetVector(base.step_delta_mm, dx * length, dy * length, dz * length);
        base.pre_velocity_mm_per_ns = static_cast<float>(velocityPre);
        base.delta_velocity_mm_per_ns = static_cast<float>(velocityPost - velocityPre);
        base.charge = -1.0F;
        base.event_id = eventID;
        base.volume_id = p.volume_id;
        base.material_id = p.material_id;

        const std::uint32_t scintillation{ScintillationCount(random, p.scintillation_yield_per_mev * deposit, resolution)};
        if (scintillation > 0) {
            g4b_optical_emission record{base};
            record.decay_time_ns = p.decay_time_ns;
            record.rise_time_ns = p.rise_time_ns;
            record.spectrum_id = p.spectrum_id;
            record.type = G4B_EMISSION_SCINTILLATION;
            record.first_photon_id = nextPhotonID;
            record.photon_count = scintillation;
            nextPhotonID += scintillation;
            out.emissions.push_back(record);
        }
        if (p.cerenkov != 0) {
            const double perMmPre{CerenkovPerMm(betaPre, p.rindex, p.cerenkov_energy_min_ev, p.cerenkov_energy_max_ev)};
            const double perMmPost{CerenkovPerMm(betaPost, p.rindex, p.cerenkov_energy_min_ev, p.cerenkov_energy_max_ev)};
            const double perMmMean{
                CerenkovPerMm(0.5 * (betaPre + betaPost), p.rindex, p.cerenkov_energy_min_ev, p.cerenkov_energy_max_ev)};
            const std::uint32_t count{random.Poisson(perMmMean * length)};
            if (count > 0) {
                g4b_optical_emission record{base};
                record.pre_mean_photon_count = static_cast<float>(perMmPre * length);
                record.post_mean_photon_count = static_cast<float>(perMmPost * length);
                record.type = G4B_EMISSION_CERENKOV;
                record.first_photon_id = nextPhotonID;
                record.photon_count = count;
                nextPhotonID += count;
                out.emissions.push_back(record);
            }
        }
        time += length / std::max(0.5 * (velocityPre + velocityPost), 1e-9);
        x += dx * length;
        y += dy * length;
        z += dz * length;
        kinetic = kineticPost;
        if (kinetic <= 0.0) {
            break;
        }
    }
}

g4b_synth_batch* Assemble(std::vector<EventResult>& events, std::uint32_t firstEventID) {
    auto* batch{new g4b_synth_batch{}};
    std::size_t total{0};
    for (const auto& e : events) {
        total += e.emissions.size();
    }
    batch->emissions.reserve(total);
    batch->emissionEventIndices.reserve(total);
    batch->eventIDs.resize(events.size());
    for (std::size_t i{}; i < events.size(); ++i) {
        batch->eventIDs[i] = firstEventID + static_cast<std::uint32_t>(i);
        for (const auto& record : events[i].emissions) {
            batch->emissions.push_back(record);
            batch->emissionEventIndices.push_back(static_cast<std::uint32_t>(i));
            batch->photons += record.photon_count;
        }
        std::vector<g4b_optical_emission>().swap(events[i].emissions);
    }
    return batch;
}

template<class F>
void ParallelFor(std::uint32_t count, std::uint32_t threads, F&& body) {
    if (threads == 0) {
        threads = std::max(1U, std::thread::hardware_concurrency());
    }
    std::atomic<std::uint32_t> next{0};
    const auto worker{[&]() {
        for (;;) {
            const std::uint32_t i{next.fetch_add(1)};
            if (i >= count) {
                break;
            }
            body(i);
        }
    }};
    std::vector<std::thread> pool;
    for (std::uint32_t t{1}; t < threads; ++t) {
        pool.emplace_back(worker);
    }
    worker();
    for (auto& thread : pool) {
        thread.join();
    }
}

}  // namespace

extern "C" {

const char* g4b_synth_last_error(void) { return gSynthError.c_str(); }

int g4b_synth_electrons(const g4b_synth_params* params, g4b_synth_batch** out) {
    if (params == nullptr || out == nullptr) {
        gSynthError = "null argument";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    if (params->energy_mode == G4B_SYNTH_ENERGY_LOG_UNIFORM && !(params->energy_min_mev > 0.0)) {
        gSynthError = "log-uniform energies need a positive minimum";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    try {
        std::vector<EventResult> events(params->event_count);
        ParallelFor(params->event_count, params->threads,
                    [&](std::uint32_t i) { GenerateElectronEvent(*params, i, events[i]); });
        *out = Assemble(events, params->first_event_id);
        if ((*out)->photons > 0xffffffffULL) {
            g4b_synth_free(*out);
            *out = nullptr;
            gSynthError = "synthetic batch exceeds 2^32 photons";
            return G4B_ERR_OVERFLOW;
        }
    } catch (const std::exception& error) {
        gSynthError = error.what();
        return G4B_ERR_INVALID_ARGUMENT;
    }
    return G4B_OK;
}

int g4b_synth_isotropic_photons(uint64_t photonCount, uint32_t photonsPerEvent, uint64_t seed, const float center[3],
                                const float half[3], double wavelengthMin, double wavelengthMax, uint32_t volumeID,
                                uint32_t materialID, g4b_synth_batch** out) {
    if (out == nullptr || center == nullptr || half == nullptr || photonsPerEvent == 0 || photonCount > 0xffffffffULL) {
        gSynthError = "bad argument";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    try {
        auto* batch{new g4b_synth_batch{}};
        batch->emissions.resize(photonCount);
        batch->emissionEventIndices.resize(photonCount);
        const auto eventCount{static_cast<std::uint32_t>((photonCount + photonsPerEvent - 1U) / photonsPerEvent)};
        batch->eventIDs.resize(eventCount);
        ParallelFor(eventCount, 0, [&](std::uint32_t ev) {
            Random random{seed * 0xD1342543DE82EF95ULL + 0x9E3779B97F4A7C15ULL * (static_cast<std::uint64_t>(ev) + 1U)};
            batch->eventIDs[ev] = ev;
            const std::uint64_t begin{static_cast<std::uint64_t>(ev) * photonsPerEvent};
            const std::uint64_t end{std::min<std::uint64_t>(begin + photonsPerEvent, photonCount)};
            for (std::uint64_t i{begin}; i < end; ++i) {
                g4b_optical_emission record{};
                SetVector(record.position_mm, center[0] + half[0] * (2.0 * random.Uniform() - 1.0),
                          center[1] + half[1] * (2.0 * random.Uniform() - 1.0),
                          center[2] + half[2] * (2.0 * random.Uniform() - 1.0));
                const double cosTheta{2.0 * random.Uniform() - 1.0};
                const double sinTheta{std::sqrt(std::max(0.0, 1.0 - cosTheta * cosTheta))};
                const double phi{2.0 * kPi * random.Uniform()};
                const double d[3]{sinTheta * std::cos(phi), sinTheta * std::sin(phi), cosTheta};
                const double e1[3]{cosTheta * std::cos(phi), cosTheta * std::sin(phi), -sinTheta};
                const double e2[3]{-std::sin(phi), std::cos(phi), 0.0};
                const double psi{2.0 * kPi * random.Uniform()};
                SetVector(record.direction, d[0], d[1], d[2]);
                SetVector(record.polarization, std::cos(psi) * e1[0] + std::sin(psi) * e2[0],
                          std::cos(psi) * e1[1] + std::sin(psi) * e2[1], std::cos(psi) * e1[2] + std::sin(psi) * e2[2]);
                const double wavelength{wavelengthMin + (wavelengthMax - wavelengthMin) * random.Uniform()};
                record.energy_ev = static_cast<float>(kHcEvNm / wavelength);
                record.event_id = ev;
                record.first_photon_id = static_cast<std::uint32_t>(i - begin);
                record.photon_count = 1;
                record.volume_id = volumeID;
                record.material_id = materialID;
                record.type = G4B_EMISSION_DIRECT;
                batch->emissions[i] = record;
                batch->emissionEventIndices[i] = ev;
            }
        });
        batch->photons = photonCount;
        *out = batch;
    } catch (const std::exception& error) {
        gSynthError = error.what();
        return G4B_ERR_INVALID_ARGUMENT;
    }
    return G4B_OK;
}

int g4b_synth_view(const g4b_synth_batch* batch, const g4b_optical_emission** emissions, uint32_t* emissionCount,
                   const uint32_t** eventIDs, uint32_t* eventCount, const uint32_t** emissionEventIndices,
                   uint64_t* photonCount) {
    if (batch == nullptr) {
        gSynthError = "null batch";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    if (emissions != nullptr) *emissions = batch->emissions.data();
    if (emissionCount != nullptr) *emissionCount = static_cast<uint32_t>(batch->emissions.size());
    if (eventIDs != nullptr) *eventIDs = batch->eventIDs.data();
    if (eventCount != nullptr) *eventCount = static_cast<uint32_t>(batch->eventIDs.size());
    if (emissionEventIndices != nullptr) *emissionEventIndices = batch->emissionEventIndices.data();
    if (photonCount != nullptr) *photonCount = batch->photons;
    return G4B_OK;
}

void g4b_synth_free(g4b_synth_batch* batch) { delete batch; }

}  // extern "C"

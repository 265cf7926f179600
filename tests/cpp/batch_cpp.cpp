// Two sources of the eigenray_basic environment (waveq3d/test/
// eigenray_test.cc:86-198) run together with wave_queue::run_batch, and
// each again on its own: every eigenray must be the same, bit for bit.
// Prints the counts and exits non-zero on any difference.
#include <cstdio>
#include <vector>

#include "../../underseamodelinglibrary_b200/cpp/usml_b200.hpp"

using namespace usml_b200;
using namespace usml_b200::types;
using namespace usml_b200::ocean;
using namespace usml_b200::eigenrays;
using namespace usml_b200::waveq3d;

int main() {
    compute_earth_radius(45.0);
    boundary_model::csptr bottom(new boundary_flat(3000.0));
    boundary_model::csptr surface(new boundary_flat());
    attenuation_model::csptr attn(new attenuation_constant(0.0));
    profile_model::csptr profile(new profile_linear(1500.0, attn));
    ocean_model::csptr ocean(new ocean_model(surface, bottom, profile));
    seq_vector::csptr freq(new seq_log(10e3, 2.0, 3));
    seq_vector::csptr de(new seq_linear(-60.0, 5.0, 60.0));
    seq_vector::csptr az(new seq_linear(-4.0, 1.0, 4.0));
    wposition target(1, 1, 45.02, -45.0, -1000.0);
    const wposition1 sources[2] = {wposition1(45.0, -45.0, -1000.0), wposition1(45.0, -45.0, -600.0)};

    std::vector<eigenray_collection*> batched, solo;
    std::vector<wave_queue*> queues;
    for (const auto& pos : sources) {
        batched.push_back(new eigenray_collection(freq, pos, target, 1));
        queues.push_back(new wave_queue(ocean, freq, pos, de, az, 0.1, &target));
        queues.back()->add_eigenray_listener(batched.back());
    }
    const double ms = wave_queue::run_batch(queues, {3.5, 3.5});
    int bad = ms > 0.0 ? 0 : 1;
    for (size_t s = 0; s < 2; ++s) {
        solo.push_back(new eigenray_collection(freq, sources[s], target, 1));
        wave_queue wave(ocean, freq, sources[s], de, az, 0.1, &target);
        wave.add_eigenray_listener(solo.back());
        wave.run(3.5);
        const auto& a = batched[s]->eigenrays(0, 0);
        const auto& b = solo[s]->eigenrays(0, 0);
        std::printf("source %zu: batched %zu solo %zu\n", s, a.size(), b.size());
        if (a.size() != b.size() || a.empty()) bad = 1;
        for (size_t k = 0; k < a.size() && k < b.size(); ++k) {
            if (a[k]->travel_time != b[k]->travel_time || a[k]->intensity != b[k]->intensity ||
                a[k]->source_de != b[k]->source_de || a[k]->surface != b[k]->surface ||
                a[k]->bottom != b[k]->bottom)
                bad = 1;
        }
    }
    for (auto* q : queues) delete q;
    for (auto* c : batched) delete c;
    for (auto* c : solo) delete c;
    std::printf("%s\n", bad ? "MISMATCH" : "batch equals solo");
    return bad;
}

// The reflect_flat case of waveq3d/test/reflection_test.cc:168-280 through
// the C++ header: one ray between the surface and a 1000 m flat bottom,
// seen by a reflection_listener.  Bounces alternate bottom / surface every
// 7.450560973 s.  Also checks the queue's read-only accessors and that a
// removed listener hears nothing more.  Prints every reflection and exits
// non-zero on any failed check.
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../underseamodelinglibrary_b200/cpp/usml_b200.hpp"

using namespace usml_b200;
using namespace usml_b200::types;
using namespace usml_b200::ocean;
using namespace usml_b200::waveq3d;

struct event {
    double time, grazing, altitude, nd_rho;
    size_t de, az, type;
};

class recorder : public reflection_listener {
   public:
    std::vector<event> events;
    void reflect(double time, size_t de, size_t az, double /*dt*/, double grazing, double /*speed*/,
                 const wposition1& position, const wvector1& ndirection, size_t type) override {
        events.push_back({time, grazing, position.altitude(), ndirection.rho(), de, az, type});
    }
};

int main() {
    compute_earth_radius(45.0);
    boundary_model::csptr bottom(new boundary_flat(1000.0));
    boundary_model::csptr surface(new boundary_flat());
    profile_model::csptr profile(new profile_linear());
    ocean_model::csptr ocean(new ocean_model(surface, bottom, profile));
    seq_vector::csptr freq(new seq_log(10.0, 10.0, 1));
    seq_vector::csptr de(new seq_linear(-5.183617057, 0.0, 1));
    seq_vector::csptr az(new seq_linear(0.0, 0.0, 1));
    const wposition1 pos(45.0, -45.0, 0.0);

    wave_queue wave(ocean, freq, pos, de, az, 0.1);
    wave.max_caustic(999);
    wave.max_upper(999);
    wave.max_lower(999);
    recorder all, early;
    wave.add_reflection_listener(&all);
    wave.add_reflection_listener(&early);
    int bad = 0;
    auto expect = [&bad](bool ok, const char* what) {
        if (!ok) {
            std::printf("check failed: %s\n", what);
            bad = 1;
        }
    };
    expect(wave.time_step() == 0.1 && wave.num_de() == 1 && wave.num_az() == 1, "time_step / num_de / num_az");
    // a source at the surface starts 0.1 m below it (wave_queue.cc:60-67)
    const wposition1 src = wave.source_pos();
    expect(std::abs(src.latitude() - 45.0) < 1e-9 && std::abs(src.longitude() + 45.0) < 1e-9 &&
               std::abs(src.altitude() + 0.1) < 1e-6,
           "source_pos");

    while (wave.time() < 10.0) wave.step();
    const size_t heard = early.events.size();
    wave.remove_reflection_listener(&early);
    wave.run(60.0);
    expect(early.events.size() == heard && heard >= 1, "removed listener");
    expect(wave.steps() == (int64_t)std::llround(wave.time() / 0.1), "steps");

    for (size_t k = 0; k < all.events.size(); ++k) {
        const event& e = all.events[k];
        std::printf("reflect %zu type %zu time %.9f grazing %.6f altitude %.3f\n", k, e.type, e.time,
                    e.grazing * 180.0 / M_PI, e.altitude);
        const size_t want = (k % 2 == 0) ? WQ3D_VERB_BOTTOM : WQ3D_VERB_SURFACE;
        expect(e.type == want && e.de == 0 && e.az == 0, "type / de / az");
        expect(std::abs(e.time - (double)(k + 1) * 7.450560973) < 1e-4, "time");
        // the earth's curvature makes the ray graze the bottom at 5.0836 deg
        // and the surface at 5.1836 deg
        const double graz = (e.type == WQ3D_VERB_BOTTOM) ? 5.0836 : 5.1836;
        expect(std::abs(e.grazing * 180.0 / M_PI - graz) < 1e-3, "grazing");
        const double alt = (e.type == WQ3D_VERB_BOTTOM) ? -1000.0 : 0.0;
        expect(std::abs(e.altitude - alt) < 0.01, "altitude");
        // the incident direction points into the boundary
        expect((e.type == WQ3D_VERB_BOTTOM) == (e.nd_rho < 0.0), "ndirection");
    }
    expect(all.events.size() >= 7 && early.events.size() < all.events.size(), "reflection count");
    std::printf("reflections %zu, %zu before removal, steps %lld\n", all.events.size(), heard,
                (long long)wave.steps());
    std::printf("%s\n", bad ? "FAILED" : "reflections ok");
    return bad;
}

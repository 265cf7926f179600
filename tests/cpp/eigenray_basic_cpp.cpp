// eigenray_basic (waveq3d/test/eigenray_test.cc:86-198) written against the
// C++ drop-in header, the way a USML caller writes it.  Prints one line per
// eigenray and exits non-zero if a known answer is missed.
#include <cmath>
#include <cstdio>

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
    wposition1 pos(45.0, -45.0, -1000.0);
    seq_vector::csptr de(new seq_linear(-60.0, 5.0, 60.0));
    seq_vector::csptr az(new seq_linear(-4.0, 1.0, 4.0));
    wposition target(1, 1, 45.02, -45.0, -1000.0);

    eigenray_collection collection(freq, pos, target, 1);
    wave_queue wave(ocean, freq, pos, de, az, 0.1, &target);
    wave.add_eigenray_listener(&collection);
    while (wave.time() < 3.5) wave.step();
    collection.sum_eigenrays();

    const auto& rays = collection.eigenrays(0, 0);
    const double tl[3] = {66.9506, 69.5211, 73.2126}, tl_tol[3] = {0.1, 0.1, 4.0};
    const double tt[3] = {1.484018789, 1.995102731, 3.051676949}, t_tol[3] = {0.002, 0.002, 0.02};
    int bad = rays.size() == 3 ? 0 : 1;
    for (size_t k = 0; k < rays.size() && k < 3; ++k) {
        const auto& r = *rays[k];
        std::printf("ray %zu t=%.9f tl=%.4f sde=%.4f tde=%.4f srf=%d btm=%d\n", k, r.travel_time,
                    r.intensity[0], r.source_de, r.target_de, r.surface, r.bottom);
        if (std::fabs(r.intensity[0] - tl[k]) > tl_tol[k]) bad = 1;
        if (std::fabs(r.travel_time - tt[k]) > t_tol[k]) bad = 1;
    }
    std::printf("total tl=%.4f\n", collection.total(0, 0).intensity[0]);
    return bad;
}

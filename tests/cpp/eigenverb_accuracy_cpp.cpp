// eigenverb_accuracy (waveq3d/test/reverb_test.cc:216-310) written against
// the C++ drop-in header: downward rays along az = 0 must meet the 1000 m
// bottom where spherical-earth geometry puts them.  Exits non-zero on a
// miss.
#include <cmath>
#include <cstdio>

#include "../../underseamodelinglibrary_b200/cpp/usml_b200.hpp"

using namespace usml_b200;
using namespace usml_b200::types;
using namespace usml_b200::ocean;
using namespace usml_b200::eigenverbs;
using namespace usml_b200::waveq3d;

int main() {
    earth::radius() = 6371000.0;
    const double depth = 1000.0, c0 = 1500.0, de_spacing = 5.0, az_spacing = 10.0;
    profile_model::csptr profile(new profile_linear(c0));
    boundary_model::csptr surface(new boundary_flat());
    reflect_loss_model::csptr loss(new reflect_loss_rayleigh(1.9, 1.10, 0.8, 0.0, 2.5));  // sand
    boundary_model::csptr bottom(new boundary_flat(depth, loss));
    auto* my_ocean = new ocean_model(surface, bottom, profile);
    my_ocean->add_volume(volume_model::csptr(new volume_flat(300.0, 10.0, -40.0)));
    ocean_model::csptr ocean(my_ocean);

    seq_vector::csptr freq(new seq_log(1000.0, 10.0, 1));
    wposition1 pos(45.0, -45.0, 0.0);
    seq_vector::csptr de(new seq_linear(-80.0, de_spacing, 60.0));
    seq_vector::csptr az(new seq_linear(-40.0, az_spacing, 40.1));

    eigenverb_collection verbs(ocean->num_volume());
    wave_queue wave(ocean, freq, pos, de, az, 0.1);
    wave.add_eigenverb_listener(&verbs);
    while (wave.time() < 3.5) wave.step();

    int bad = 0, checked = 0;
    for (const auto& v : verbs.eigenverbs(eigenverb_model::BOTTOM)) {
        if (!(v->source_de < 0.0 && v->source_az == 0.0)) continue;
        const int segments = v->bottom + v->surface + 1;
        const double R = earth::radius(), Rb = R - depth;
        const double p = R * std::sin(std::fabs(v->source_de)), q = R * R - Rb * Rb;
        double path = p - std::sqrt(p * p - q);
        const double alpha = std::acos((R * R + Rb * Rb - path * path) / (2 * R * Rb));
        const double grazing = std::fabs(v->source_de) - alpha;
        path *= segments;
        const double de_plus = v->source_de + 0.25 * to_radians(de_spacing);
        const double de_minus = v->source_de - 0.25 * to_radians(de_spacing);
        const double az_plus = v->source_az + 0.25 * to_radians(az_spacing);
        const double az_minus = v->source_az - 0.25 * to_radians(az_spacing);
        const double area = (std::sin(de_plus) - std::sin(de_minus)) * (az_plus - az_minus);
        const double de_delta = de_plus - de_minus, az_delta = area / de_delta;
        const double len = path * de_delta / std::sin(grazing), wid = path * az_delta;
        std::printf("verb de=%.1f s=%d b=%d t=%.6f L=%.4f (%.4f) W=%.4f (%.4f)\n", to_degrees(v->source_de),
                    v->surface, v->bottom, v->travel_time, v->length, len, v->width, wid);
        if (std::fabs(v->travel_time - path / c0) > 1e-3 || std::fabs(v->grazing - grazing) > 1e-6 ||
            std::fabs(v->direction - v->source_az) > 1e-6 || std::fabs(v->length - len) > 0.1 ||
            std::fabs(v->width - wid) > 0.1)
            bad = 1;
        ++checked;
    }
    std::printf("checked %d, interfaces %zu\n", checked, verbs.num_interfaces());
    return (bad || checked < 10) ? 1 : 0;
}

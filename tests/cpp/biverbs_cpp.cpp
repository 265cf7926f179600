// The reference's biverb case (biverbs/test/biverbs_test.cc:41-158)
// through the C++ header: 80 analytic bottom footprints around a sensor at
// (0, 0, 0), overlapped with themselves (a monostatic pair) by
// biverb_generator under the -30 dB constant bottom scattering of
// ocean_utils::make_iso.  The search area is the whole quadrilateral
// around each receiver footprint, which gives 109 biverbs here.  Prints
// the count and exits non-zero on any failed check.
#include <cmath>
#include <cstdio>
#include <memory>

#include "../../underseamodelinglibrary_b200/cpp/usml_b200.hpp"

using namespace usml_b200;
using namespace usml_b200::types;
using namespace usml_b200::ocean;
using namespace usml_b200::eigenverbs;
using namespace usml_b200::biverbs;

static const double de_spacing = 10.0;
static const double az_spacing = 10.0;

static eigenverb_model::csptr create_eigenverb(const wposition1& source_pos, double depth, double de, double az,
                                               size_t num_freq) {
    auto verb = std::make_shared<eigenverb_model>();
    const double de_rad = to_radians(de), az_rad = to_radians(az);
    const double grazing = std::abs(de_rad);
    const double slant_range = depth / std::sin(grazing);
    const double horz_range = depth / std::tan(grazing);
    verb->sound_speed = 1500.0;
    verb->travel_time = slant_range / verb->sound_speed;
    verb->length = 0.5 * slant_range * to_radians(de_spacing) / std::sin(grazing);
    verb->width = 0.5 * slant_range * to_radians(az_spacing) * std::cos(grazing);
    verb->position = wposition1(source_pos, horz_range, az_rad);
    verb->position.altitude(-depth);
    verb->direction = az_rad;
    verb->grazing = grazing;
    verb->de_index = (size_t)((90.0 + de) / de_spacing - 1.0);
    verb->az_index = (size_t)(az / az_spacing);
    verb->source_de = de_rad;
    verb->source_az = az_rad;
    verb->power.assign(num_freq, verb->length * verb->width / (slant_range * slant_range));
    return verb;
}

int main() {
    const double depth = 1000.0;
    boundary_model::csptr surface(new boundary_flat(0.0, nullptr, std::make_shared<scattering_constant>(-30.0)));
    boundary_model::csptr bottom(new boundary_flat(depth, nullptr, std::make_shared<scattering_constant>(-30.0)));
    profile_model::csptr profile(new profile_linear(1500.0));
    ocean_model::csptr ocean(new ocean_model(surface, bottom, profile));
    seq_vector::csptr freq(new seq_linear(3000.0, 1.0, 1));
    const wposition1 sensor(0.0, 0.0, 0.0);

    auto verbs = std::make_shared<eigenverb_collection>(0);
    for (double az = 0.0; az <= 90.0; az += az_spacing)
        for (double de = -90.0 + de_spacing; de < 0.0; de += de_spacing)
            verbs->add_eigenverb(create_eigenverb(sensor, depth, de, az, freq->size()), eigenverb_model::BOTTOM);

    int bad = 0;
    auto expect = [&bad](bool ok, const char* what) {
        if (!ok) {
            std::printf("check failed: %s\n", what);
            bad = 1;
        }
    };
    expect(verbs->size(eigenverb_model::BOTTOM) == 80, "80 eigenverbs");
    biverb_generator gen(ocean, verbs, verbs, freq);
    gen.run();
    expect(gen.done(), "done");
    const auto& list = gen.collection()->biverbs(eigenverb_model::BOTTOM);
    expect(list.size() == 109, "109 biverbs");
    expect(gen.collection()->size(eigenverb_model::SURFACE) == 0, "no surface biverbs");
    size_t selfs = 0;
    double last = 0.0;
    for (const auto& b : list) {
        expect(b->travel_time >= last, "ordered by travel time");
        last = b->travel_time;
        expect(b->power.size() == 1 && b->power[0] >= biverb_collection::power_threshold, "power");
        expect(b->duration > 0.0, "duration");
        if (b->source_index == b->receiver_index) {
            ++selfs;
            const auto& v = verbs->eigenverbs(eigenverb_model::BOTTOM)[b->source_index];
            expect(b->travel_time == 2.0 * v->travel_time, "self overlap time");
        }
    }
    expect(selfs == 80, "every footprint overlaps itself");
    std::printf("biverbs %zu, first time %.9f power %.9e\n", list.size(), list.empty() ? 0.0 : list[0]->travel_time,
                list.empty() ? 0.0 : list[0]->power[0]);
    std::printf("%s\n", bad ? "FAILED" : "biverbs ok");
    return bad;
}

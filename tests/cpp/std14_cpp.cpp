// The reference's speed study (studies/cmp_speed/cmp_speed.cc:33-114, the
// STD14 gridded environment near Hawaii) written against the C++ drop-in
// header with profile_grid, boundary_grid and data_grid.  The grids and the
// target ring come from the file named on the command line (written by the
// Python test from the package's STD14 data); the program prints one line
// per eigenray and the curr() front's first rays.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <vector>

#include "../../underseamodelinglibrary_b200/cpp/usml_b200.hpp"

using namespace usml_b200;
using namespace usml_b200::types;
using namespace usml_b200::ocean;
using namespace usml_b200::eigenrays;
using namespace usml_b200::waveq3d;

/* an axis with the values, increments and search kind it had in Python */
struct seq_given : seq_vector {
    seq_given(int kind, const std::vector<double>& v, const std::vector<double>& inc) : _kind(kind) {
        _data = v;
        _inc = inc;
    }
    int axis_kind() const override { return _kind; }
    int _kind;
};

struct reader {
    std::ifstream in;
    explicit reader(const char* path) : in(path, std::ios::binary) {
        if (!in) throw std::runtime_error("cannot open input");
    }
    int32_t i32() {
        int32_t v;
        in.read(reinterpret_cast<char*>(&v), 4);
        return v;
    }
    double f64() {
        double v;
        in.read(reinterpret_cast<char*>(&v), 8);
        return v;
    }
    std::vector<double> vec(size_t n) {
        std::vector<double> v(n);
        in.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(8 * n));
        return v;
    }
    std::shared_ptr<data_grid> grid() {
        const int nd = i32();
        std::vector<seq_vector::csptr> axes;
        size_t total = 1;
        for (int d = 0; d < nd; ++d) {
            const int kind = i32();
            const size_t n = (size_t)i32();
            const auto v = vec(n);
            const auto inc = vec(n);
            axes.push_back(std::make_shared<seq_given>(kind, v, inc));
            total *= n;
        }
        std::vector<int> interp(nd), edge(nd);
        for (int d = 0; d < nd; ++d) interp[d] = i32();
        for (int d = 0; d < nd; ++d) edge[d] = i32();
        auto g = std::make_shared<data_grid>(axes, vec(total));
        for (int d = 0; d < nd; ++d) {
            g->interp_type((size_t)d, interp[d]);
            g->edge_limit((size_t)d, edge[d] != 0);
        }
        return g;
    }
};

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    reader rd(argv[1]);
    earth::radius() = rd.f64();
    auto ssp = rd.grid();
    auto bathy = rd.grid();
    const double src_lat = rd.f64(), src_lng = rd.f64(), src_alt = rd.f64();
    const double time_max = rd.f64();
    const size_t nt = (size_t)rd.i32();
    wposition targets(nt, 1, 0.0, 0.0, 0.0);
    for (size_t k = 0; k < nt; ++k) {
        targets.latitude(k, 0, rd.f64());
        targets.longitude(k, 0, rd.f64());
        targets.altitude(k, 0, rd.f64());
    }
    profile_model::csptr profile(new profile_grid(ssp));
    boundary_model::csptr bottom(new boundary_grid(bathy));
    boundary_model::csptr surface(new boundary_flat());
    ocean_model::csptr ocean(new ocean_model(surface, bottom, profile));
    seq_vector::csptr freq(new seq_linear(250.0, 1.0, 1));
    seq_vector::csptr de(new seq_rayfan(-90.0, 90.0, 181));
    seq_vector::csptr az(new seq_linear(0.0, 15.0, 360.0));
    wposition1 pos(src_lat, src_lng, src_alt);

    eigenray_collection collection(freq, pos, targets, 1);
    wave_queue wave(ocean, freq, pos, de, az, 0.1, &targets, wave_queue::HYBRID_GAUSSIAN, WQ3D_FP64);
    wave.add_eigenray_listener(&collection);
    while (wave.time() < time_max) wave.step();
    for (size_t t = 0; t < nt; ++t)
        for (const auto& r : collection.eigenrays(t, 0))
            std::printf("ray %zu %.12f %.9f %.9f %.9f %.9f %.9f %d %d %d\n", t, r->travel_time, r->intensity[0],
                        r->source_de, r->source_az, r->target_de, r->target_az, r->surface, r->bottom,
                        r->caustic);
    const wave_front f = wave.curr();
    for (size_t k = 0; k < f.rho.size(); k += 997)
        std::printf("front %zu %.6f %.12f %.12f %d\n", k, f.rho[k], f.theta[k], f.phi[k], f.bottom[k]);
    std::printf("steps %lld\n", (long long)wave.steps());
    return 0;
}

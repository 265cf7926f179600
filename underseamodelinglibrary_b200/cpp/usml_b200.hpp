/*
 * usml_b200.hpp -- C++ drop-in for USML's WaveQ3D interface, over the C ABI
 * of include/wq3d.h (header only; link with libwq3d.so).
 *
 * The classes keep the reference's names, constructor arguments and call
 * order (the types/seq_ and types/wposition headers, the ocean/ models, waveq3d/wave_queue.h,
 * eigenrays/eigenray_collection.h), with std::vector in place of Boost
 * uBLAS.  Engine errors become std::runtime_error / std::invalid_argument,
 * as the reference throws.
 */
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "wq3d.h"

namespace usml_b200 {

inline void check(int rc) {
    if (rc == WQ3D_OK) return;
    const std::string msg = wq3d_last_error_string();
    if (rc == WQ3D_ERR_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error("wq3d error " + std::to_string(rc) + ": " + msg);
}

namespace types {

inline double to_radians(double t) { return t * (M_PI / 180.0); }
inline double to_degrees(double t) { return t * (180.0 / M_PI); }

/* seq_vector family (types/seq_vector.h, seq_linear.h, seq_log.h,
 * seq_data.h, seq_rayfan.cc) */
class seq_vector {
   public:
    typedef std::shared_ptr<const seq_vector> csptr;
    /** the axis search the engine uses for this sequence (find_index of
     * seq_linear.h:89-94, seq_log.h:88-94 or seq_data.cc:15-36) */
    virtual int axis_kind() const { return WQ3D_AXIS_DATA; }
    size_t size() const { return _data.size(); }
    double operator()(size_t i) const { return _data[i]; }
    double increment(size_t i) const {
        if (i > _data.size() - 1) i = _data.size() - 1;
        return _inc[i];
    }
    const std::vector<double>& data() const { return _data; }
    const std::vector<double>& increments() const { return _inc; }
    virtual ~seq_vector() {}

   protected:
    std::vector<double> _data, _inc;
};

class seq_linear : public seq_vector {
   public:
    int axis_kind() const override { return WQ3D_AXIS_LINEAR; }
    seq_linear(double first, double increment, int size) { init(first, increment, (size_t)size); }
    seq_linear(double first, double increment, double last) {
        const size_t n = (increment == 0.0)
                             ? 1
                             : (size_t)std::max(1.0, std::floor(1.0 + (last + increment / 10 - first) / increment));
        init(first, increment, n);
    }

   private:
    void init(double first, double inc, size_t n) {
        _data.resize(n);
        _inc.assign(n, inc);
        double v = first;
        for (size_t k = 0; k < n; ++k) {
            _data[k] = v;
            v += inc;
        }
    }
};

class seq_log : public seq_vector {
   public:
    int axis_kind() const override { return WQ3D_AXIS_LOG; }
    seq_log(double first, double increment, int size) { init(first, increment, (size_t)size); }
    seq_log(double first, double increment, double last) {
        const size_t n = (increment == 1.0)
                             ? 1
                             : (size_t)std::max(1.0, std::floor(1.0 + std::log((last + increment / 10) / first) /
                                                                          std::log(increment)));
        init(first, increment, n);
    }

   private:
    void init(double first, double inc, size_t n) {
        _data.resize(n);
        _inc.assign(n, 0.0);
        double v = first;
        for (size_t k = 0; k < n; ++k) {
            _data[k] = v;
            v *= inc;
            if (k > 0) {
                _inc[k - 1] = _data[k] - _data[k - 1];
                _inc[k] = _inc[k - 1];
            }
        }
    }
};

class seq_data : public seq_vector {
   public:
    explicit seq_data(const std::vector<double>& v) { init(v); }

   protected:
    seq_data() {}
    void init(const std::vector<double>& v) {
        _data = v;
        _inc.assign(v.size(), 0.0);
        if (v.size() < 2) return;
        double left = v[1] - v[0];
        _inc[0] = left;
        for (size_t n = 1; n < v.size(); ++n) {
            double right = left;
            if (n < v.size() - 1) {
                right = v[n + 1] - v[n];
                if (left * right <= 0) throw std::invalid_argument("series not monotonic");
            }
            left = right;
            _inc[n] = left;
        }
    }
};

class seq_rayfan : public seq_data {
   public:
    seq_rayfan(double first = -90.0, double last = 90.0, size_t size = 181, double center = 0.0,
               double spread = 6.0) {
        if (first > last) std::swap(first, last);
        const double a0 = std::atan((first - center) / spread);
        const double a1 = std::atan((last - center) / spread);
        const double scale = (a1 - a0) / double(size - 1);
        std::vector<double> v(size);
        for (size_t n = 0; n < size; ++n) v[n] = center + std::tan(a0 + scale * (double)n) * spread;
        init(v);
    }
};

/* data_grid<N> (types/data_grid.h, gen_grid.h:83-520): values on up to
 * three axes, row-major with the last axis fastest; linear interpolation
 * with edge limiting on every axis unless set otherwise
 * (data_grid.h:315-316) */
class data_grid {
   public:
    typedef std::shared_ptr<const data_grid> csptr;
    data_grid(const std::vector<seq_vector::csptr>& axes, const std::vector<double>& data)
        : _axes(axes), _data(data) {
        if (axes.empty() || axes.size() > 3) throw std::invalid_argument("data_grid takes 1 to 3 axes");
        size_t n = 1;
        for (const auto& a : axes) n *= a->size();
        if (n != data.size()) throw std::invalid_argument("data_grid: data size does not match the axes");
        for (size_t d = 0; d < 3; ++d) {
            _interp[d] = WQ3D_INTERP_LINEAR;
            _edge[d] = 1;
        }
    }
    size_t dim() const { return _axes.size(); }
    const seq_vector::csptr& axis(size_t d) const { return _axes.at(d); }
    /** data_grid::interp_type (data_grid.h:137-145): WQ3D_INTERP_* */
    void interp_type(size_t d, int kind) { _interp[d] = kind; }
    int interp_type(size_t d) const { return _interp[d]; }
    /** data_grid::edge_limit (data_grid.h:159-166) */
    void edge_limit(size_t d, bool on) { _edge[d] = on ? 1 : 0; }
    const std::vector<double>& data() const { return _data; }
    /** the engine's description; the pointers stay valid while this grid lives */
    void fill(wq3d_grid_desc* g) const {
        g->ndim = (int)_axes.size();
        for (size_t d = 0; d < _axes.size(); ++d) {
            g->axis[d] = _axes[d]->data().data();
            g->axis_inc[d] = _axes[d]->increments().data();
            g->axis_size[d] = _axes[d]->size();
            g->axis_kind[d] = _axes[d]->axis_kind();
            g->interp[d] = _interp[d];
            g->edge_limit[d] = _edge[d];
        }
        g->data = _data.data();
    }

   private:
    std::vector<seq_vector::csptr> _axes;
    std::vector<double> _data;
    int _interp[3];
    int _edge[3];
};

/* wposition::earth_radius and compute_earth_radius (types/wposition.cc) */
struct earth {
    static double& radius() {
        static double r = 6371000.0;
        return r;
    }
};
inline void compute_earth_radius(double latitude) {
    const double a = 6378137.0, f = 1.0 / 298.257223563, e2 = f * (2.0 - f);
    const double s = std::sin(to_radians(latitude));
    const double w = std::sqrt(1.0 - e2 * s * s);
    earth::radius() = std::sqrt((a * (1 - e2) / (w * w * w)) * (a / w));
}

class wposition1 {
   public:
    wposition1() {}
    wposition1(double lat, double lng, double alt) {
        latitude(lat);
        longitude(lng);
        altitude(alt);
    }
    /* great circle range (m) and bearing (rad) from a point
     * (types/wposition1.cc:23-37) */
    wposition1(const wposition1& location, double range, double bearing) {
        const double lat1 = to_radians(location.latitude());
        const double lng1 = to_radians(location.longitude());
        const double R = earth::radius() + location.altitude();
        range /= R;
        const double lat2 = std::asin(std::sin(lat1) * std::cos(range) + std::cos(lat1) * std::sin(range) * std::cos(bearing));
        const double lng2 = lng1 + std::atan2(std::sin(bearing) * std::sin(range) * std::cos(lat1),
                                              std::cos(range) - std::sin(lat1) * std::sin(lat2));
        latitude(to_degrees(lat2));
        longitude(to_degrees(lng2));
        altitude(location.altitude());
    }
    double rho() const { return _r; }
    double theta() const { return _t; }
    double phi() const { return _p; }
    void rho(double v) { _r = v; }
    void theta(double v) { _t = v; }
    void phi(double v) { _p = v; }
    double latitude() const { return 90.0 - to_degrees(_t); }
    double longitude() const { return to_degrees(_p); }
    double altitude() const { return _r - earth::radius(); }
    void latitude(double v) { _t = to_radians(90.0 - v); }
    void longitude(double v) { _p = to_radians(v); }
    void altitude(double v) { _r = v + earth::radius(); }

   private:
    double _r = 0, _t = 0, _p = 0;
};

/* wvector1 (types/wvector1.h): one vector in spherical earth coordinates */
class wvector1 {
   public:
    wvector1() {}
    wvector1(double rho, double theta, double phi) : _r(rho), _t(theta), _p(phi) {}
    double rho() const { return _r; }
    double theta() const { return _t; }
    double phi() const { return _p; }
    void rho(double v) { _r = v; }
    void theta(double v) { _t = v; }
    void phi(double v) { _p = v; }

   private:
    double _r = 0, _t = 0, _p = 0;
};

class wposition {
   public:
    wposition(size_t rows = 1, size_t cols = 1, double lat = 0.0, double lng = 0.0, double alt = 0.0)
        : _n1(rows), _n2(cols), _v(rows * cols, wposition1(lat, lng, alt)) {}
    size_t size1() const { return _n1; }
    size_t size2() const { return _n2; }
    wposition1& at(size_t r, size_t c) { return _v[r * _n2 + c]; }
    const wposition1& at(size_t r, size_t c) const { return _v[r * _n2 + c]; }
    /* element accessors of types/wposition.h */
    double latitude(size_t r, size_t c) const { return at(r, c).latitude(); }
    double longitude(size_t r, size_t c) const { return at(r, c).longitude(); }
    double altitude(size_t r, size_t c) const { return at(r, c).altitude(); }
    void latitude(size_t r, size_t c, double v) { at(r, c).latitude(v); }
    void longitude(size_t r, size_t c, double v) { at(r, c).longitude(v); }
    void altitude(size_t r, size_t c, double v) { at(r, c).altitude(v); }
    std::vector<double> packed() const {
        const size_t n = _v.size();
        std::vector<double> out(3 * n);
        for (size_t i = 0; i < n; ++i) {
            out[i] = _v[i].rho();
            out[n + i] = _v[i].theta();
            out[2 * n + i] = _v[i].phi();
        }
        return out;
    }

   private:
    size_t _n1, _n2;
    std::vector<wposition1> _v;
};

}  // namespace types

namespace ocean {

struct attenuation_model {
    typedef std::shared_ptr<const attenuation_model> csptr;
    int kind = WQ3D_ATTEN_THORP;
    double coef = 0.0;
};
struct attenuation_thorp : attenuation_model {};
struct attenuation_constant : attenuation_model {
    explicit attenuation_constant(double c) {
        kind = WQ3D_ATTEN_CONSTANT;
        coef = c;
    }
};

class profile_model {
   public:
    typedef std::shared_ptr<const profile_model> csptr;
    explicit profile_model(const attenuation_model::csptr& a) : _atten(a) {}
    void flat_earth(bool f) { _flat = f; }
    void fill(wq3d_profile_desc* d) const {
        d->kind = _kind;
        for (int k = 0; k < 4; ++k) d->p[k] = _p[k];
        d->flat_earth = _flat ? 1 : 0;
        d->attenuation = _atten ? _atten->kind : WQ3D_ATTEN_THORP;
        d->attenuation_coef = _atten ? _atten->coef : 0.0;
        fill_grid(d);
    }
    virtual void fill_grid(wq3d_profile_desc*) const {}
    virtual ~profile_model() {}

   protected:
    int _kind = WQ3D_PROFILE_LINEAR;
    double _p[4] = {0, 0, 0, 0};
    bool _flat = false;
    attenuation_model::csptr _atten;
};

struct profile_linear : profile_model {
    explicit profile_linear(double c0 = 1500.0, const attenuation_model::csptr& a = nullptr) : profile_model(a) {
        _p[0] = c0;
    }
    profile_linear(double c0, double g0, const attenuation_model::csptr& a = nullptr) : profile_model(a) {
        _p[0] = c0;
        _p[1] = g0;
        _p[3] = g0;
    }
    profile_linear(double c0, double g0, double z1, double g1, const attenuation_model::csptr& a = nullptr)
        : profile_model(a) {
        _p[0] = c0;
        _p[1] = g0;
        _p[2] = z1;
        _p[3] = g1;
    }
};

struct profile_munk : profile_model {
    explicit profile_munk(double axis_depth = 1300.0, double scale = 1300.0, double axis_speed = 1500.0,
                          double epsilon = 7.37e-3, const attenuation_model::csptr& a = nullptr)
        : profile_model(a) {
        _kind = WQ3D_PROFILE_MUNK;
        _p[0] = axis_depth;
        _p[1] = scale;
        _p[2] = axis_speed;
        _p[3] = epsilon;
    }
};

/* profile_catenary (ocean/profile_catenary.cc:14-29): c = c1 cosh((z - z1) / g1) */
struct profile_catenary : profile_model {
    profile_catenary(double c1, double g1, double z1, const attenuation_model::csptr& a = nullptr)
        : profile_model(a) {
        _kind = WQ3D_PROFILE_CATENARY;
        _p[0] = c1;
        _p[1] = g1;
        _p[2] = z1;
    }
};

/* profile_n2 (ocean/profile_n2.cc:14-24): the n^2 linear profile */
struct profile_n2 : profile_model {
    profile_n2(double c0, double g0, const attenuation_model::csptr& a = nullptr) : profile_model(a) {
        _kind = WQ3D_PROFILE_N2;
        _p[0] = c0;
        _p[1] = g0;
    }
};

/* profile_grid<N> (ocean/profile_grid.h:68-130): sound speed on a grid over
 * (rho[, theta[, phi]]) */
struct profile_grid : profile_model {
    explicit profile_grid(const types::data_grid::csptr& grid, const attenuation_model::csptr& a = nullptr)
        : profile_model(a), _grid(grid) {
        _kind = WQ3D_PROFILE_GRID;
    }
    void fill_grid(wq3d_profile_desc* d) const { _grid->fill(&d->grid); }

   private:
    types::data_grid::csptr _grid;
};

struct reflect_loss_model {
    typedef std::shared_ptr<const reflect_loss_model> csptr;
    wq3d_reflect_loss_desc d{WQ3D_LOSS_DEFAULT, {0, 0, 0, 0, 0}};
};
struct reflect_loss_constant : reflect_loss_model {
    explicit reflect_loss_constant(double amp, double phase = 0.0) { d = {WQ3D_LOSS_CONSTANT, {amp, phase, 0, 0, 0}}; }
};
struct reflect_loss_rayleigh : reflect_loss_model {
    reflect_loss_rayleigh(double density, double speed, double att = 0.0, double shear = 0.0, double satt = 0.0) {
        d = {WQ3D_LOSS_RAYLEIGH, {density, speed, att, shear, satt}};
    }
};

/* reflect_loss_eckart (ocean/reflect_loss_eckart.h:76-85): rough-surface
 * loss from the wind speed (m/s) */
struct reflect_loss_eckart : reflect_loss_model {
    explicit reflect_loss_eckart(double wind_speed) { d = {WQ3D_LOSS_ECKART, {wind_speed, 0, 0, 0, 0}}; }
};

/* scattering strength models (ocean/scattering_{constant,lambert,chapman}.h),
 * evaluated on the GPU by wq3d_biverbs */
struct scattering_model {
    typedef std::shared_ptr<const scattering_model> csptr;
    wq3d_scattering_desc d{WQ3D_SCATTER_CONSTANT, 0, -300.0};
};
struct scattering_constant : scattering_model {
    explicit scattering_constant(double amplitude = -300.0) { d = {WQ3D_SCATTER_CONSTANT, 0, amplitude}; }
};
struct scattering_lambert : scattering_model {
    explicit scattering_lambert(double bss = -27.0) { d = {WQ3D_SCATTER_LAMBERT, 0, bss}; }
};
struct scattering_chapman : scattering_model {
    explicit scattering_chapman(double wind_speed) { d = {WQ3D_SCATTER_CHAPMAN, 0, wind_speed}; }
};

class boundary_model {
   public:
    typedef std::shared_ptr<const boundary_model> csptr;
    explicit boundary_model(const scattering_model::csptr& scattering = nullptr)
        : _scattering(scattering ? scattering : std::make_shared<scattering_constant>()) {}
    virtual void fill(wq3d_boundary_desc* d) const = 0;
    virtual ~boundary_model() {}
    /** boundary_model::scattering: scattering_constant(-300 dB) unless given */
    const scattering_model::csptr& scattering() const { return _scattering; }

   private:
    scattering_model::csptr _scattering;
};

class boundary_flat : public boundary_model {
   public:
    explicit boundary_flat(double depth = 0.0, const reflect_loss_model::csptr& loss = nullptr,
                           const scattering_model::csptr& scattering = nullptr)
        : boundary_model(scattering), _depth(depth), _loss(loss) {}
    void fill(wq3d_boundary_desc* d) const override {
        d->kind = WQ3D_BOUNDARY_FLAT;
        d->depth = _depth;
        d->loss = _loss ? _loss->d : wq3d_reflect_loss_desc{WQ3D_LOSS_DEFAULT, {0, 0, 0, 0, 0}};
    }

   private:
    double _depth;
    reflect_loss_model::csptr _loss;
};

class boundary_slope : public boundary_model {
   public:
    boundary_slope(const types::wposition1& loc, double depth, double lat_slope, double lng_slope = 0.0,
                   const reflect_loss_model::csptr& loss = nullptr,
                   const scattering_model::csptr& scattering = nullptr)
        : boundary_model(scattering), _loc(loc), _depth(depth), _lat(lat_slope), _lng(lng_slope), _loss(loss) {}
    void fill(wq3d_boundary_desc* d) const override {
        d->kind = WQ3D_BOUNDARY_SLOPE;
        d->depth = _depth;
        d->location[0] = _loc.rho();
        d->location[1] = _loc.theta();
        d->location[2] = _loc.phi();
        d->lat_slope = _lat;
        d->lng_slope = _lng;
        d->loss = _loss ? _loss->d : wq3d_reflect_loss_desc{WQ3D_LOSS_DEFAULT, {0, 0, 0, 0, 0}};
    }

   private:
    types::wposition1 _loc;
    double _depth, _lat, _lng;
    reflect_loss_model::csptr _loss;
};

/* boundary_grid<N> (ocean/boundary_grid.h:40-204): boundary rho on a grid
 * over theta[, phi]; the Rayleigh sand loss unless one is given
 * (boundary_grid.h:56-59) */
class boundary_grid : public boundary_model {
   public:
    explicit boundary_grid(const types::data_grid::csptr& grid, const reflect_loss_model::csptr& loss = nullptr,
                           const scattering_model::csptr& scattering = nullptr)
        : boundary_model(scattering), _grid(grid), _loss(loss) {}
    void fill(wq3d_boundary_desc* d) const override {
        d->kind = WQ3D_BOUNDARY_GRID;
        _grid->fill(&d->grid);
        d->loss = _loss ? _loss->d : wq3d_reflect_loss_desc{WQ3D_LOSS_DEFAULT, {0, 0, 0, 0, 0}};
    }

   private:
    types::data_grid::csptr _grid;
    reflect_loss_model::csptr _loss;
};

/* volume_flat (ocean/volume_flat.h:32-37): a scattering layer at a
 * constant depth */
struct volume_model {
    typedef std::shared_ptr<const volume_model> csptr;
    wq3d_volume_desc d{0.0, 0.0, -300.0};
    scattering_model::csptr scattering = std::make_shared<scattering_constant>();
};
struct volume_flat : volume_model {
    explicit volume_flat(double depth = 0.0, double thickness = 0.0, double amplitude = -300.0) {
        d = {depth, thickness, amplitude};
        scattering = std::make_shared<scattering_constant>(amplitude);
    }
    /* volume_flat(depth, thickness, scattering) (volume_flat.h:47-50) */
    volume_flat(double depth, double thickness, const scattering_model::csptr& model) {
        d = {depth, thickness, model->d.kind == WQ3D_SCATTER_CONSTANT ? model->d.p : -300.0};
        scattering = model;
    }
};

/* ocean_model (ocean/ocean_model.h); the device copy is built on first
 * use, so volume layers can be added after construction as in the
 * reference */
class ocean_model {
   public:
    typedef std::shared_ptr<const ocean_model> csptr;
    ocean_model(const boundary_model::csptr& surface, const boundary_model::csptr& bottom,
                const profile_model::csptr& profile)
        : _surface(surface), _bottom(bottom), _profile(profile) {
        _d.earth_radius = types::earth::radius();
        profile->fill(&_d.profile);
        surface->fill(&_d.surface);
        bottom->fill(&_d.bottom);
    }
    /* ocean_model::add_volume (ocean/ocean_model.h:52) */
    void add_volume(const volume_model::csptr& layer) {
        if (_h) throw std::logic_error("add volume layers before the ocean is first used");
        if (_d.num_volume >= WQ3D_MAX_VOLUME) throw std::invalid_argument("too many volume layers");
        _d.volume[_d.num_volume++] = layer->d;
        _volume.push_back(layer);
    }
    size_t num_volume() const { return (size_t)_d.num_volume; }
    /** the scattering model of an interface, as ocean_model::scattering
     * picks it (ocean/ocean_model.h:88-112) */
    const scattering_model::csptr& scattering_model_of(size_t interface) const {
        if (interface == 0) return _bottom->scattering();
        if (interface == 1) return _surface->scattering();
        return _volume.at((interface - 2) / 2)->scattering;
    }
    const wq3d_ocean* handle() const {
        if (!_h) {
            wq3d_ocean* o = nullptr;
            check(wq3d_ocean_create(&_d, &o));
            _h.reset(o, [](wq3d_ocean* p) { wq3d_ocean_destroy(p); });
        }
        return _h.get();
    }

   private:
    boundary_model::csptr _surface, _bottom;
    profile_model::csptr _profile;
    std::vector<volume_model::csptr> _volume;
    wq3d_ocean_desc _d{};
    mutable std::shared_ptr<wq3d_ocean> _h;
};

}  // namespace ocean

namespace eigenrays {

/* eigenrays/eigenray_model.h */
struct eigenray_model {
    typedef std::shared_ptr<const eigenray_model> csptr;
    double travel_time = 0, source_de = 0, source_az = 0, target_de = 0, target_az = 0;
    std::vector<double> intensity, phase;
    int surface = 0, bottom = 0, caustic = 0, upper = 0, lower = 0;
};

/* eigenrays/eigenray_listener.h:41-53 */
class eigenray_listener {
   public:
    virtual void add_eigenray(size_t t1, size_t t2, eigenray_model::csptr ray, size_t run_id) = 0;
    virtual void check_eigenrays(double /*time*/, size_t /*run_id*/) {}
    virtual ~eigenray_listener() {}
};

/* eigenrays/eigenray_collection.{h,cc} (add and coherent sum) */
class eigenray_collection : public eigenray_listener {
   public:
    eigenray_collection(const types::seq_vector::csptr& freq, const types::wposition1&,
                        const types::wposition& targets, size_t = 0, bool coherent = true)
        : _freq(freq), _n1(targets.size1()), _n2(targets.size2()), _rays(_n1 * _n2), _total(_n1 * _n2),
          _coherent(coherent) {}
    void add_eigenray(size_t t1, size_t t2, eigenray_model::csptr ray, size_t) override {
        _rays[t1 * _n2 + t2].push_back(ray);
    }
    const std::vector<eigenray_model::csptr>& eigenrays(size_t t1, size_t t2) const { return _rays[t1 * _n2 + t2]; }
    const eigenray_model& total(size_t t1, size_t t2) const { return _total[t1 * _n2 + t2]; }
    /** eigenray_collection::sum_eigenrays (eigenray_collection.cc:105-191)
     * on the GPU (wq3d_sum_eigenrays) */
    void sum_eigenrays() {
        const size_t nf = _freq->size();
        std::vector<wq3d_eigenray> rec;
        std::vector<double> inten, phase;
        for (size_t t = 0; t < _rays.size(); ++t)
            for (const auto& r : _rays[t]) {
                wq3d_eigenray e{};
                e.time = r->travel_time;
                e.source_de = r->source_de;
                e.source_az = r->source_az;
                e.target_de = r->target_de;
                e.target_az = r->target_az;
                e.surface = r->surface;
                e.bottom = r->bottom;
                e.caustic = r->caustic;
                e.upper = r->upper;
                e.lower = r->lower;
                e.t1 = (int32_t)(t / _n2);
                e.t2 = (int32_t)(t % _n2);
                rec.push_back(e);
                inten.insert(inten.end(), r->intensity.begin(), r->intensity.end());
                phase.insert(phase.end(), r->phase.begin(), r->phase.end());
            }
        std::vector<wq3d_eigenray> tot(_rays.size());
        std::vector<double> ti(_rays.size() * nf), tp(_rays.size() * nf);
        check(wq3d_sum_eigenrays(rec.data(), inten.data(), phase.data(), rec.size(), _freq->data().data(), nf,
                                 _n1, _n2, _coherent ? 1 : 0, tot.data(), ti.data(), tp.data()));
        for (size_t t = 0; t < _rays.size(); ++t) {
            eigenray_model& o = _total[t];
            o.travel_time = tot[t].time;
            o.source_de = tot[t].source_de;
            o.source_az = tot[t].source_az;
            o.target_de = tot[t].target_de;
            o.target_az = tot[t].target_az;
            o.surface = tot[t].surface;
            o.bottom = tot[t].bottom;
            o.caustic = tot[t].caustic;
            o.upper = tot[t].upper;
            o.lower = tot[t].lower;
            o.intensity.assign(ti.begin() + t * nf, ti.begin() + (t + 1) * nf);
            o.phase.assign(tp.begin() + t * nf, tp.begin() + (t + 1) * nf);
        }
    }

   private:
    types::seq_vector::csptr _freq;
    size_t _n1, _n2;
    std::vector<std::vector<eigenray_model::csptr>> _rays;
    std::vector<eigenray_model> _total;
    bool _coherent;
};

}  // namespace eigenrays

namespace eigenverbs {

/* eigenverbs/eigenverb_model.h:34-150 */
struct eigenverb_model {
    typedef std::shared_ptr<const eigenverb_model> csptr;
    enum interface_type { BOTTOM = WQ3D_VERB_BOTTOM, SURFACE = WQ3D_VERB_SURFACE,
                          VOLUME_UPPER = WQ3D_VERB_VOLUME_UPPER, VOLUME_LOWER = WQ3D_VERB_VOLUME_LOWER };
    double travel_time = 0;
    std::vector<double> power;
    double length = 0, width = 0;
    types::wposition1 position;
    double direction = 0, grazing = 0, sound_speed = 0;
    size_t de_index = 0, az_index = 0;
    double source_de = 0, source_az = 0;
    int surface = 0, bottom = 0, caustic = 0, upper = 0, lower = 0;
};

/* eigenverbs/eigenverb_listener.h:23-41 */
class eigenverb_listener {
   public:
    virtual void add_eigenverb(eigenverb_model::csptr verb, size_t interface_num) = 0;
    virtual ~eigenverb_listener() {}
};

/* eigenverbs/eigenverb_collection.h: one list per interface */
class eigenverb_collection : public eigenverb_listener {
   public:
    /** size of the biverb search area, in footprint lengths and widths
     * (eigenverb_collection.cc:32) */
    static inline double search_scale = 1.5;
    explicit eigenverb_collection(size_t num_volumes = 0) : _collection((1 + num_volumes) * 2) {}
    size_t num_interfaces() const { return _collection.size(); }
    size_t size(size_t interface_num) const { return _collection[interface_num].size(); }
    const std::vector<eigenverb_model::csptr>& eigenverbs(size_t interface_num) const {
        return _collection[interface_num];
    }
    void add_eigenverb(eigenverb_model::csptr verb, size_t interface_num) override {
        _collection[interface_num].push_back(verb);
    }

   private:
    std::vector<std::vector<eigenverb_model::csptr>> _collection;
};

}  // namespace eigenverbs

namespace biverbs {

/* biverbs/biverb_model.h:24-104, plus the indices of the source and
 * receiver eigenverbs it overlaps */
struct biverb_model {
    typedef std::shared_ptr<const biverb_model> csptr;
    double travel_time = 0;
    std::vector<double> power;
    double duration = 0;
    size_t de_index = 0, az_index = 0;
    double source_de = 0, source_az = 0, receiver_de = 0, receiver_az = 0;
    int source_surface = 0, source_bottom = 0, source_caustic = 0, source_upper = 0, source_lower = 0;
    int receiver_surface = 0, receiver_bottom = 0, receiver_caustic = 0, receiver_upper = 0, receiver_lower = 0;
    size_t source_index = 0, receiver_index = 0;
};

/* biverbs/biverb_collection.h: one list per interface, ordered by travel
 * time; equal travel times keep the order they were added in (the
 * reference's multimap) */
class biverb_collection {
   public:
    typedef std::shared_ptr<const biverb_collection> csptr;
    /** biverb_collection.cc:28 */
    static inline double power_threshold = 1e-20;
    explicit biverb_collection(size_t num_volumes = 0) : _collection((1 + num_volumes) * 2) {}
    size_t num_interfaces() const { return _collection.size(); }
    size_t size(size_t interface_num) const { return _collection[interface_num].size(); }
    const std::vector<biverb_model::csptr>& biverbs(size_t interface_num) const { return _collection[interface_num]; }
    void add_biverbs(const std::vector<biverb_model::csptr>& list, size_t interface_num) {
        auto& c = _collection[interface_num];
        c.insert(c.end(), list.begin(), list.end());
        std::stable_sort(c.begin(), c.end(), [](const biverb_model::csptr& a, const biverb_model::csptr& b) {
            return a->travel_time < b->travel_time;
        });
    }

   private:
    std::vector<std::vector<biverb_model::csptr>> _collection;
};

/* biverb_generator (biverbs/biverb_generator.cc:26-82): one wq3d_biverbs
 * call per interface; the ocean and frequencies, process-wide singletons
 * in the reference, are arguments */
class biverb_generator {
   public:
    biverb_generator(const ocean::ocean_model::csptr& ocean,
                     const std::shared_ptr<const eigenverbs::eigenverb_collection>& src,
                     const std::shared_ptr<const eigenverbs::eigenverb_collection>& rcv,
                     const types::seq_vector::csptr& freq)
        : _ocean(ocean), _src(src), _rcv(rcv), _freq(freq) {}
    void abort() { _abort = true; }
    bool done() const { return _done; }
    const biverb_collection::csptr& collection() const { return _collection; }

    void run() {
        if (_abort) return;
        auto coll = std::make_shared<biverb_collection>(_ocean->num_volume());
        const size_t nf = _freq->size();
        for (size_t interface = 0; interface < _rcv->num_interfaces(); ++interface) {
            if (interface >= _src->num_interfaces()) break;
            const auto& sv = _src->eigenverbs(interface);
            const auto& rv = _rcv->eigenverbs(interface);
            if (sv.empty() || rv.empty()) continue;
            std::vector<wq3d_eigenverb> s, r;
            std::vector<double> sp, rp;
            pack(sv, nf, &s, &sp);
            pack(rv, nf, &r, &rp);
            const wq3d_scattering_desc sc = _ocean->scattering_model_of(interface)->d;
            size_t n = 0;
            call(s, sp, r, rp, sc, nullptr, nullptr, 0, &n);
            std::vector<wq3d_biverb> out(n);
            std::vector<double> power(n * nf);
            call(s, sp, r, rp, sc, out.data(), power.data(), n, &n);
            std::vector<biverb_model::csptr> list;
            list.reserve(n);
            for (size_t k = 0; k < n; ++k) list.push_back(to_model(out[k], &power[k * nf], nf));
            coll->add_biverbs(list, interface);
            if (_abort) return;
        }
        _collection = coll;
        _done = true;
    }

   private:
    static void pack(const std::vector<eigenverbs::eigenverb_model::csptr>& verbs, size_t nf,
                     std::vector<wq3d_eigenverb>* recs, std::vector<double>* power) {
        recs->assign(verbs.size(), wq3d_eigenverb{});
        power->assign(verbs.size() * nf, 0.0);
        for (size_t i = 0; i < verbs.size(); ++i) {
            const auto& v = *verbs[i];
            wq3d_eigenverb& e = (*recs)[i];
            e.travel_time = v.travel_time;
            e.length = v.length;
            e.width = v.width;
            e.position[0] = v.position.rho();
            e.position[1] = v.position.theta();
            e.position[2] = v.position.phi();
            e.direction = v.direction;
            e.grazing = v.grazing;
            e.sound_speed = v.sound_speed;
            e.source_de = v.source_de;
            e.source_az = v.source_az;
            e.de = (int32_t)v.de_index;
            e.az = (int32_t)v.az_index;
            e.surface = v.surface;
            e.bottom = v.bottom;
            e.caustic = v.caustic;
            e.upper = v.upper;
            e.lower = v.lower;
            for (size_t f = 0; f < nf; ++f) (*power)[i * nf + f] = v.power.size() == nf ? v.power[f] : v.power.at(0);
        }
    }
    void call(const std::vector<wq3d_eigenverb>& s, const std::vector<double>& sp,
              const std::vector<wq3d_eigenverb>& r, const std::vector<double>& rp, const wq3d_scattering_desc& sc,
              wq3d_biverb* out, double* power, size_t capacity, size_t* n) const {
        check(wq3d_biverbs(s.data(), sp.data(), s.size(), r.data(), rp.data(), r.size(), _freq->data().data(),
                           _freq->size(), &sc, types::earth::radius(), eigenverbs::eigenverb_collection::search_scale,
                           biverb_collection::power_threshold, out, power, capacity, n));
    }
    static biverb_model::csptr to_model(const wq3d_biverb& b, const double* power, size_t nf) {
        auto m = std::make_shared<biverb_model>();
        m->travel_time = b.travel_time;
        m->power.assign(power, power + nf);
        m->duration = b.duration;
        m->de_index = (size_t)b.de_index;
        m->az_index = (size_t)b.az_index;
        m->source_de = b.source_de;
        m->source_az = b.source_az;
        m->receiver_de = b.receiver_de;
        m->receiver_az = b.receiver_az;
        m->source_surface = b.source_surface;
        m->source_bottom = b.source_bottom;
        m->source_caustic = b.source_caustic;
        m->source_upper = b.source_upper;
        m->source_lower = b.source_lower;
        m->receiver_surface = b.receiver_surface;
        m->receiver_bottom = b.receiver_bottom;
        m->receiver_caustic = b.receiver_caustic;
        m->receiver_upper = b.receiver_upper;
        m->receiver_lower = b.receiver_lower;
        m->source_index = (size_t)b.source;
        m->receiver_index = (size_t)b.receiver;
        return m;
    }

    ocean::ocean_model::csptr _ocean;
    std::shared_ptr<const eigenverbs::eigenverb_collection> _src, _rcv;
    types::seq_vector::csptr _freq;
    biverb_collection::csptr _collection;
    bool _abort = false, _done = false;
};

}  // namespace biverbs

namespace waveq3d {

/* reflection_listener (waveq3d/reflection_listener.h:46-49): one call per
 * boundary collision; type 0 is the bottom, 1 the surface */
class reflection_listener {
   public:
    virtual ~reflection_listener() {}
    virtual void reflect(double time, size_t de, size_t az, double dt, double grazing, double speed,
                         const types::wposition1& position, const types::wvector1& ndirection,
                         size_t type) = 0;
};

/* Host copy of one wavefront (waveq3d/wave_front.h:152-258), the data
 * the reference's wave_queue::curr()/next()/prev()/past() expose; arrays are
 * num_de x num_az row-major (de, az), attenuation and phase with the
 * frequency fastest. */
struct wave_front {
    size_t num_de = 0, num_az = 0, num_freq = 0;
    std::vector<double> rho, theta, phi, sound_speed, distance, path_length, attenuation, phase;
    std::vector<double> ndir[3], pos_grad[3], ndir_grad[3], sound_grad[3];
    std::vector<int32_t> surface, bottom, caustic, upper, lower;
    std::vector<uint8_t> on_edge;
    size_t index(size_t de, size_t az) const { return de * num_az + az; }
};

/* wave_queue (waveq3d/wave_queue.h:122-264) */
class wave_queue {
   public:
    enum spreading_type { CLASSIC_RAY = WQ3D_CLASSIC_RAY, HYBRID_GAUSSIAN = WQ3D_HYBRID_GAUSSIAN };

    wave_queue(const ocean::ocean_model::csptr& ocean, const types::seq_vector::csptr& freq,
               const types::wposition1& pos, const types::seq_vector::csptr& de,
               const types::seq_vector::csptr& az, double time_step, const types::wposition* targets = nullptr,
               spreading_type type = HYBRID_GAUSSIAN, int precision = WQ3D_FP32C)
        : _ocean(ocean), _freq(freq), _time_step(time_step), _num_de(de->size()), _num_az(az->size()) {
        wq3d_queue_desc d{};
        d.freq = freq->data().data();
        d.num_freq = freq->size();
        d.source[0] = pos.rho();
        d.source[1] = pos.theta();
        d.source[2] = pos.phi();
        d.de = de->data().data();
        d.de_inc = de->increments().data();
        d.num_de = de->size();
        d.az = az->data().data();
        d.az_inc = az->increments().data();
        d.num_az = az->size();
        d.time_step = time_step;
        std::vector<double> tg;
        if (targets) {
            tg = targets->packed();
            d.targets = tg.data();
            d.num_targets1 = targets->size1();
            d.num_targets2 = targets->size2();
        }
        d.spreading = type;
        d.precision = precision;
        d.earth_radius = types::earth::radius();
        wq3d_queue* q = nullptr;
        check(wq3d_queue_create(ocean->handle(), &d, &q));
        _q.reset(q, [](wq3d_queue* p) { wq3d_queue_destroy(p); });
    }

    void add_eigenray_listener(eigenrays::eigenray_listener* l) {
        _listeners.push_back(l);
        install();
    }
    void add_eigenverb_listener(eigenverbs::eigenverb_listener* l) {
        _verb_listeners.push_back(l);
        install();
    }
    void add_reflection_listener(reflection_listener* l) {
        _refl_listeners.push_back(l);
        install();
    }
    void remove_eigenray_listener(eigenrays::eigenray_listener* l) { drop(_listeners, l); }
    void remove_eigenverb_listener(eigenverbs::eigenverb_listener* l) { drop(_verb_listeners, l); }
    void remove_reflection_listener(reflection_listener* l) { drop(_refl_listeners, l); }
    void step() { check(wq3d_queue_step(_q.get(), 1)); }
    void run(double time_max) { check(wq3d_queue_run(_q.get(), time_max, nullptr)); }
    /** thread_task::abort: the run stops before its next chunk of steps */
    void abort() { check(wq3d_queue_abort(_q.get())); }
    /**
     * Runs several queues together on one GPU, each until its time()
     * reaches its time_max (wq3d_batch_run), where the reference runs one
     * wavefront_generator task per queue on a thread pool.  Listeners are
     * called per queue in the reference's order.  Returns the device
     * milliseconds of the batch.
     */
    static double run_batch(const std::vector<wave_queue*>& queues, const std::vector<double>& time_max) {
        if (queues.size() != time_max.size()) throw std::invalid_argument("one time_max per queue");
        std::vector<wq3d_queue*> handles;
        for (auto* q : queues) handles.push_back(q->_q.get());
        double ms = 0.0;
        check(wq3d_batch_run(handles.data(), handles.size(), time_max.data(), nullptr, &ms));
        return ms;
    }
    double time() const {
        double t = 0.0;
        check(wq3d_queue_time(_q.get(), &t));
        return t;
    }
    double time_step() const { return _time_step; }
    /** wave_queue::past()/prev()/curr()/next() (wave_queue.h:179-216), as
     * host copies of the fronts */
    wave_front past() const { return front(WQ3D_FRONT_PAST); }
    wave_front prev() const { return front(WQ3D_FRONT_PREV); }
    wave_front curr() const { return front(WQ3D_FRONT_CURR); }
    wave_front next() const { return front(WQ3D_FRONT_NEXT); }
    size_t num_de() const { return _num_de; }
    size_t num_az() const { return _num_az; }
    /** steps taken since the queue was made (AB3 and start-up alike) */
    int64_t steps() const {
        int64_t n = 0;
        check(wq3d_queue_steps(_q.get(), &n));
        return n;
    }
    types::wposition1 source_pos() const {
        double s[3];
        check(wq3d_queue_source(_q.get(), s));
        types::wposition1 p;
        p.rho(s[0]);
        p.theta(s[1]);
        p.phi(s[2]);
        return p;
    }
    void intensity_threshold(double v) {
        _th.intensity = std::abs(v);
        check(wq3d_queue_set_thresholds(_q.get(), &_th));
    }
    void eigenverb_threshold(double v) {
        _th.eigenverb = std::abs(v);
        check(wq3d_queue_set_thresholds(_q.get(), &_th));
    }
    void max_bottom(int v) {
        _th.max_bottom = v;
        check(wq3d_queue_set_thresholds(_q.get(), &_th));
    }
    void max_surface(int v) {
        _th.max_surface = v;
        check(wq3d_queue_set_thresholds(_q.get(), &_th));
    }
    void max_caustic(int v) {
        _th.max_caustic = v;
        check(wq3d_queue_set_thresholds(_q.get(), &_th));
    }
    void max_upper(int v) {
        _th.max_upper = v;
        check(wq3d_queue_set_thresholds(_q.get(), &_th));
    }
    void max_lower(int v) {
        _th.max_lower = v;
        check(wq3d_queue_set_thresholds(_q.get(), &_th));
    }

   private:
    wave_front front(int which) const {
        wave_front f;
        f.num_de = _num_de;
        f.num_az = _num_az;
        f.num_freq = _freq->size();
        const size_t n = _num_de * _num_az, nf = f.num_freq;
        for (auto* v : {&f.rho, &f.theta, &f.phi, &f.sound_speed, &f.distance, &f.path_length}) v->resize(n);
        for (int k = 0; k < 3; ++k)
            for (auto* v : {&f.ndir[k], &f.pos_grad[k], &f.ndir_grad[k], &f.sound_grad[k]}) v->resize(n);
        f.attenuation.resize(n * nf);
        f.phase.resize(n * nf);
        for (auto* v : {&f.surface, &f.bottom, &f.caustic, &f.upper, &f.lower}) v->resize(n);
        f.on_edge.resize(n);
        wq3d_front_view view{};
        view.rho = f.rho.data();
        view.theta = f.theta.data();
        view.phi = f.phi.data();
        for (int k = 0; k < 3; ++k) {
            view.ndir[k] = f.ndir[k].data();
            view.pos_grad[k] = f.pos_grad[k].data();
            view.ndir_grad[k] = f.ndir_grad[k].data();
            view.sound_grad[k] = f.sound_grad[k].data();
        }
        view.sound_speed = f.sound_speed.data();
        view.distance = f.distance.data();
        view.path_length = f.path_length.data();
        view.attenuation = f.attenuation.data();
        view.phase = f.phase.data();
        view.surface = f.surface.data();
        view.bottom = f.bottom.data();
        view.caustic = f.caustic.data();
        view.upper = f.upper.data();
        view.lower = f.lower.data();
        view.on_edge = f.on_edge.data();
        check(wq3d_queue_get_front(_q.get(), which, &view));
        return f;
    }
    template <class L>
    void drop(std::vector<L*>& v, L* l) {
        v.erase(std::remove(v.begin(), v.end(), l), v.end());
        install();
    }
    void install() {
        wq3d_callbacks cb{};
        if (!_listeners.empty()) {
            cb.add_eigenray = &wave_queue::on_ray;
            cb.check_eigenrays = &wave_queue::on_check;
        }
        if (!_verb_listeners.empty()) cb.add_eigenverb = &wave_queue::on_verb;
        if (!_refl_listeners.empty()) cb.reflect = &wave_queue::on_reflect;
        check(wq3d_queue_set_callbacks(_q.get(), &cb, this));
    }
    static void on_reflect(void* ctx, const wq3d_reflection* r) {
        auto* self = static_cast<wave_queue*>(ctx);
        types::wposition1 pos;
        pos.rho(r->position[0]);
        pos.theta(r->position[1]);
        pos.phi(r->position[2]);
        const types::wvector1 nd(r->ndirection[0], r->ndirection[1], r->ndirection[2]);
        for (auto* l : self->_refl_listeners)
            l->reflect(r->time, (size_t)r->de, (size_t)r->az, r->dt, r->grazing, r->speed, pos, nd,
                       (size_t)r->type);
    }
    static void on_verb(void* ctx, const wq3d_eigenverb* v, const double* power, size_t nf, int interface_num) {
        auto* self = static_cast<wave_queue*>(ctx);
        auto verb = std::make_shared<eigenverbs::eigenverb_model>();
        verb->travel_time = v->travel_time;
        verb->power.assign(power, power + nf);
        verb->length = v->length;
        verb->width = v->width;
        verb->position.rho(v->position[0]);
        verb->position.theta(v->position[1]);
        verb->position.phi(v->position[2]);
        verb->direction = v->direction;
        verb->grazing = v->grazing;
        verb->sound_speed = v->sound_speed;
        verb->de_index = (size_t)v->de;
        verb->az_index = (size_t)v->az;
        verb->source_de = v->source_de;
        verb->source_az = v->source_az;
        verb->surface = v->surface;
        verb->bottom = v->bottom;
        verb->caustic = v->caustic;
        verb->upper = v->upper;
        verb->lower = v->lower;
        for (auto* l : self->_verb_listeners) l->add_eigenverb(verb, (size_t)interface_num);
    }
    static void on_ray(void* ctx, size_t t1, size_t t2, const wq3d_eigenray* r, const double* inten,
                       const double* phase, size_t nf, uint64_t run) {
        auto* self = static_cast<wave_queue*>(ctx);
        auto ray = std::make_shared<eigenrays::eigenray_model>();
        ray->travel_time = r->time;
        ray->source_de = r->source_de;
        ray->source_az = r->source_az;
        ray->target_de = r->target_de;
        ray->target_az = r->target_az;
        ray->surface = r->surface;
        ray->bottom = r->bottom;
        ray->caustic = r->caustic;
        ray->upper = r->upper;
        ray->lower = r->lower;
        ray->intensity.assign(inten, inten + nf);
        ray->phase.assign(phase, phase + nf);
        for (auto* l : self->_listeners) l->add_eigenray(t1, t2, ray, run);
    }
    static void on_check(void* ctx, double time, uint64_t run) {
        for (auto* l : static_cast<wave_queue*>(ctx)->_listeners) l->check_eigenrays(time, run);
    }

    ocean::ocean_model::csptr _ocean;
    types::seq_vector::csptr _freq;
    std::shared_ptr<wq3d_queue> _q;
    std::vector<eigenrays::eigenray_listener*> _listeners;
    std::vector<eigenverbs::eigenverb_listener*> _verb_listeners;
    std::vector<reflection_listener*> _refl_listeners;
    double _time_step;
    size_t _num_de, _num_az;
    wq3d_thresholds _th{300.0, 300.0, 999, 999, 999, 999, 999};
};

}  // namespace waveq3d
}  // namespace usml_b200

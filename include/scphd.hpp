// scphd.hpp — header-only C++ host class over the C ABI (scphd.h), mirroring the
// reference class SCPHDCameraCalibration (src/scphdcameracalibration.cuh:29-44) so
// that a driver written against the reference (src/main.cpp:53-99) compiles with
// only its include line and constructor argument changed.
//
//   reference                                   here
//   SCPHDCameraCalibration(const char* cfg)     same (a libconfig file, scphd_config_from_file), or
//                                               SCPHDCameraCalibration(const scphd_config&)
//   void predict(double dt)                     same
//   void update(vector<double> u,               same, plus an overload with a disparity
//               vector<double> v, bool fixed)   vector for (u,v,d) measurements
//   void resample()                             same
//   void checkStuff()                           same: prints "nan weight detected" and
//                                               exits with status 2 (src/.cu:812-821)
//   void writeMat(const char*)                  same (MAT level 5, scphd_write_mat), and the
//                                               particles()/weights()/mixture() accessors
//
// Errors of the C ABI raise scphd::Error (the reference had no error reporting on
// this path besides exit(2)).
#ifndef SCPHD_HPP
#define SCPHD_HPP

#include "scphd.h"
#include "scphd_io.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

namespace scphd {

class Error : public std::runtime_error {
public:
    Error(scphd_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    scphd_status status;
};

inline void check_status(scphd_status s) {
    if (s != SCPHD_OK) throw Error(s, std::string("scphd: ") + scphd_last_error());
}

}  // namespace scphd

class SCPHDCameraCalibration {
public:
    explicit SCPHDCameraCalibration(const scphd_config& cfg) : cfg_(cfg) {
        scphd::check_status(scphd_create(&cfg_, &f_));
    }
    // from a configuration file in the reference's libconfig syntax (library defaults
    // for every key the file does not set)
    explicit SCPHDCameraCalibration(const char* config_file) {
        scphd_config_defaults(&cfg_);
        scphd_run_options opts = {1 << 30, 0, 0, 0};
        scphd::check_status(scphd_config_from_file(config_file, &cfg_, &opts));
        scphd::check_status(scphd_create(&cfg_, &f_));
    }
    ~SCPHDCameraCalibration() {
        if (f_) scphd_destroy(f_);
    }
    SCPHDCameraCalibration(const SCPHDCameraCalibration&) = delete;
    SCPHDCameraCalibration& operator=(const SCPHDCameraCalibration&) = delete;

    void predict(double dt) { scphd::check_status(scphd_predict(f_, dt)); }

    void update(std::vector<double> u, std::vector<double> v, bool fixed_camera) {
        if (u.size() != v.size()) throw scphd::Error(SCPHD_ERR_INVALID, "scphd: u and v differ in length");
        scphd::check_status(scphd_update(f_, u.data(), v.data(), nullptr, (int32_t)u.size(), fixed_camera));
    }

    void update(std::vector<double> u, std::vector<double> v, std::vector<double> d, bool fixed_camera) {
        if (u.size() != v.size() || u.size() != d.size())
            throw scphd::Error(SCPHD_ERR_INVALID, "scphd: u, v, d differ in length");
        scphd::check_status(scphd_update(f_, u.data(), v.data(), d.data(), (int32_t)u.size(), fixed_camera));
    }

    // returns whether resampling happened (the reference returns void)
    bool resample() {
        int32_t r = 0;
        scphd::check_status(scphd_resample(f_, &r));
        return r != 0;
    }

    void writeMat(const char* path, bool save_all_maps = false) {
        scphd::check_status(scphd_write_mat(f_, path, save_all_maps ? 1 : 0));
    }

    void checkStuff() {
        scphd_status s = scphd_check(f_);
        if (s == SCPHD_ERR_NAN) {
            std::printf("nan weight detected\n");
            std::exit(2);
        }
        scphd::check_status(s);
    }

    // writeMat content: parent states (n x 12) and linear weights
    std::vector<double> particles() const {
        std::vector<double> st((size_t)cfg_.n_parents * 12);
        scphd::check_status(scphd_get_particles(f_, st.data(), nullptr));
        return st;
    }
    std::vector<double> weights() const {
        std::vector<double> lw(cfg_.n_parents);
        scphd::check_status(scphd_get_particles(f_, nullptr, lw.data()));
        for (double& w : lw) w = std::exp(w);
        return lw;
    }
    std::vector<int32_t> mapSizes() const {
        std::vector<int32_t> n(cfg_.n_parents);
        scphd::check_status(scphd_get_map_sizes(f_, n.data()));
        return n;
    }
    // merged (which = SCPHD_MIX_MERGED) or refitted (SCPHD_MIX_FITTED) mixture of parent p
    std::vector<double> mixture(int which, int p) const {
        int32_t n = 0;
        scphd::check_status(scphd_get_mixture(f_, which, p, nullptr, &n));
        std::vector<double> out((size_t)n * (which == SCPHD_MIX_FITTED ? 29 : 28));
        if (n) scphd::check_status(scphd_get_mixture(f_, which, p, out.data(), &n));
        return out;
    }

    const scphd_config& config() const { return cfg_; }
    scphd_filter* handle() const { return f_; }

private:
    scphd_config cfg_;
    scphd_filter* f_ = nullptr;
};

#endif  // SCPHD_HPP

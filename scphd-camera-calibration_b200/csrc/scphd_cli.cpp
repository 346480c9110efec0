// scphd_calibrate — command-line driver of the filter, the counterpart of the
// reference's src/main.cpp:53-99: read the measurement cells Z1 (fixed camera) and
// Z2 (camera being calibrated) from a MAT file, build the filter from a configuration
// file, write prior.mat, then for k < min(frames, max_steps): predict(0.5); update
// with Z1[k] on even k (fixed camera) and Z2[k] on odd k, or Z2[k] always in slam mode;
// write k.mat; check for NaN weights (exit 2, as checkStuff); resample.
//
//   scphd_calibrate CONFIG DATA [--out DIR] [--device N] [--fp32] [--dry-run] [--quiet]
//
// Frames with three rows (u; v; d) run the (u, v, d) update when the configuration sets
// meas_dim = 3; otherwise the first two rows are used, as the reference does.
// max_measurements defaults to the largest frame of the data.  --dry-run reads and
// checks everything, prints a JSON summary, and touches no GPU.
#include "scphd.h"
#include "scphd_io.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct Frames {
    int rows = 2;
    std::vector<int32_t> sizes;
    std::vector<int64_t> offs;
    std::vector<double> data;
    const double* row(int k, int q) const { return data.data() + offs[k] + (int64_t)q * sizes[k]; }
};

bool read_frames(const char* path, const char* var, Frames& fr) {
    int32_t n = 0, rows = 0;
    if (scphd_read_mat_frames(path, var, &n, &rows, nullptr, nullptr, 0) != SCPHD_OK) {
        fprintf(stderr, "scphd_calibrate: %s\n", scphd_last_error());
        return false;
    }
    fr.rows = rows;
    fr.sizes.assign(n, 0);
    // the data size is not known before the second call: grow until it fits
    int64_t cap = 1 << 16;
    while (true) {
        fr.data.assign(cap, 0.0);
        scphd_status s = scphd_read_mat_frames(path, var, &n, &rows, fr.sizes.data(), fr.data.data(), cap);
        if (s == SCPHD_OK) break;
        if (s != SCPHD_ERR_CAPACITY) {
            fprintf(stderr, "scphd_calibrate: %s\n", scphd_last_error());
            return false;
        }
        cap *= 4;
    }
    fr.offs.assign(n, 0);
    int64_t at = 0;
    for (int k = 0; k < n; ++k) {
        fr.offs[k] = at;
        at += (int64_t)rows * fr.sizes[k];
    }
    return true;
}

int usage() {
    fprintf(stderr, "Usage: scphd_calibrate CONFIG DATA [--out DIR] [--device N] [--fp32] [--dry-run] [--quiet]\n");
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) return usage();
    const char* cfg_path = argv[1];
    const char* data_path = argv[2];
    std::string out = ".";
    int device = -1;
    bool dry = false, quiet = false, fp32 = false;
    for (int i = 3; i < argc; ++i) {
        if (!strcmp(argv[i], "--out") && i + 1 < argc) out = argv[++i];
        else if (!strcmp(argv[i], "--device") && i + 1 < argc) device = atoi(argv[++i]);
        else if (!strcmp(argv[i], "--dry-run")) dry = true;
        else if (!strcmp(argv[i], "--quiet")) quiet = true;
        else if (!strcmp(argv[i], "--fp32")) fp32 = true;
        else return usage();
    }
    Frames z1, z2;
    if (!read_frames(data_path, "Z1", z1) || !read_frames(data_path, "Z2", z2)) return 1;
    const int n_steps = (int)std::min(z1.sizes.size(), z2.sizes.size());
    scphd_config cfg;
    scphd_config_defaults(&cfg);
    cfg.max_measurements = 0;   // from the data unless the file sets it
    scphd_run_options opts = {1 << 30, 0, 0, 0};
    if (scphd_config_from_file(cfg_path, &cfg, &opts) != SCPHD_OK) {
        fprintf(stderr, "scphd_calibrate: %s\n", scphd_last_error());
        return 1;
    }
    if (device >= 0) cfg.device = device;
    if (fp32) cfg.precision = SCPHD_FP32;
    int mmax = 1;
    for (int k = 0; k < n_steps; ++k) mmax = std::max({mmax, (int)z1.sizes[k], (int)z2.sizes[k]});
    if (cfg.max_measurements <= 0) cfg.max_measurements = (mmax + 31) / 32 * 32;
    if (cfg.meas_dim == 3 && (z1.rows < 3 || z2.rows < 3)) {
        fprintf(stderr, "scphd_calibrate: meas_dim = 3 needs (u; v; d) frames\n");
        return 1;
    }
    const int kmax = std::min(n_steps, opts.max_steps);
    int64_t bytes = 0;
    if (scphd_device_bytes(&cfg, &bytes) != SCPHD_OK) {
        fprintf(stderr, "scphd_calibrate: %s\n", scphd_last_error());
        return 1;
    }
    if (dry) {
        long long nz1 = 0, nz2 = 0;
        double s1 = 0, s2 = 0;
        for (int k = 0; k < n_steps; ++k) {
            nz1 += z1.sizes[k];
            nz2 += z2.sizes[k];
            for (int q = 0; q < z1.rows; ++q)
                for (int i = 0; i < z1.sizes[k]; ++i) s1 += z1.row(k, q)[i];
            for (int q = 0; q < z2.rows; ++q)
                for (int i = 0; i < z2.sizes[k]; ++i) s2 += z2.row(k, q)[i];
        }
        printf("{\"frames\": %d, \"rows\": %d, \"steps\": %d, \"z1_measurements\": %lld, \"z2_measurements\": %lld, "
               "\"z1_sum\": %.17g, \"z2_sum\": %.17g, \"n_parents\": %d, \"particles_per_feature\": %d, "
               "\"max_measurements\": %d, \"meas_dim\": %d, \"precision\": %d, \"kappa\": %.17g, "
               "\"min_weight\": %.17g, \"slam\": %d, \"save_all_maps\": %d, \"device_bytes\": %lld}\n",
               n_steps, z1.rows, kmax, nz1, nz2, s1, s2, cfg.n_parents, cfg.particles_per_feature,
               cfg.max_measurements, cfg.meas_dim, cfg.precision, cfg.kappa, cfg.min_weight, opts.slam,
               opts.save_all_maps, (long long)bytes);
        return 0;
    }
    scphd_filter* f = nullptr;
    if (scphd_create(&cfg, &f) != SCPHD_OK) {
        fprintf(stderr, "scphd_calibrate: %s\n", scphd_last_error());
        return 1;
    }
    auto check = [&](scphd_status s) {
        if (s == SCPHD_OK) return;
        fprintf(stderr, "scphd_calibrate: %s\n", scphd_last_error());
        scphd_destroy(f);
        exit(s == SCPHD_ERR_NAN ? 2 : 1);
    };
    check(scphd_write_mat(f, (out + "/prior.mat").c_str(), opts.save_all_maps));
    for (int k = 0; k < kmax; ++k) {
        if (!quiet) printf("k = %d\n", k);
        check(scphd_predict(f, 0.5));
        const bool fixed = !opts.slam && (k % 2) == 0;
        const Frames& z = fixed ? z1 : z2;
        const double* d = cfg.meas_dim == 3 ? z.row(k, 2) : nullptr;
        check(scphd_update(f, z.row(k, 0), z.row(k, 1), d, z.sizes[k], fixed ? 1 : 0));
        check(scphd_write_mat(f, (out + "/" + std::to_string(k) + ".mat").c_str(), opts.save_all_maps));
        const scphd_status cs = scphd_check(f);
        if (cs == SCPHD_ERR_NAN) {
            printf("nan weight detected\n");
            scphd_destroy(f);
            return 2;
        }
        check(cs);
        int32_t resampled = 0;
        check(scphd_resample(f, &resampled));
    }
    scphd_destroy(f);
    return 0;
}

// Reference-shaped driver (the loop of src/main.cpp:78-97) over the C++ host class
// include/scphd.hpp.  Reads frames from a flat binary file written by the test:
//   int32 n_frames; per frame: int32 n, int32 fixed, n doubles u, n doubles v
// Config fields are passed on the command line as key=value (n_parents, ppf, seed).
// Writes n_parents x 12 states then n_parents weights (doubles) to the output file.
#include "scphd.hpp"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

int main(int argc, char** argv) {
    if (argc < 3) {
        std::printf("usage: host_driver frames.bin out.bin [key=value ...]\n");
        return 1;
    }
    scphd_config cfg;
    scphd_config_defaults(&cfg);
    for (int i = 3; i < argc; ++i) {
        const char* kv = argv[i];
        if (!std::strncmp(kv, "n_parents=", 10)) cfg.n_parents = std::atoi(kv + 10);
        if (!std::strncmp(kv, "ppf=", 4)) cfg.particles_per_feature = std::atoi(kv + 4);
        if (!std::strncmp(kv, "seed=", 5)) cfg.seed = std::strtoull(kv + 5, nullptr, 10);
        if (!std::strncmp(kv, "max_meas=", 9)) cfg.max_measurements = std::atoi(kv + 9);
    }
    FILE* fp = std::fopen(argv[1], "rb");
    if (!fp) return 1;
    int32_t nf = 0;
    if (std::fread(&nf, 4, 1, fp) != 1) return 1;
    try {
        SCPHDCameraCalibration calibration(cfg);
        for (int k = 0; k < nf; ++k) {
            int32_t n = 0, fixed = 0;
            if (std::fread(&n, 4, 1, fp) != 1 || std::fread(&fixed, 4, 1, fp) != 1) return 1;
            std::vector<double> u(n), v(n);
            if (std::fread(u.data(), 8, n, fp) != (size_t)n || std::fread(v.data(), 8, n, fp) != (size_t)n) return 1;
            calibration.predict(0.5);
            calibration.update(u, v, fixed != 0);
            calibration.checkStuff();
            calibration.resample();
        }
        std::vector<double> st = calibration.particles(), w = calibration.weights();
        FILE* fo = std::fopen(argv[2], "wb");
        std::fwrite(st.data(), 8, st.size(), fo);
        std::fwrite(w.data(), 8, w.size(), fo);
        std::fclose(fo);
    } catch (const scphd::Error& e) {
        std::printf("%s\n", e.what());
        return 3;
    }
    std::fclose(fp);
    return 0;
}

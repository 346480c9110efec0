// scphd_oracle.cpp — TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// A plain C++ FP64 restatement of one SC-PHD filter step of the reference
// (cheesinglee/scphd-camera-calibration), used only by tests/, by
// __graft_entry__.smoke() and by the CPU-baseline legs of bench.py, as the
// checker.  The product (the CUDA library) never links or calls it.
//
// What is restated, with the reference file:line each part follows:
//   predict            src/scphdcameracalibration.cu:1034-1151, functors :129-178,
//                      src/OrientedLinearCVMotionModel3D.cuh:40-54,
//                      src/linearcvmotionmodel3d.cuh:28-40, wrapAngle src/device_math.cu:308-318
//   world<->disparity  src/disparitymeasurementmodel.cu:3-217, in-FOV pD src/kernels.cu:37-45
//   fit                normalizeWeightsKernel src/kernels.cu:996-1018,
//                      fitGaussiansKernel src/kernels.cu:102-438, computePdKernel :82-99
//   births             src/scphdcameracalibration.cu:2589-2638
//   non-detections     src/scphdcameracalibration.cu:1290-1420 (+ recombine :1422-1574)
//   detections         computeDetectionsKernel src/kernels.cu:470-603 (H = [I_k 0])
//   normalisers        src/scphdcameracalibration.cu:1729-1768, log_sum_exp functor :506-517
//   update/prune flags updateKernel src/kernels.cu:608-659
//   parent weights     src/scphdcameracalibration.cu:1813-1876 (log domain or as written)
//   merge              phdUpdateMergeKernel src/kernels.cu:662-874, computeMahalDist
//                      src/device_math.cu:374-454, cholesky :123-150, isPosDef :800-812
//   resample sampling  sample_disparity_gaussian src/scphdcameracalibration.cu:640-690
//   resample           src/scphdcameracalibration.cu:2641-2817
//
// Deliberate differences from the reference, all shared with the device code:
//   * random numbers come from Philox4x32-7 streams keyed by
//     (seed, frame, stage, parent, gaussian, sample) with Box-Muller normals,
//     instead of time()-seeded minstd engines (src/scphdcameracalibration.cu:1047-1118);
//   * reductions are sequential left-to-right in FP64;
//   * maps are keyed per parent explicitly, so the reduce_by_key defects on empty
//     maps and M == 1 (:1750-1756, :2562-2585) do not arise;
//   * meas_dim 3 generalises H = [I_2 0] to [I_3 0] and births take the measured d;
//   * a stereo baseline multiplies d and vd (baseline 1 is the reference);
//   * a parent's map is capped at max_gaussians entries, keeping the largest
//     weights (the reference's maps are unbounded);
//   * the merge's argmax compares weights rounded to single precision (equal keys
//     are ties, ordered by the reference's index rule), as does the capacity cut.
#include "scphd.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double kLog0 = -FLT_MAX;   // LOG0, src/device_math.cu:8
const double kPi = M_PI;

// ---------------------------------------------------------------- random streams
enum Stage { ST_PRIOR = 1, ST_CAM = 2, ST_FEAT = 3, ST_SAMPLE = 4, ST_RESAMPLE = 5 };

// Philox4x32 (Salmon, Moraes, Dror and Shaw, SC'11) with R rounds.  The streams use
// kPhiloxRounds = 7 rounds, the fewest the authors report passing TestU01's BigCrush;
// R = 10 is the Random123 default whose known-answer vectors pin the round function.
const int kPhiloxRounds = 7;

void philox4x32(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4], int rounds) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < rounds; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

inline uint32_t ctr_word3(int frame, int stage, int block) {
    return ((uint32_t)frame << 12) | ((uint32_t)stage << 8) | (uint32_t)block;
}

inline double u01_of(uint32_t w) { return ((double)w + 0.5) * 0x1p-32; }

struct Stream {
    uint64_t seed;
    void words(uint32_t s, uint32_t j, uint32_t p, uint32_t c3, uint32_t w[4]) const {
        const uint32_t ctr[4] = {s, j, p, c3};
        const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
        philox4x32(ctr, key, w, kPhiloxRounds);
    }
    // four standard normals from one Philox block (two Box-Muller pairs)
    void normals4(uint32_t s, uint32_t j, uint32_t p, uint32_t c3, double z[4]) const {
        uint32_t w[4];
        words(s, j, p, c3, w);
        for (int h = 0; h < 2; ++h) {
            double r = std::sqrt(-2.0 * std::log(u01_of(w[2 * h])));
            double th = (2.0 * kPi) * u01_of(w[2 * h + 1]);
            z[2 * h] = r * std::cos(th);
            z[2 * h + 1] = r * std::sin(th);
        }
    }
};

// ---------------------------------------------------------------- small math
double safe_log(double x) { return x <= 0 ? kLog0 : std::log(x); }   // device_math.cu:22-29

double wrap_angle(double a) {                                         // device_math.cu:308-318
    double r = std::fmod(a, double(2 * kPi));
    if (r > kPi) r -= 2 * kPi;
    else if (r < -kPi) r += 2 * kPi;
    return r;
}

// lower Cholesky of a column-major n x n matrix, as src/device_math.cu:123-150
void cholesky(const double* A, double* L, int n) {
    for (int i = 0; i < n * n; ++i) L[i] = 0.0;
    L[0] = std::sqrt(A[0]);
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j <= i; ++j) {
            double tmp = A[i + j * n];
            if (i == j) {
                for (int k = 0; k < j; ++k) tmp -= L[j + k * n] * L[j + k * n];
                L[i + j * n] = std::sqrt(tmp);
            } else {
                for (int k = 0; k < j; ++k) tmp -= L[i + k * n] * L[j + k * n];
                L[i + j * n] = tmp / L[j + j * n];
            }
        }
    }
}

bool is_pos_def6(const double* cov) {                                 // device_math.cu:800-812
    double L[36];
    cholesky(cov, L, 6);
    for (int i = 0; i < 36; ++i)
        if (std::isnan(L[i])) return false;
    return true;
}

// PD test of an update's posterior covariance.  The reference's isPosDef (a Cholesky
// without NaN) is decided by the sign of a rounding error when the posterior is exactly
// singular, as it is after refitting a cloud with fewer in-view samples than dimensions;
// here (and on the device) such a matrix is classed not PD: every pivot must exceed
// 1e-10 of its diagonal entry.  Elsewhere the two tests agree.
bool is_pos_def6_strict(const double* cov) {
    double L[36];
    for (int i = 0; i < 36; ++i) L[i] = 0.0;
    for (int i = 0; i < 6; ++i) {
        for (int j = 0; j <= i; ++j) {
            double tmp = cov[i + j * 6];
            if (i == j) {
                for (int k = 0; k < j; ++k) tmp -= L[j + k * 6] * L[j + k * 6];
                if (!(tmp > 1e-10 * cov[i + i * 6])) return false;
                L[i + j * 6] = std::sqrt(tmp);
            } else {
                for (int k = 0; k < j; ++k) tmp -= L[i + k * 6] * L[j + k * 6];
                L[i + j * 6] = tmp / L[j + j * 6];
            }
        }
    }
    for (int i = 0; i < 36; ++i)
        if (std::isnan(L[i])) return false;
    return true;
}

void triangular_inverse(const double* L, double* Li, int n) {         // device_math.cu:153-175
    for (int col = 0; col < n; ++col)
        for (int i = 0; i < n; ++i) {
            if (i >= col) {
                double val = (i == col) ? 1.0 : 0.0;
                for (int j = 0; j < i; ++j) val -= L[i + j * n] * Li[j + col * n];
                Li[i + col * n] = val / L[i + i * n];
            } else {
                Li[i + col * n] = 0.0;
            }
        }
}

// ---------------------------------------------------------------- types
struct Ext { double c[6]; double a[6]; };   // Extrinsics, src/types.h:137-140
struct G6 { double w; double mean[6]; double cov[36]; };   // Gaussian6D, src/types.h:19-53

struct Cloud {           // one daughter Gaussian carried as a weighted sample cloud
    double W = 0;        // dev_feature_weights_
    std::vector<double> x;    // 6 x P, coordinate-major (x,y,z,vx,vy,vz)
    std::vector<double> om;   // P sample weights (dev_particle_weights_)
};

double mahal6(const G6& a, const G6& b) {                             // device_math.cu:374-454
    double innov[6], sigma[36], L[36], Li[36];
    for (int i = 0; i < 6; ++i) innov[i] = a.mean[i] - b.mean[i];
    for (int i = 0; i < 36; ++i) sigma[i] = a.cov[i] + b.cov[i];
    cholesky(sigma, L, 6);
    triangular_inverse(L, Li, 6);
    double dist = 0;
    for (int i = 0; i < 6; ++i) {
        double sum = 0;
        for (int j = 0; j <= i; ++j) sum += innov[j] * Li[i + j * 6];
        dist += sum * sum;
    }
    return dist;
}

void force_symmetric(G6& g) {                                         // device_math.cu:722-737
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < i; ++j) {
            int lo = i + j * 6, up = j + i * 6;
            g.cov[lo] = (g.cov[lo] + g.cov[up]) / 2;
            g.cov[up] = g.cov[lo];
        }
}

// Order in which phdUpdateMergeKernel's argmax (src/kernels.cu:704-739) resolves equal
// weights: within a thread the earliest of its strided indices wins (strict '<'),
// across the 256-thread tree the lower slot wins at every level, which prefers
// thread ids by their bit-reversed value.  r is the index relative to the map's
// update offset.
uint32_t tie_key(uint32_t r) {
    uint32_t t = r & 255u, rev = 0;
    for (int b = 0; b < 8; ++b) rev |= ((t >> b) & 1u) << (7 - b);
    return (rev << 24) | (r >> 8);
}

// Order key of a weight in the greedy merge's argmax and in the map-capacity cut: the
// weight rounded to single precision.  Exact ties are common (every birth of an
// unexplained measurement has weight w0 / (M w0 + kappa)) and so are FP64 weights that
// differ only in their last bits (a Gaussian term 1e-15 of a normaliser); any two
// implementations of the FP64 sums order such near-ties differently, so equal
// single-precision keys count as ties and the index rules order them.
inline float order_key(double w) { return (float)w; }

// greedy merge of src/kernels.cu:662-874 on one map
void merge_map(const std::vector<G6>& comps, std::vector<uint8_t>& flags, double min_sep,
               std::vector<G6>& out, std::vector<int>* member_of) {
    const int n = (int)comps.size();
    if (member_of) member_of->assign(n, -1);
    std::vector<int> members;
    while (true) {
        int best = -1;
        for (int i = 0; i < n; ++i) {
            if (flags[i]) continue;
            const float kb = best < 0 ? 0.f : order_key(comps[best].w), ki = order_key(comps[i].w);
            if (best < 0 || kb < ki || (kb == ki && tie_key(i) < tie_key(best))) best = i;
        }
        if (best < 0) break;
        const G6 maxF = comps[best];
        double W = 0, mean[6] = {0, 0, 0, 0, 0, 0};
        members.clear();
        for (int i = 0; i < n; ++i) {
            if (flags[i]) continue;
            double dist = mahal6(maxF, comps[i]);
            if (dist < min_sep) {
                W += comps[i].w;
                for (int k = 0; k < 6; ++k) mean[k] += comps[i].w * comps[i].mean[k];
                members.push_back(i);
            }
        }
        if (W == 0) break;
        G6 m;
        m.w = W;
        for (int k = 0; k < 6; ++k) m.mean[k] = mean[k] / W;
        double cov[36] = {0};
        for (int i : members) {
            double dlt[6];
            for (int k = 0; k < 6; ++k) dlt[k] = m.mean[k] - comps[i].mean[k];
            for (int a = 0; a < 6; ++a)
                for (int b = 0; b < 6; ++b)
                    cov[a * 6 + b] += comps[i].w * (comps[i].cov[a * 6 + b] + dlt[a] * dlt[b]);
            flags[i] = 1;
        }
        for (int k = 0; k < 36; ++k) m.cov[k] = cov[k] / W;
        force_symmetric(m);
        out.push_back(is_pos_def6(m.cov) ? m : maxF);
        if (member_of)
            for (int i : members) (*member_of)[i] = (int)out.size() - 1;
    }
}

// Entries kept when a map of weights w is cut to cap entries: the cap largest order
// keys (weights rounded to single precision), equal keys in entry order (a stable
// sort by decreasing key).
void cap_keep(const std::vector<double>& w, int cap, std::vector<char>& keep) {
    std::vector<int> order(w.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return order_key(w[a]) > order_key(w[b]); });
    keep.assign(w.size(), 0);
    for (int i = 0; i < cap && i < (int)w.size(); ++i) keep[order[i]] = 1;
}

// systematic resampling as written, src/scphdcameracalibration.cu:2660-2702
void systematic(const std::vector<double>& w, double r0, std::vector<int>& idx) {
    const int n = (int)w.size();
    idx.assign(n, 0);
    double interval = 1.0 / n;
    double r = r0;
    double c = w[0];
    int i = 0;
    for (int j = 0; j < n; ++j) {
        while (r > c) {
            i++;
            if (i >= n || i < 0) {
                double max_weight = -1;
                int max_idx = -1;
                for (int k = 0; k < n; ++k)
                    if (w[k] > max_weight) { max_weight = w[k]; max_idx = k; }
                i = max_idx;
                c = 2;
                break;
            }
            c += w[i];
        }
        idx[j] = i;
        r += interval;
    }
}

// ---------------------------------------------------------------- the filter
struct Oracle {
    scphd_config cfg;
    Stream rng;
    int N, P, K;
    int frame = 0;
    int weight_mode = 0;   // 0 log domain, 1 linear as written
    long long truncations = 0;   // maps cut at max_gaussians since create
    long long unit_weight_fits = 0;   // in-view clouds whose weights were all 0 (fitted with weights 1)
    std::vector<Ext> ext;
    std::vector<double> lw;          // log weights (mode 0) or linear weights (mode 1)
    std::vector<std::vector<Cloud>> maps;
    // inspection of the last update / resample
    int last_M = 0;
    std::vector<std::vector<G6>> fitted;
    std::vector<std::vector<double>> pbar;
    std::vector<std::vector<G6>> merged;
    std::vector<double> ell, loglik;
    std::vector<int> resample_idx;
    std::vector<int> survivors;
    std::vector<std::vector<double>> precut;   // entry weights of each new map before the cap

    explicit Oracle(const scphd_config& c) : cfg(c) {
        rng.seed = c.seed;
        N = c.n_parents; P = c.particles_per_feature; K = c.meas_dim;
        ext.resize(N);
        lw.assign(N, -std::log((double)N));
        maps.assign(N, {});
        // uniform prior, src/scphdcameracalibration.cu:910-979 (injected stream)
        for (int p = 0; p < N; ++p) {
            double u[12];
            for (int b = 0; b < 3; ++b) {
                uint32_t w[4];
                rng.words(0, 0, (uint32_t)p, ctr_word3(0, ST_PRIOR, b), w);
                for (int q = 0; q < 4; ++q) u[4 * b + q] = u01_of(w[q]);
            }
            for (int q = 0; q < 6; ++q) {
                ext[p].c[q] = u[q] * (c.prior_b[q] - c.prior_a[q]) + c.prior_a[q];
                ext[p].a[q] = u[6 + q] * (c.prior_b[6 + q] - c.prior_a[6 + q]) + c.prior_a[6 + q];
            }
        }
    }

    double linear_weight(int p) const { return weight_mode ? lw[p] : std::exp(lw[p]); }

    // ------------------------------------------------ disparity measurement model
    void world_to_camera(const double* X, const Ext& e, double* pc) const {   // .cu:3-80
        double x = e.c[0], y = e.c[1], z = e.c[2];
        double ct = std::cos(e.a[0]), st = std::sin(e.a[0]);
        double cf = std::cos(e.a[1]), sf = std::sin(e.a[1]);
        double cp = std::cos(e.a[2]), sp = std::sin(e.a[2]);
        pc[0] = cf * cp * X[0] + (ct * sp + st * sf * cp) * X[1] + (st * sp - ct * sf * cp) * X[2]
              - cf * cp * x - (ct * sp + st * sf * cp) * y - (st * sp - ct * sf * cp) * z;
        pc[1] = -cf * sp * X[0] + (ct * cp - st * sf * sp) * X[1] + (st * cp + ct * sf * sp) * X[2]
              - (-cf * sp) * x - (ct * cp - st * sf * sp) * y - (st * cp + ct * sf * sp) * z;
        pc[2] = sf * X[0] - st * cf * X[1] + ct * cf * X[2] - sf * x - (-st * cf) * y - (ct * cf) * z;
        pc[3] = cf * cp * X[3] + (ct * sp + st * sf * cp) * X[4] + (st * sp - ct * sf * cp) * X[5];
        pc[4] = -cf * sp * X[3] + (ct * cp - st * sf * sp) * X[4] + (st * cp + ct * sf * sp) * X[5];
        pc[5] = sf * X[3] - st * cf * X[4] + ct * cf * X[5];
    }
    void camera_to_world(const double* C, const Ext& e, double* pw) const {   // .cu:82-144
        double x = e.c[0], y = e.c[1], z = e.c[2];
        double ct = std::cos(e.a[0]), st = std::sin(e.a[0]);
        double cf = std::cos(e.a[1]), sf = std::sin(e.a[1]);
        double cp = std::cos(e.a[2]), sp = std::sin(e.a[2]);
        pw[0] = cf * cp * C[0] - cf * sp * C[1] + sf * C[2] + x;
        pw[1] = (ct * sp + st * sf * cp) * C[0] + (ct * cp - st * sf * sp) * C[1] - st * cf * C[2] + y;
        pw[2] = (st * sp - ct * sf * cp) * C[0] + (st * cp + ct * sf * sp) * C[1] + ct * cf * C[2] + z;
        pw[3] = cf * cp * C[3] - cf * sp * C[4] + sf * C[5];
        pw[4] = (ct * sp + st * sf * cp) * C[3] + (ct * cp - st * sf * sp) * C[4] - st * cf * C[5];
        pw[5] = (st * sp - ct * sf * cp) * C[3] + (st * cp + ct * sf * sp) * C[4] + ct * cf * C[5];
    }
    void measure(const double* X, const Ext& e, double* y) const {            // .cu:165-196
        double c[6];
        world_to_camera(X, e, c);
        const double fx = cfg.fx, fy = cfg.fy, B = cfg.baseline;
        double x = c[0], yy = c[1], z = c[2], vx = c[3], vy = c[4], vz = c[5];
        y[0] = cfg.u0 - fx / z * x;
        y[1] = cfg.v0 - fy / z * yy;
        y[2] = -fx * B / z;
        y[3] = -fx * (vx * z - vz * x) / (z * z);
        y[4] = -fy * (vy * z - vz * yy) / (z * z);
        y[5] = fx * B * vz / (z * z);
    }
    void invert(const double* y, const Ext& e, double* X) const {              // .cu:198-217
        const double fx = cfg.fx, fy = cfg.fy, B = cfg.baseline;
        double u = y[0], v = y[1], d = y[2], vu = y[3], vv = y[4], vd = y[5];
        double c[6];
        c[0] = (u - cfg.u0) * B / d;
        c[1] = (fx / fy) * (v - cfg.v0) * B / d;
        c[2] = -fx * B / d;
        c[3] = B * (vu * d - vd * (u - cfg.u0)) / (d * d);
        c[4] = (fx / fy) * (vv * d - vd * (v - cfg.v0)) * B / (d * d);
        c[5] = fx * B * vd / (d * d);
        camera_to_world(c, e, X);
    }
    bool in_range(const double* y) const {                                    // kernels.cu:37-41
        return y[0] >= 0 && y[0] <= 2 * cfg.u0 && y[1] >= 0 && y[1] <= 2 * cfg.v0 && y[2] >= 0;
    }

    // ------------------------------------------------ predict
    void predict(double dt) {
        frame++;
        const int f = frame;
#pragma omp parallel for schedule(dynamic, 16)
        for (int p = 0; p < N; ++p) {
            double z[8];
            rng.normals4(0, 0, (uint32_t)p, ctr_word3(f, ST_CAM, 0), z);
            rng.normals4(0, 0, (uint32_t)p, ctr_word3(f, ST_CAM, 1), z + 4);
            double a[6];
            for (int q = 0; q < 6; ++q) a[q] = cfg.cam_std[q] * z[q];
            Ext& e = ext[p];
            for (int q = 0; q < 3; ++q) {   // linearcvmotionmodel3d.cuh:28-40
                e.c[q] = (e.c[q] + e.c[q + 3] * dt) + 0.5 * a[q] * dt * dt;
                e.c[q + 3] = e.c[q + 3] + a[q] * dt;
                e.a[q] = (e.a[q] + e.a[q + 3] * dt) + 0.5 * a[3 + q] * dt * dt;
                e.a[q + 3] = e.a[q + 3] + a[3 + q] * dt;
            }
            for (int q = 0; q < 3; ++q) e.a[q] = wrap_angle(e.a[q]);
            // feature clouds, predict_features :154-178, then w *= ps :1144-1150
            std::vector<Cloud>& mp = maps[p];
            for (size_t j = 0; j < mp.size(); ++j) {
                Cloud& cl = mp[j];
                for (int s = 0; s < P; ++s) {
                    double zz[4];
                    rng.normals4((uint32_t)s, (uint32_t)j, (uint32_t)p, ctr_word3(f, ST_FEAT, 0), zz);
                    for (int q = 0; q < 3; ++q) {
                        double ax = cfg.feat_std[q] * zz[q];
                        double x = cl.x[q * P + s], vx = cl.x[(q + 3) * P + s];
                        cl.x[q * P + s] = x + vx * dt + 0.5 * ax * dt * dt;
                        cl.x[(q + 3) * P + s] = vx + ax * dt;
                    }
                }
                cl.W *= cfg.ps;
            }
        }
    }

    // ------------------------------------------------ Kalman detection term for (g, z)
    // computeDetectionsKernel, src/kernels.cu:498-598, for H = [I_K 0]
    void detect(const G6& f, double pdbar, const double* z, G6& out) const {
        const double* p = f.cov;
        double Rv[3] = {cfg.std_u * cfg.std_u, cfg.std_v * cfg.std_v, cfg.std_d * cfg.std_d};
        double innov[3], S[9], Si[9];
        for (int a = 0; a < K; ++a) innov[a] = z[a] - f.mean[a];
        for (int a = 0; a < K; ++a)
            for (int b = 0; b < K; ++b) S[a + b * K] = p[a + b * 6] + (a == b ? Rv[a] : 0.0);
        for (int a = 0; a < K; ++a)   // enforce symmetry, kernels.cu:513-515
            for (int b = 0; b < a; ++b) {
                double s = (S[a + b * K] + S[b + a * K]) / 2;
                S[a + b * K] = s; S[b + a * K] = s;
            }
        double det;
        if (K == 2) {
            det = S[0] * S[3] - S[1] * S[2];
            Si[0] = S[3] / det; Si[1] = -S[1] / det; Si[2] = -S[2] / det; Si[3] = S[0] / det;
        } else {
            det = S[0] * (S[4] * S[8] - S[7] * S[5]) - S[3] * (S[1] * S[8] - S[7] * S[2]) +
                  S[6] * (S[1] * S[5] - S[4] * S[2]);
            Si[0] = (S[4] * S[8] - S[7] * S[5]) / det;
            Si[1] = (S[7] * S[2] - S[1] * S[8]) / det;
            Si[2] = (S[1] * S[5] - S[4] * S[2]) / det;
            Si[3] = (S[6] * S[5] - S[3] * S[8]) / det;
            Si[4] = (S[0] * S[8] - S[6] * S[2]) / det;
            Si[5] = (S[2] * S[3] - S[0] * S[5]) / det;
            Si[6] = (S[3] * S[7] - S[6] * S[4]) / det;
            Si[7] = (S[6] * S[1] - S[0] * S[7]) / det;
            Si[8] = (S[0] * S[4] - S[3] * S[1]) / det;
        }
        double dist = 0;
        for (int a = 0; a < K; ++a)
            for (int b = 0; b < K; ++b) dist += innov[a] * Si[a + b * K] * innov[b];
        out.w = safe_log(pdbar) + safe_log(f.w) - 0.5 * dist - 0.5 * K * safe_log(2 * kPi) -
                0.5 * safe_log(det);
        // K = P H' S^-1 (6 x K, column-major)
        double Kg[18];
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < K; ++c) {
                double s = 0;
                for (int a = 0; a < K; ++a) s += p[r + a * 6] * Si[a + c * K];
                Kg[r + c * 6] = s;
            }
        for (int r = 0; r < 6; ++r) {
            double s = f.mean[r];
            for (int c = 0; c < K; ++c) s += innov[c] * Kg[r + c * 6];
            out.mean[r] = s;
        }
        // Joseph form (I - K H) P (I - K H)' + K R K'
        double A[36], AP[36];
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c)
                A[r + c * 6] = (r == c ? 1.0 : 0.0) - (c < K ? Kg[r + c * 6] : 0.0);
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c) {
                double s = 0;
                for (int a = 0; a < 6; ++a) s += A[r + a * 6] * p[a + c * 6];
                AP[r + c * 6] = s;
            }
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c) {
                double s = 0;
                for (int a = 0; a < 6; ++a) s += AP[r + a * 6] * A[c + a * 6];
                for (int a = 0; a < K; ++a) s += Kg[r + a * 6] * Rv[a] * Kg[c + a * 6];
                out.cov[r + c * 6] = s;
            }
        if (!is_pos_def6_strict(out.cov)) out.w = safe_log(0);   // kernels.cu:597-598
    }

    // Map capacity.  The reference keeps every merged component and every retained
    // non-detection cloud (compaction src/scphdcameracalibration.cu:1923-1942 copies
    // all of them); this implementation bounds a parent's map at max_gaussians
    // entries.  When the new map (merged components in merge order, then the retained
    // non-detection clouds in Gaussian order) holds more, the max_gaussians entries of
    // largest weight are kept, equal weights in entry order, and the kept entries
    // keep their order.  max_gaussians <= 0 means no cap.
    void cap_map(std::vector<Cloud>& out, std::vector<double>& precut) {
        const int cap = cfg.max_gaussians;
        precut.resize(out.size());
        for (size_t i = 0; i < out.size(); ++i) precut[i] = out[i].W;
        if (cap <= 0 || (int)out.size() <= cap) return;
        std::vector<double> w(out.size());
        for (size_t i = 0; i < out.size(); ++i) w[i] = out[i].W;
        std::vector<char> keep;
        cap_keep(w, cap, keep);
        std::vector<Cloud> kept;
        kept.reserve(cap);
        for (size_t i = 0; i < out.size(); ++i)
            if (keep[i]) kept.push_back(std::move(out[i]));
        out.swap(kept);
#pragma omp atomic
        ++truncations;
    }

    static double lse(double a, double b) {   // log_sum_exp functor, .cu:506-517
        if (a > b) return a + safe_log(1 + std::exp(b - a));
        return b + safe_log(1 + std::exp(a - b));
    }

    // ------------------------------------------------ update
    void update(const double* zu, const double* zv, const double* zd, int M, bool fixed) {
        last_M = M;
        fitted.assign(N, {});
        pbar.assign(N, {});
        merged.assign(N, {});
        ell.assign((size_t)N * M, 0.0);
        loglik.assign(N, 0.0);
        survivors.assign(N, 0);
        precut.assign(N, {});
        const double bpc = safe_log(M * cfg.w0 + cfg.kappa);   // .cu:1744-1745
        const double log_w0 = safe_log(cfg.w0);
        const Ext zero_ext = {{0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0}};
        const int f = frame;
#pragma omp parallel for schedule(dynamic, 4)
        for (int p = 0; p < N; ++p) {
            const Ext& e = fixed ? zero_ext : ext[p];
            std::vector<Cloud>& mp = maps[p];
            const int G = (int)mp.size();
            std::vector<G6>& fit = fitted[p];
            fit.resize(G);
            pbar[p].resize(G);
            std::vector<Cloud> nd;   // non-detection clouds, in disparity space
            std::vector<double> ydisp(6 * P), pds(P), om(P);
            for (int j = 0; j < G; ++j) {
                Cloud& cl = mp[j];
                int n_in = 0;
                for (int s = 0; s < P; ++s) {
                    double X[6], y[6];
                    for (int q = 0; q < 6; ++q) X[q] = cl.x[q * P + s];
                    measure(X, e, y);
                    for (int q = 0; q < 6; ++q) ydisp[q * P + s] = y[q];
                    pds[s] = in_range(y) ? cfg.pd : 0.0;
                    n_in += in_range(y);
                    om[s] = cl.om[s] * pds[s];       // .cu:1602-1609
                }
                double sum = 0;
                for (int s = 0; s < P; ++s) sum += om[s];
                if (sum == 0 && n_in > 0) {   // every weight becomes exp(LOG0 - LOG0) = 1
#pragma omp atomic
                    ++unit_weight_fits;
                }
                for (int s = 0; s < P; ++s) om[s] = std::exp(safe_log(om[s]) - safe_log(sum));
                G6& g = fit[j];
                g.w = cl.W;
                for (int q = 0; q < 6; ++q) {   // zero-weight samples do not contribute
                    double m = 0;
                    for (int s = 0; s < P; ++s)
                        if (om[s] != 0) m += ydisp[q * P + s] * om[s];
                    g.mean[q] = m;
                }
                double W = 0, SS = 0;
                for (int s = 0; s < P; ++s) { W += om[s]; SS += om[s] * om[s]; }
                double norm = W / (W * W + SS);
                for (int a = 0; a < 6; ++a)
                    for (int b = 0; b <= a; ++b) {
                        double c = 0;
                        for (int s = 0; s < P; ++s)
                            if (om[s] != 0)
                                c += (ydisp[a * P + s] - g.mean[a]) * (ydisp[b * P + s] - g.mean[b]) * om[s];
                        g.cov[a + b * 6] = c / norm;
                        g.cov[b + a * 6] = c / norm;
                    }
                pbar[p][j] = (double)n_in * cfg.pd / P;   // mean of pD_s (computePdKernel :82-99)
                double wnd = cl.W * (1 - pbar[p][j]);   // nondetect_weight, .cu:540-546
                if (wnd >= cfg.min_weight) {             // copy_if geq(min_weight), .cu:1351-1374
                    Cloud c;
                    c.W = wnd;
                    c.x = ydisp;
                    c.om.resize(P);
                    for (int s = 0; s < P; ++s) c.om[s] = 1.0 - pds[s];   // .cu:1415-1418
                    nd.push_back(std::move(c));
                }
            }
            // detection terms, m-major: index m*G + j (kernels.cu:490-492, 625-630)
            std::vector<G6> comps((size_t)G * M + M);
            std::vector<double> logw((size_t)G * M);
            for (int m = 0; m < M; ++m) {
                double z[3] = {zu[m], zv[m], zd ? zd[m] : 0.0};
                for (int j = 0; j < G; ++j) {
                    detect(fit[j], pbar[p][j], z, comps[(size_t)m * G + j]);
                    logw[(size_t)m * G + j] = comps[(size_t)m * G + j].w;
                }
            }
            double sum_ell = 0;
            for (int m = 0; m < M; ++m) {
                double l;
                if (G > 0) {
                    l = logw[(size_t)m * G];
                    for (int j = 1; j < G; ++j) l = lse(l, logw[(size_t)m * G + j]);
                    l = lse(l, bpc);
                } else {
                    l = bpc;
                }
                ell[(size_t)p * M + m] = l;
                sum_ell += l;
            }
            // births, .cu:2589-2638
            for (int m = 0; m < M; ++m) {
                G6& b = comps[(size_t)G * M + m];
                std::memset(b.cov, 0, sizeof(b.cov));
                b.mean[0] = zu[m]; b.mean[1] = zv[m];
                b.mean[2] = (K == 3 && zd) ? zd[m] : cfg.d0;
                b.mean[3] = cfg.vu0; b.mean[4] = cfg.vv0; b.mean[5] = cfg.vd0;
                b.cov[0] = cfg.std_u * cfg.std_u;
                b.cov[7] = cfg.std_v * cfg.std_v;
                b.cov[14] = (K == 3) ? cfg.std_d * cfg.std_d : cfg.var_d0;
                b.cov[21] = cfg.var_vu0; b.cov[28] = cfg.var_vv0; b.cov[35] = cfg.var_vd0;
                b.w = log_w0;
            }
            // updateKernel: normalise, prune flags, src/kernels.cu:622-657
            std::vector<uint8_t> flags(comps.size());
            for (size_t i = 0; i < comps.size(); ++i) {
                int m = i < (size_t)G * M ? (int)(i / (size_t)(G > 0 ? G : 1)) : (int)(i - (size_t)G * M);
                comps[i].w = std::exp(comps[i].w - ell[(size_t)p * M + m]);
                flags[i] = (comps[i].w < cfg.min_weight) || !is_pos_def6_strict(comps[i].cov);
                survivors[p] += !flags[i];
            }
            // parent log-likelihood, .cu:1813-1849: sum_m ell + sum_j w_j (predicted)
            double card = 0;
            for (int j = 0; j < G; ++j) card += mp[j].W;
            loglik[p] = sum_ell + card;
            // merge
            std::vector<G6>& mg = merged[p];
            merge_map(comps, flags, cfg.min_separation, mg, nullptr);
            // new map: sampled merged Gaussians then non-detection clouds, in world space
            std::vector<Cloud> out;
            out.reserve(mg.size() + nd.size());
            for (size_t i = 0; i < mg.size(); ++i) {
                Cloud c;
                c.W = mg[i].w;
                c.x.resize(6 * P);
                c.om.assign(P, 1.0 / P);
                double L[36];
                cholesky(mg[i].cov, L, 6);
                for (int s = 0; s < P; ++s) {
                    double z[8];
                    rng.normals4((uint32_t)s, (uint32_t)i, (uint32_t)p, ctr_word3(f, ST_SAMPLE, 0), z);
                    rng.normals4((uint32_t)s, (uint32_t)i, (uint32_t)p, ctr_word3(f, ST_SAMPLE, 1), z + 4);
                    double y[6], X[6];
                    for (int a = 0; a < 6; ++a) {     // sample_disparity_gaussian, .cu:672-682
                        double v = 0;
                        for (int b = 0; b <= a; ++b) v += L[a + b * 6] * z[b];
                        y[a] = v + mg[i].mean[a];
                    }
                    invert(y, e, X);
                    for (int q = 0; q < 6; ++q) c.x[q * P + s] = X[q];
                }
                out.push_back(std::move(c));
            }
            for (Cloud& c : nd) {   // computeEuclideanParticles, .cu:1222-1286
                std::vector<double> X6(6 * P);
                for (int s = 0; s < P; ++s) {
                    double y[6], X[6];
                    for (int q = 0; q < 6; ++q) y[q] = c.x[q * P + s];
                    invert(y, e, X);
                    for (int q = 0; q < 6; ++q) X6[q * P + s] = X[q];
                }
                c.x.swap(X6);
                out.push_back(std::move(c));
            }
            cap_map(out, precut[p]);
            mp.swap(out);
        }
        if (!fixed) {   // parent weights, .cu:1813-1876
            if (weight_mode == 0) {
                double mx = -INFINITY;
                for (int p = 0; p < N; ++p) { lw[p] += loglik[p]; mx = std::max(mx, lw[p]); }
                double s = 0;
                for (int p = 0; p < N; ++p) s += std::exp(lw[p] - mx);
                double ls = mx + std::log(s);
                for (int p = 0; p < N; ++p) lw[p] -= ls;
            } else {
                for (int p = 0; p < N; ++p) lw[p] *= std::exp(loglik[p]);
                double s = 0;
                for (int p = 0; p < N; ++p) s += lw[p];
                for (int p = 0; p < N; ++p) lw[p] /= s;
            }
        }
    }

    // ------------------------------------------------ resample
    int resample() {
        std::vector<double> w(N);
        double ss = 0;
        for (int p = 0; p < N; ++p) { w[p] = linear_weight(p); ss += w[p] * w[p]; }
        double neff = 1.0 / (N * ss);                    // computeNeff, .cu:2641-2649
        if (neff >= cfg.min_neff) return 0;
        uint32_t wd[4];
        rng.words(0, 0, 0, ctr_word3(frame, ST_RESAMPLE, 0), wd);
        double r0 = u01_of(wd[0]) * (1.0 / N);
        systematic(w, r0, resample_idx);
        std::vector<Ext> ne(N);
        std::vector<std::vector<Cloud>> nm(N);
        for (int j = 0; j < N; ++j) { ne[j] = ext[resample_idx[j]]; nm[j] = maps[resample_idx[j]]; }
        ext.swap(ne);
        maps.swap(nm);
        for (int p = 0; p < N; ++p) lw[p] = weight_mode ? 1.0 / N : -std::log((double)N);
        return 1;
    }
};

void g6_to_packed(const G6& g, double* out, bool with_pd, double pd) {
    int o = 0;
    out[o++] = g.w;
    if (with_pd) out[o++] = pd;
    for (int q = 0; q < 6; ++q) out[o++] = g.mean[q];
    for (int a = 0; a < 6; ++a)
        for (int b = 0; b <= a; ++b) out[o++] = g.cov[a + b * 6];
}

void packed_to_g6(const double* in, G6& g) {
    g.w = in[0];
    for (int q = 0; q < 6; ++q) g.mean[q] = in[1 + q];
    int o = 7;
    for (int a = 0; a < 6; ++a)
        for (int b = 0; b <= a; ++b) {
            g.cov[a + b * 6] = in[o];
            g.cov[b + a * 6] = in[o];
            ++o;
        }
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

void* orc_create(const scphd_config* cfg) { return new Oracle(*cfg); }
void orc_destroy(void* h) { delete static_cast<Oracle*>(h); }
void orc_set_weight_mode(void* h, int mode) {
    Oracle* o = static_cast<Oracle*>(h);
    if (mode != o->weight_mode)
        for (int p = 0; p < o->N; ++p) o->lw[p] = mode ? std::exp(o->lw[p]) : std::log(o->lw[p]);
    o->weight_mode = mode;
}
int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}
void orc_predict(void* h, double dt) { static_cast<Oracle*>(h)->predict(dt); }
void orc_update(void* h, const double* u, const double* v, const double* d, int M, int fixed) {
    static_cast<Oracle*>(h)->update(u, v, d, M, fixed != 0);
}
int orc_resample(void* h) { return static_cast<Oracle*>(h)->resample(); }
int orc_frame(void* h) { return static_cast<Oracle*>(h)->frame; }
// the frame counter keys the random streams: a state copied into a fresh oracle with
// the same counter replays the same work
void orc_set_frame(void* h, int frame) { static_cast<Oracle*>(h)->frame = frame; }

void orc_get_particles(void* h, double* states, double* logw) {
    Oracle* o = static_cast<Oracle*>(h);
    for (int p = 0; p < o->N; ++p) {
        if (states) {
            std::memcpy(states + 12 * p, o->ext[p].c, 6 * sizeof(double));
            std::memcpy(states + 12 * p + 6, o->ext[p].a, 6 * sizeof(double));
        }
        if (logw) logw[p] = o->weight_mode ? std::log(o->lw[p]) : o->lw[p];
    }
}
int orc_map_size(void* h, int p) { return (int)static_cast<Oracle*>(h)->maps[p].size(); }
void orc_get_map(void* h, int p, double* W, double* xyz, double* om) {
    Oracle* o = static_cast<Oracle*>(h);
    const int P = o->P;
    const std::vector<Cloud>& mp = o->maps[p];
    for (size_t j = 0; j < mp.size(); ++j) {
        if (W) W[j] = mp[j].W;
        if (xyz) std::memcpy(xyz + j * 6 * P, mp[j].x.data(), 6 * P * sizeof(double));
        if (om) std::memcpy(om + j * P, mp[j].om.data(), P * sizeof(double));
    }
}
void orc_set_state(void* h, const double* states, const double* logw, const int* sizes,
                   const double* W, const double* xyz, const double* om) {
    Oracle* o = static_cast<Oracle*>(h);
    const int P = o->P;
    size_t g = 0;
    for (int p = 0; p < o->N; ++p) {
        std::memcpy(o->ext[p].c, states + 12 * p, 6 * sizeof(double));
        std::memcpy(o->ext[p].a, states + 12 * p + 6, 6 * sizeof(double));
        o->lw[p] = o->weight_mode ? std::exp(logw[p]) : logw[p];
        o->maps[p].assign(sizes[p], Cloud());
        for (int j = 0; j < sizes[p]; ++j, ++g) {
            Cloud& c = o->maps[p][j];
            c.W = W[g];
            c.x.assign(xyz + g * 6 * P, xyz + (g + 1) * 6 * P);
            c.om.assign(om + g * P, om + (g + 1) * P);
        }
    }
}
int orc_fitted_count(void* h, int p) { return (int)static_cast<Oracle*>(h)->fitted[p].size(); }
void orc_get_fitted(void* h, int p, double* out) {   // rows of 29
    Oracle* o = static_cast<Oracle*>(h);
    for (size_t j = 0; j < o->fitted[p].size(); ++j)
        g6_to_packed(o->fitted[p][j], out + 29 * j, true, o->pbar[p][j]);
}
int orc_merged_count(void* h, int p) { return (int)static_cast<Oracle*>(h)->merged[p].size(); }
void orc_get_merged(void* h, int p, double* out) {   // rows of 28
    Oracle* o = static_cast<Oracle*>(h);
    for (size_t j = 0; j < o->merged[p].size(); ++j) g6_to_packed(o->merged[p][j], out + 28 * j, false, 0);
}
void orc_get_normalizers(void* h, double* ell, double* loglik) {
    Oracle* o = static_cast<Oracle*>(h);
    if (ell) std::memcpy(ell, o->ell.data(), o->ell.size() * sizeof(double));
    if (loglik) std::memcpy(loglik, o->loglik.data(), o->loglik.size() * sizeof(double));
}
void orc_get_survivors(void* h, int* out) {
    Oracle* o = static_cast<Oracle*>(h);
    std::memcpy(out, o->survivors.data(), o->survivors.size() * sizeof(int));
}
void orc_get_resample_indices(void* h, int* idx) {
    Oracle* o = static_cast<Oracle*>(h);
    for (size_t j = 0; j < o->resample_idx.size(); ++j) idx[j] = o->resample_idx[j];
}

// ---- stand-alone stages
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    philox4x32(ctr, key, out, kPhiloxRounds);
}
void orc_philox_rounds(const uint32_t ctr[4], const uint32_t key[2], int rounds, uint32_t out[4]) {
    philox4x32(ctr, key, out, rounds);
}
void orc_normals4(uint64_t seed, uint32_t s, uint32_t j, uint32_t p, uint32_t c3, double z[4]) {
    Stream st{seed};
    st.normals4(s, j, p, c3, z);
}
uint32_t orc_ctr_word3(int frame, int stage, int block) { return ctr_word3(frame, stage, block); }

void orc_merge(const double* comps, const uint8_t* flags_in, int n, double min_sep, double* out,
               int* n_out, int* member_of) {
    std::vector<G6> c(n);
    for (int i = 0; i < n; ++i) packed_to_g6(comps + 28 * i, c[i]);
    std::vector<uint8_t> flags(flags_in, flags_in + n);
    std::vector<G6> mg;
    std::vector<int> mem;
    merge_map(c, flags, min_sep, mg, &mem);
    for (size_t i = 0; i < mg.size(); ++i) g6_to_packed(mg[i], out + 28 * i, false, 0);
    *n_out = (int)mg.size();
    if (member_of) for (int i = 0; i < n; ++i) member_of[i] = mem[i];
}
void orc_systematic(const double* w, int n, double u01, int* idx) {
    std::vector<double> ww(w, w + n);
    std::vector<int> out;
    systematic(ww, u01 * (1.0 / n), out);
    std::memcpy(idx, out.data(), n * sizeof(int));
}
double orc_mahal6(const double* a28, const double* b28) {
    G6 a, b;
    packed_to_g6(a28, a);
    packed_to_g6(b28, b);
    return mahal6(a, b);
}
int orc_is_pos_def(const double* cov36) { return is_pos_def6(cov36); }
double orc_wrap_angle(double a) { return wrap_angle(a); }
uint32_t orc_tie_key(uint32_t r) { return tie_key(r); }
// the map-capacity cut on a list of entry weights: keep[i] = 1 for kept entries
void orc_cap_keep(const double* w, int n, int cap, uint8_t* keep) {
    std::vector<double> ww(w, w + n);
    std::vector<char> k;
    cap_keep(ww, cap, k);
    for (int i = 0; i < n; ++i) keep[i] = (uint8_t)k[i];
}
long long orc_truncations(void* h) { return static_cast<Oracle*>(h)->truncations; }
long long orc_unit_weight_fits(void* h) { return static_cast<Oracle*>(h)->unit_weight_fits; }
// entry weights of parent p's new map before the capacity cut (last update); returns
// the count, writes them when out is not null
int orc_precut_weights(void* h, int p, double* out) {
    const std::vector<double>& w = static_cast<Oracle*>(h)->precut[p];
    if (out) std::memcpy(out, w.data(), w.size() * sizeof(double));
    return (int)w.size();
}

// world -> disparity of one point with extrinsic e (12), using the filter's model
void orc_measure(void* h, const double* X, const double* e12, double* y) {
    Oracle* o = static_cast<Oracle*>(h);
    Ext e;
    std::memcpy(e.c, e12, 6 * sizeof(double));
    std::memcpy(e.a, e12 + 6, 6 * sizeof(double));
    o->measure(X, e, y);
}
void orc_invert(void* h, const double* y, const double* e12, double* X) {
    Oracle* o = static_cast<Oracle*>(h);
    Ext e;
    std::memcpy(e.c, e12, 6 * sizeof(double));
    std::memcpy(e.a, e12 + 6, 6 * sizeof(double));
    o->invert(y, e, X);
}
// one detection term: fitted Gaussian (29: w, pd, mean, packed cov) and measurement z
void orc_detect(void* h, const double* g29, const double* z, double* out28) {
    Oracle* o = static_cast<Oracle*>(h);
    G6 g, r;
    double tmp[28];
    tmp[0] = g29[0];
    std::memcpy(tmp + 1, g29 + 2, 27 * sizeof(double));
    packed_to_g6(tmp, g);
    o->detect(g, g29[1], z, r);
    g6_to_packed(r, out28, false, 0);
}

}  // extern "C"

// ref_glue.cpp — TEST INFRASTRUCTURE.  extern "C" entry points over the reference's
// own sources compiled for the host (see ref_shim.h): they run the reference's
// per-thread kernels by setting threadIdx/blockIdx in a loop, and call its
// __host__ __device__ model and matrix functions, so tests can compare the
// oracle's restatement with the reference code itself.  Only tests link this.
#include "types.h"
#include "kernels.cuh"
#include "device_math.cuh"
#include "disparitymeasurementmodel.cuh"
#include "OrientedLinearCVMotionModel3D.cuh"

#include <cstring>
#include <vector>

thread_local ShimDim3 threadIdx, blockIdx, blockDim, gridDim;

template <int N, int N2> double computeMahalDist(Gaussian<N, N2> a, Gaussian<N, N2> b);
template <int N, int N2> bool isPosDef(Gaussian<N, N2> g);

namespace {
DisparityMeasurementModel model_of(const double* m8) {
    // fx, fy, u0, v0, std_u, std_v, pd, lambda
    return DisparityMeasurementModel(m8[0], m8[1], m8[2], m8[3], m8[4], m8[5], m8[6], m8[7]);
}
Extrinsics ext_of(const double* e) {
    Extrinsics x;
    x.cartesian = {e[0], e[1], e[2], e[3], e[4], e[5]};
    x.angular = {e[6], e[7], e[8], e[9], e[10], e[11]};
    return x;
}
void packed_to_g(const double* in, Gaussian6D& g) {   // w, mean[6], packed lower cov[21]
    g.weight = in[0];
    for (int q = 0; q < 6; ++q) g.mean[q] = in[1 + q];
    int o = 7;
    for (int a = 0; a < 6; ++a)
        for (int b = 0; b <= a; ++b) { g.cov[a + 6 * b] = in[o]; g.cov[b + 6 * a] = in[o]; ++o; }
    g.dims = 6;
}
void g_to_full(const Gaussian6D& g, double* out37) {   // w, mean[6]... no: w + cov full 36 col-major
    out37[0] = g.weight;
    std::memcpy(out37 + 1, g.mean, 6 * sizeof(double));
    std::memcpy(out37 + 7, g.cov, 36 * sizeof(double));
}
void launch1d(int n, int block, void (*body)(void*), void* ctx) {
    blockDim = {(unsigned)block, 1, 1};
    gridDim = {(unsigned)((n + block - 1) / block), 1, 1};
    for (unsigned b = 0; b < gridDim.x; ++b)
        for (unsigned t = 0; t < blockDim.x; ++t) {
            blockIdx = {b, 0, 0};
            threadIdx = {t, 0, 0};
            body(ctx);
        }
}
}  // namespace

extern "C" {

double ref_safe_log(double x) { return safeLog(x); }
double ref_wrap_angle(double a) { return wrapAngle(a); }
void ref_cholesky(const double* A, double* L, int n) { cholesky(const_cast<double*>(A), L, n); }
int ref_is_pos_def(const double* cov36) {
    Gaussian6D g;
    std::memcpy(g.cov, cov36, 36 * sizeof(double));
    g.weight = 1; g.dims = 6;
    return isPosDef(g) ? 1 : 0;
}
double ref_mahal(const double* a28, const double* b28) {
    Gaussian6D a, b;
    packed_to_g(a28, a);
    packed_to_g(b28, b);
    return computeMahalDist(a, b);
}
void ref_measure(const double* m8, const double* X, const double* e12, double* y) {
    DisparityMeasurementModel m = model_of(m8);
    EuclideanPoint p = {X[0], X[1], X[2], X[3], X[4], X[5]};
    DisparityPoint d = m.computeMeasurement(p, ext_of(e12));
    y[0] = d.u; y[1] = d.v; y[2] = d.d; y[3] = d.vu; y[4] = d.vv; y[5] = d.vd;
}
void ref_invert(const double* m8, const double* y, const double* e12, double* X) {
    DisparityMeasurementModel m = model_of(m8);
    DisparityPoint d;
    d.u = y[0]; d.v = y[1]; d.d = y[2]; d.vu = y[3]; d.vv = y[4]; d.vd = y[5];
    EuclideanPoint p = m.invertMeasurement(d, ext_of(e12));
    X[0] = p.x; X[1] = p.y; X[2] = p.z; X[3] = p.vx; X[4] = p.vy; X[5] = p.vz;
}
// OrientedLinearCVMotionModel3D::computeNoisyMotion on one 12-D state
void ref_noisy_motion(double* e12, double dt, const double* a6) {
    OrientedLinearCVMotionModel3D model(1, 1, 1, 1, 1, 1);
    EuclideanPoint c = {e12[0], e12[1], e12[2], e12[3], e12[4], e12[5]};
    EuclideanPoint a = {e12[6], e12[7], e12[8], e12[9], e12[10], e12[11]};
    model.computeNoisyMotion(c, a, dt, a6[0], a6[1], a6[2], a6[3], a6[4], a6[5]);
    double out[12] = {c.x, c.y, c.z, c.vx, c.vy, c.vz, a.x, a.y, a.z, a.vx, a.vy, a.vz};
    std::memcpy(e12, out, sizeof(out));
}

// worldToDisparityKernel (src/kernels.cu:6-47) over n points; indices[i] selects ex row
void ref_world_to_disparity(const double* m8, const double* X6xn, int n, const double* ex12,
                            const int* indices, double* y6xn, double* pd) {
    std::vector<double> x[6], y[6];
    for (int q = 0; q < 6; ++q) { x[q].assign(X6xn + q * n, X6xn + (q + 1) * n); y[q].assign(n, 0); }
    int n_ext = 0;
    for (int i = 0; i < n; ++i) n_ext = std::max(n_ext, indices[i] + 1);
    std::vector<Extrinsics> ex(n_ext);
    for (int k = 0; k < n_ext; ++k) ex[k] = ext_of(ex12 + 12 * k);
    struct Ctx { DisparityMeasurementModel m; std::vector<double>* x; std::vector<double>* y;
                 Extrinsics* ex; int* idx; int n; double* pd; };
    Ctx c{model_of(m8), x, y, ex.data(), const_cast<int*>(indices), n, pd};
    launch1d(n, 128, [](void* v) {
        Ctx* c = static_cast<Ctx*>(v);
        worldToDisparityKernel(c->x[0].data(), c->x[1].data(), c->x[2].data(), c->x[3].data(),
                               c->x[4].data(), c->x[5].data(), c->m, c->ex, c->idx, c->n,
                               c->y[0].data(), c->y[1].data(), c->y[2].data(), c->y[3].data(),
                               c->y[4].data(), c->y[5].data(), c->pd);
    }, &c);
    for (int q = 0; q < 6; ++q) std::memcpy(y6xn + q * n, y[q].data(), n * sizeof(double));
}

// computeDetectionsKernel (src/kernels.cu:470-603) for one map of G fitted Gaussians
// (rows of 29: w, pd, mean[6], packed cov[21]) and M (u,v) measurements.  Output
// G*M rows of 43 (weight, mean[6], full col-major cov[36]) in the kernel's layout
// m*G + j.
void ref_detections(const double* m8, const double* fit29, int G, const double* u,
                    const double* v, int M, double* out43) {
    std::vector<Gaussian6D> feats(G), det((size_t)G * M);
    std::vector<double> pd(G);
    for (int j = 0; j < G; ++j) {
        double row[28];
        row[0] = fit29[29 * j];
        std::memcpy(row + 1, fit29 + 29 * j + 2, 27 * sizeof(double));
        packed_to_g(row, feats[j]);
        pd[j] = fit29[29 * j + 1];
    }
    int offsets[2] = {0, G};
    std::vector<int> midx((size_t)G * M);
    DisparityMeasurementModel m = model_of(m8);
    blockDim = {128, 1, 1};
    gridDim = {(unsigned)((G + 127) / 128), (unsigned)M, 1};
    for (unsigned by = 0; by < gridDim.y; ++by)
        for (unsigned bx = 0; bx < gridDim.x; ++bx)
            for (unsigned t = 0; t < 128; ++t) {
                blockIdx = {bx, by, 0};
                threadIdx = {t, 0, 0};
                computeDetectionsKernel(feats.data(), const_cast<double*>(u), const_cast<double*>(v),
                                        pd.data(), m, offsets, G, M, det.data(), midx.data());
            }
    for (size_t i = 0; i < det.size(); ++i) g_to_full(det[i], out43 + 43 * i);
}

// updateKernel (src/kernels.cu:608-659) for one map: detections (G*M rows of 43),
// births (M rows of 43), normalisers (M).  Output (G+1)*M rows of 43 and flags.
void ref_update(const double* det43, int G, const double* birth43, const double* norms, int M,
                double min_weight, double* out43, unsigned char* flags) {
    auto load = [](const double* r, Gaussian6D& g) {
        g.weight = r[0];
        std::memcpy(g.mean, r + 1, 6 * sizeof(double));
        std::memcpy(g.cov, r + 7, 36 * sizeof(double));
        g.dims = 6;
    };
    std::vector<Gaussian6D> det((size_t)G * M + 1), births(M + 1), upd((size_t)(G + 1) * M + 1);
    for (size_t i = 0; i < (size_t)G * M; ++i) load(det43 + 43 * i, det[i]);
    for (int i = 0; i < M; ++i) load(birth43 + 43 * i, births[i]);
    std::vector<bool> fl((size_t)(G + 1) * M + 1);
    bool* flp = new bool[(size_t)(G + 1) * M + 1];
    int offsets[2] = {0, G};
    blockDim = {256, 1, 1};
    gridDim = {1, 1, 1};
    for (unsigned t = 0; t < 256; ++t) {
        blockIdx = {0, 0, 0};
        threadIdx = {t, 0, 0};
        updateKernel(det.data(), births.data(), const_cast<double*>(norms), offsets, 1, M,
                     upd.data(), flp, min_weight);
    }
    for (size_t i = 0; i < (size_t)(G + 1) * M; ++i) { g_to_full(upd[i], out43 + 43 * i); flags[i] = flp[i]; }
    delete[] flp;
}

}  // extern "C"

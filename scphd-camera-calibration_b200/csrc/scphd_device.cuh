// scphd_device.cuh — device math of the SC-PHD filter step, templated on the
// arithmetic type T (float for the fast path, double for the FP64 path).
//
// Storage conventions (shared by every kernel):
//   * a symmetric 6x6 matrix is packed lower-triangular row-major: element (a,b),
//     a >= b, at a*(a+1)/2 + b (21 values);
//   * a mixture component row is 32 T: [0] weight, [1..6] mean, [7..27] packed cov;
//   * a fitted row is 32 T: [0] weight, [1] mean pD, [2..7] mean, [8..28] packed cov;
//   * a prep row (per fitted Gaussian, measurement-independent Kalman terms) is
//     48 T: [0] log-constant c, [1] PD flag of the posterior cov, [2..7] packed
//     S^-1 (k x k, packed lower), [8..25] gain K (6 x 3, row-major), [26..46]
//     packed posterior covariance.
#pragma once

#include <cstdint>
#include <cfloat>
#include <cuda_runtime.h>

namespace scphd {

constexpr int kRow = 32;
constexpr int kPrep = 48;
constexpr int kPrepSi = 2, kPrepK = 8, kPrepCov = 26;
constexpr int kMaxLanesSamples = 8;   // particles_per_feature <= 256

enum Stage : uint32_t { ST_PRIOR = 1, ST_CAM = 2, ST_FEAT = 3, ST_SAMPLE = 4, ST_RESAMPLE = 5 };

__host__ __device__ inline int tri(int a, int b) { return a >= b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a; }

__host__ __device__ inline uint32_t ctr_word3(uint32_t frame, uint32_t stage, uint32_t block) {
    return (frame << 12) | (stage << 8) | block;
}

// Philox4x32 (Salmon, Moraes, Dror and Shaw, SC'11) with 7 rounds, the fewest the
// authors report passing TestU01's BigCrush; counter (s, j, p, c3), key = seed
constexpr int kPhiloxRounds = 7;
__host__ __device__ inline void philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                       uint32_t k0, uint32_t k1, uint32_t out[4]) {
#pragma unroll
    for (int r = 0; r < kPhiloxRounds; ++r) {
        // one 32x32 -> 64-bit product per multiplier gives both halves
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// The same generator with its round keys taken from a table (rk[2r], rk[2r+1] = the
// keys of round r): with the table in kernel parameters the keys cost no instructions.
__device__ __forceinline__ void philox_rk(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, const uint32_t* rk,
                                          uint32_t out[4]) {
#pragma unroll
    for (int r = 0; r < kPhiloxRounds; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c1 ^ rk[2 * r], n2 = hi0 ^ c3 ^ rk[2 * r + 1];
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

__host__ __device__ inline double u01(uint32_t w) { return ((double)w + 0.5) * 0x1p-32; }

// four standard normals (two Box-Muller pairs) from one Philox block
template <typename T> struct Normals;
template <> struct Normals<double> {
    __device__ static void four(const uint32_t w[4], double z[4]) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            double r = sqrt(-2.0 * log(u01(w[2 * h])));
            double s, c;
            sincos((2.0 * 3.14159265358979323846) * u01(w[2 * h + 1]), &s, &c);
            z[2 * h] = r * c;
            z[2 * h + 1] = r * s;
        }
    }
};
template <> struct Normals<float> {
    __device__ static void four(const uint32_t w[4], float z[4]) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float ua = __fmaf_rn((float)w[2 * h], 0x1p-32f, 0x1p-33f);
            float ub = __fmaf_rn((float)w[2 * h + 1], 0x1p-32f, 0x1p-33f);
            ua = fminf(ua, 0.99999994f);
            float r = sqrtf(-2.0f * logf(ua));
            float s, c;
            sincospif(2.0f * ub, &s, &c);
            z[2 * h] = r * c;
            z[2 * h + 1] = r * s;
        }
    }
};

// One Box-Muller pair from two 32-bit words: z0 = r cos(2 pi u_b), z1 = r sin(2 pi u_b),
// r = sqrt(-2 log u_a), the same pair Normals<T>::four produces.  The FP32 form uses
// the MUFU approximations (lg2, sin, cos) with the angle shifted into [-pi, pi):
// cos(2 pi u) = -cos(2 pi (u - 1/2)), sin likewise.
template <typename T> struct Pair;
template <> struct Pair<double> {
    __device__ static void two(uint32_t wa, uint32_t wb, double& z0, double& z1) {
        double r = sqrt(-2.0 * log(u01(wa)));
        double s, c;
        sincos((2.0 * 3.14159265358979323846) * u01(wb), &s, &c);
        z0 = r * c;
        z1 = r * s;
    }
};
template <> struct Pair<float> {
    __device__ static void two(uint32_t wa, uint32_t wb, float& z0, float& z1) {
        const float ua = fminf(__fmaf_rn((float)wa, 0x1p-32f, 0x1p-33f), 0.99999994f);
        // r^2 = -2 ln u_a = (-2 ln 2) log2 u_a, one multiply on the hardware base-2 log.
        // The approximate log (absolute error up to about 1e-7 near 1) of the largest u_a
        // below 1 can come out as 0 or above: r is 0 there instead of NaN
        const float r2 = __log2f(ua) * -1.3862943611198906f;
        const float r = r2 > 0.0f ? r2 * rsqrtf(r2) : 0.0f;
        // the angle 2 pi (u_b - 1/2) = 2 pi ((w_b + 1/2) 2^-32 - 1/2) in one multiply-add
        const float th = __fmaf_rn((float)wb, 6.283185307179586f * 0x1p-32f, 6.283185307179586f * (0x1p-33f - 0.5f));
        float s, c;
        __sincosf(th, &s, &c);
        z0 = -r * c;
        z1 = -r * s;
    }
};

template <typename T> __device__ __forceinline__ T tsqrt(T x);
template <> __device__ __forceinline__ float tsqrt(float x) { return sqrtf(x); }
template <> __device__ __forceinline__ double tsqrt(double x) { return sqrt(x); }
template <typename T> __device__ __forceinline__ T texp(T x);
template <> __device__ __forceinline__ float texp(float x) { return expf(x); }
template <> __device__ __forceinline__ double texp(double x) { return exp(x); }
// exp for the FP64 likelihood's normaliser sums and survivor weights (the FP32
// likelihood works in base 2, exp2_approx); the FP32 form is the hardware base-2
// exponential of x log2(e) (__expf: relative error about 2 ulp + |x| 2^-22)
__device__ __forceinline__ float texp_sum(float x) { return __expf(x); }
__device__ __forceinline__ double texp_sum(double x) { return exp(x); }
template <typename T> __device__ __forceinline__ T tlog(T x);
template <> __device__ __forceinline__ float tlog(float x) { return logf(x); }
template <> __device__ __forceinline__ double tlog(double x) { return log(x); }

template <typename T> __device__ __forceinline__ T tneg_inf();
template <> __device__ __forceinline__ float tneg_inf() { return -INFINITY; }
template <> __device__ __forceinline__ double tneg_inf() { return -INFINITY; }

// ------------------------------------------------------------------ camera model
// Rotation terms of the reference's world<->camera transform
// (src/disparitymeasurementmodel.cu:3-144), evaluated once per parent in FP64.
template <typename T> struct Pose {
    T R[9];    // world->camera rows
    T t[3];    // camera position in the world
};

__device__ inline void pose_terms(const double* e12, double R[9]) {
    double ct, st, cf, sf, cp, sp;
    sincos(e12[6], &st, &ct);
    sincos(e12[7], &sf, &cf);
    sincos(e12[8], &sp, &cp);
    R[0] = cf * cp; R[1] = ct * sp + st * sf * cp; R[2] = st * sp - ct * sf * cp;
    R[3] = -cf * sp; R[4] = ct * cp - st * sf * sp; R[5] = st * cp + ct * sf * sp;
    R[6] = sf; R[7] = -st * cf; R[8] = ct * cf;
}

template <typename T> __device__ inline Pose<T> make_pose(const double* e12) {
    double R[9];
    pose_terms(e12, R);
    Pose<T> P;
#pragma unroll
    for (int i = 0; i < 9; ++i) P.R[i] = (T)R[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) P.t[i] = (T)e12[i];
    return P;
}

struct Model {   // measurement model constants (FP64 copy; kernels cast to T)
    double fx, fy, u0, v0, B, pd;
    double var[3];   // std_u^2, std_v^2, std_d^2
};
// The cloud fit's model constants (the transforms' and the feature noise) rounded to
// FP32 on the host (the same round-to-nearest as a device cast), read by the FP32
// kernels straight from the kernel parameters
struct ModelF {
    float fx, fy, u0, v0, B, pd;
    float feat_std[3];
};

// Weight of a Gaussian's non-detection term, W (1 - mean pD), rounded step by step
// (no contraction) so that the cloud-fit and merge kernels decide identically
// whether the term survives the min_weight prune.
__device__ __forceinline__ float nd_weight(float W, float pbar) { return __fmul_rn(W, __fsub_rn(1.0f, pbar)); }
__device__ __forceinline__ double nd_weight(double W, double pbar) { return __dmul_rn(W, __dsub_rn(1.0, pbar)); }

// Reciprocal in the transforms: correctly rounded in FP64; in FP32 the hardware
// approximation (max 2 ulp), inside the FP32 mode's tolerance against FP64.
__device__ __forceinline__ double trcp(double x) { return 1.0 / x; }
__device__ __forceinline__ float trcp(float x) { return __fdividef(1.0f, x); }

// world point -> (u, v, d, vu, vv, vd), computeMeasurement (:165-196) with baseline B
template <typename T, typename M>
__device__ inline void measure(const T X[6], const Pose<T>& P, const M& m, T y[6]) {
    T d0 = X[0] - P.t[0], d1 = X[1] - P.t[1], d2 = X[2] - P.t[2];
    T x = P.R[0] * d0 + P.R[1] * d1 + P.R[2] * d2;
    T yy = P.R[3] * d0 + P.R[4] * d1 + P.R[5] * d2;
    T z = P.R[6] * d0 + P.R[7] * d1 + P.R[8] * d2;
    T vx = P.R[0] * X[3] + P.R[1] * X[4] + P.R[2] * X[5];
    T vy = P.R[3] * X[3] + P.R[4] * X[4] + P.R[5] * X[5];
    T vz = P.R[6] * X[3] + P.R[7] * X[4] + P.R[8] * X[5];
    const T fx = (T)m.fx, fy = (T)m.fy, B = (T)m.B;
    T iz = trcp(z), iz2 = iz * iz;
    y[0] = (T)m.u0 - fx * iz * x;
    y[1] = (T)m.v0 - fy * iz * yy;
    y[2] = -fx * B * iz;
    y[3] = -fx * (vx * z - vz * x) * iz2;
    y[4] = -fy * (vy * z - vz * yy) * iz2;
    y[5] = fx * B * vz * iz2;
}

// (u, v, d, vu, vv, vd) -> world point, invertMeasurement (:198-217) with baseline B
template <typename T, typename M>
__device__ inline void invert(const T y[6], const Pose<T>& P, const M& m, T X[6]) {
    const T fx = (T)m.fx, fy = (T)m.fy, B = (T)m.B, u0 = (T)m.u0, v0 = (T)m.v0;
    T u = y[0], v = y[1], d = y[2], vu = y[3], vv = y[4], vd = y[5];
    T id = trcp(d), id2 = id * id, r = fx / fy;
    T c0 = (u - u0) * B * id;
    T c1 = r * (v - v0) * B * id;
    T c2 = -fx * B * id;
    T c3 = B * (vu * d - vd * (u - u0)) * id2;
    T c4 = r * (vv * d - vd * (v - v0)) * B * id2;
    T c5 = fx * B * vd * id2;
    // camera -> world: X = R^T c + t
    X[0] = P.R[0] * c0 + P.R[3] * c1 + P.R[6] * c2 + P.t[0];
    X[1] = P.R[1] * c0 + P.R[4] * c1 + P.R[7] * c2 + P.t[1];
    X[2] = P.R[2] * c0 + P.R[5] * c1 + P.R[8] * c2 + P.t[2];
    X[3] = P.R[0] * c3 + P.R[3] * c4 + P.R[6] * c5;
    X[4] = P.R[1] * c3 + P.R[4] * c4 + P.R[7] * c5;
    X[5] = P.R[2] * c3 + P.R[5] * c4 + P.R[8] * c5;
}

template <typename T, typename M>
__device__ inline bool in_range(const T y[6], const M& m) {   // kernels.cu:37-41
    return y[0] >= T(0) && y[0] <= T(2 * m.u0) && y[1] >= T(0) && y[1] <= T(2 * m.v0) && y[2] >= T(0);
}

// ------------------------------------------------------------------ 6x6 algebra
// Cholesky in the order of src/device_math.cu:123-150 on a packed matrix; returns
// false if any factor entry is NaN (isPosDef, :800-812).
template <typename T>
__device__ inline bool chol6(const T* A, T* L) {
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            T tmp = A[tri(i, j)];
            if (i == j) {
#pragma unroll
                for (int k = 0; k < j; ++k) tmp -= L[tri(j, k)] * L[tri(j, k)];
                L[tri(i, i)] = tsqrt(tmp);
            } else {
#pragma unroll
                for (int k = 0; k < j; ++k) tmp -= L[tri(i, k)] * L[tri(j, k)];
                L[tri(i, j)] = tmp / L[tri(j, j)];
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 21; ++i) ok = ok && !isnan(L[i]);
    return ok;
}

// FP32 form of the factorisation: each pivot's reciprocal square root is taken once
// and the column below the pivot is scaled by it (hardware rsqrt, max 2 ulp), in the
// same order.  A pivot <= 0 gives NaN (0 * inf, or the rsqrt of a negative number): the
// PD outcome is the division form's, except that an exactly zero last pivot also
// reports not PD.  The FP64 form keeps the square roots and divisions.
template <>
__device__ inline bool chol6<float>(const float* A, float* L) {
    float inv[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            float tmp = A[tri(i, j)];
            if (i == j) {
#pragma unroll
                for (int k = 0; k < j; ++k) tmp -= L[tri(j, k)] * L[tri(j, k)];
                inv[i] = rsqrtf(tmp);
                L[tri(i, i)] = tmp * inv[i];
            } else {
#pragma unroll
                for (int k = 0; k < j; ++k) tmp -= L[tri(i, k)] * L[tri(j, k)];
                L[tri(i, j)] = tmp * inv[j];
            }
        }
    }
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 21; ++i) ok = ok && !isnan(L[i]);
    return ok;
}

// sqrt(w) of a sample weight w > 0 for the moment rows: in FP32 w rsqrt(w) for normal
// w (max 2 ulp; the rows only need r r = w to a few ulp), else the square root
__device__ __forceinline__ float weight_root(float w) {
    if (w >= 1.17549435e-38f) return w * rsqrtf(w);
    return sqrtf(w);
}
__device__ __forceinline__ double weight_root(double w) { return sqrt(w); }

// x / w where one w divides several values (inv = 1 / w): in FP32 the product with the
// reciprocal (within 1.5 ulp of the quotient), in FP64 the correctly rounded quotient.
__device__ __forceinline__ float div_by(float x, float w, float inv) { (void)w; return x * inv; }
__device__ __forceinline__ double div_by(double x, double w, double inv) { (void)inv; return x / w; }

// A map or merge row's 28 leading values (weight, mean[6], packed 6x6[21]) in 16-byte
// pieces; rows start 16-byte aligned (kRow values apart from an aligned base).
__device__ __forceinline__ void row28_load(const float* src, float v[28]) {
    const float4* q = reinterpret_cast<const float4*>(src);
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        const float4 x = q[i];
        v[4 * i] = x.x; v[4 * i + 1] = x.y; v[4 * i + 2] = x.z; v[4 * i + 3] = x.w;
    }
}
__device__ __forceinline__ void row28_load(const double* src, double v[28]) {
    const double2* q = reinterpret_cast<const double2*>(src);
#pragma unroll
    for (int i = 0; i < 14; ++i) {
        const double2 x = q[i];
        v[2 * i] = x.x; v[2 * i + 1] = x.y;
    }
}
__device__ __forceinline__ void row28_store(float* dst, const float v[28]) {
    float4* q = reinterpret_cast<float4*>(dst);
#pragma unroll
    for (int i = 0; i < 7; ++i) q[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
}
__device__ __forceinline__ void row28_store(double* dst, const double v[28]) {
    double2* q = reinterpret_cast<double2*>(dst);
#pragma unroll
    for (int i = 0; i < 14; ++i) q[i] = make_double2(v[2 * i], v[2 * i + 1]);
}

// PD test of an update's posterior covariance: a Cholesky whose every pivot exceeds
// 1e-10 of its diagonal entry.  Unlike the reference's isPosDef (no NaN in the factor),
// an exactly singular posterior -- after a refit from fewer in-view samples than
// dimensions -- is classed not PD instead of by the sign of a rounding error.
template <typename T>
__device__ inline bool posterior_pd(const T* A) {
    T L[21];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            T tmp = A[tri(i, j)];
            if (i == j) {
#pragma unroll
                for (int k = 0; k < j; ++k) tmp -= L[tri(j, k)] * L[tri(j, k)];
                if (!(tmp > T(1e-10) * A[tri(i, i)])) return false;
                L[tri(i, i)] = tsqrt(tmp);
            } else {
#pragma unroll
                for (int k = 0; k < j; ++k) tmp -= L[tri(i, k)] * L[tri(j, k)];
                L[tri(i, j)] = tmp / L[tri(j, j)];
            }
        }
    }
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 21; ++i) ok = ok && !isnan(L[i]);
    return ok;
}

// FP32 form of the same test: one rsqrt per pivot, the column scaled by it (max 2 ulp).
// An exactly singular posterior leaves FP32 rounding residues of about 1e-7 of the
// diagonal in its pivots (FP64: about 1e-16), which would pass a 1e-10 test; the FP32
// test therefore asks for 1e-5 of the diagonal, so that such posteriors are classed not
// PD as in FP64.
template <>
__device__ inline bool posterior_pd<float>(const float* A) {
    float L[21], inv[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            float tmp = A[tri(i, j)];
            if (i == j) {
#pragma unroll
                for (int k = 0; k < j; ++k) tmp -= L[tri(j, k)] * L[tri(j, k)];
                if (!(tmp > 1e-5f * A[tri(i, i)])) return false;
                inv[i] = rsqrtf(tmp);
                L[tri(i, i)] = tmp * inv[i];
            } else {
#pragma unroll
                for (int k = 0; k < j; ++k) tmp -= L[tri(i, k)] * L[tri(j, k)];
                L[tri(i, j)] = tmp * inv[j];
            }
        }
    }
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 21; ++i) ok = ok && !isnan(L[i]);
    return ok;
}

// squared Mahalanobis distance of computeMahalDist<6,36> (src/device_math.cu:374-454):
// Cholesky of (Sa + Sb), triangular inverse (:153-175), sum_i (sum_{j<=i} dj Linv_ij)^2
template <typename T>
__device__ inline T mahal6(const T* ma, const T* Sa, const T* mb, const T* Sb) {
    T S[21], L[21], Li[21], dlt[6];
#pragma unroll
    for (int i = 0; i < 21; ++i) S[i] = Sa[i] + Sb[i];
#pragma unroll
    for (int i = 0; i < 6; ++i) dlt[i] = ma[i] - mb[i];
    chol6(S, L);
#pragma unroll
    for (int col = 0; col < 6; ++col) {
#pragma unroll
        for (int i = col; i < 6; ++i) {
            T val = (i == col) ? T(1) : T(0);
#pragma unroll
            for (int j = col; j < i; ++j) val -= L[tri(i, j)] * Li[tri(j, col)];
            Li[tri(i, col)] = val / L[tri(i, i)];
        }
    }
    T dist = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        T s = 0;
#pragma unroll
        for (int j = 0; j <= i; ++j) s += dlt[j] * Li[tri(i, j)];
        dist += s * s;
    }
    return dist;
}

// FP32 form of the same distance: each pivot's reciprocal square root is taken once
// and the factor, its inverse and the distance use multiplications (hardware rsqrt,
// max 2 ulp), in the same summation order.  The FP64 form keeps the divisions.
template <>
__device__ inline float mahal6<float>(const float* ma, const float* Sa, const float* mb, const float* Sb) {
    float S[21], L[21], Li[21], dlt[6], inv[6];
#pragma unroll
    for (int i = 0; i < 21; ++i) S[i] = Sa[i] + Sb[i];
#pragma unroll
    for (int i = 0; i < 6; ++i) dlt[i] = ma[i] - mb[i];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            float tmp = S[tri(i, j)];
            if (i == j) {
#pragma unroll
                for (int k = 0; k < j; ++k) tmp -= L[tri(j, k)] * L[tri(j, k)];
                inv[i] = rsqrtf(tmp);
                L[tri(i, i)] = tmp * inv[i];
            } else {
#pragma unroll
                for (int k = 0; k < j; ++k) tmp -= L[tri(i, k)] * L[tri(j, k)];
                L[tri(i, j)] = tmp * inv[j];
            }
        }
    }
#pragma unroll
    for (int col = 0; col < 6; ++col) {
#pragma unroll
        for (int i = col; i < 6; ++i) {
            float val = (i == col) ? 1.0f : 0.0f;
#pragma unroll
            for (int j = col; j < i; ++j) val -= L[tri(i, j)] * Li[tri(j, col)];
            Li[tri(i, col)] = val * inv[i];
        }
    }
    float dist = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        float s = 0;
#pragma unroll
        for (int j = 0; j <= i; ++j) s += dlt[j] * Li[tri(i, j)];
        dist += s * s;
    }
    return dist;
}

// Measurement-independent Kalman terms of one fitted Gaussian, computed by one thread:
// S = H P H' + R, S^-1, the log-constant log pD + log w - k/2 log 2pi - 1/2 log|S|,
// the gain K = P H' S^-1 and the Joseph-form posterior covariance
// P - K(HP) - (HP)'K' + K(HPH')K' + K R K' (src/kernels.cu:506-595), then the
// posterior's PD test (isPosDef, src/device_math.cu:800-812).  P is the fitted
// packed covariance, Pn scratch for the posterior (21 values); dst receives [0]
// log-constant, [1] PD flag, [2..7] S^-1 packed, [8..25] K (6 x 3 row-major),
// [26..46] posterior covariance packed.
template <typename T, int K>
__device__ inline void kalman_prep(T w, T pdbar, const T* P, const Model& m, T* Pn, T* dst) {
    T S[6], Si[6];
    S[0] = P[0] + (T)m.var[0];
    S[1] = P[1];
    S[2] = P[2] + (T)m.var[1];
    T det;
    if (K == 2) {
        det = S[0] * S[2] - S[1] * S[1];
        const T idet = T(1) / det;
        Si[0] = div_by(S[2], det, idet); Si[1] = div_by(-S[1], det, idet); Si[2] = div_by(S[0], det, idet);
        Si[3] = Si[4] = Si[5] = 0;
    } else {
        S[3] = P[3]; S[4] = P[4]; S[5] = P[5] + (T)m.var[2];
        T a = S[0], b = S[1], c = S[2], d = S[3], e = S[4], f = S[5];
        T A00 = c * f - e * e, A10 = d * e - b * f, A11 = a * f - d * d;
        T A20 = b * e - c * d, A21 = b * d - a * e, A22 = a * c - b * b;
        det = a * A00 + b * A10 + d * A20;
        const T idet = T(1) / det;
        Si[0] = div_by(A00, det, idet); Si[1] = div_by(A10, det, idet); Si[2] = div_by(A11, det, idet);
        Si[3] = div_by(A20, det, idet); Si[4] = div_by(A21, det, idet); Si[5] = div_by(A22, det, idet);
    }
    const T log2pi = (T)1.8378770664093454835606594728112;
    T cst;
    if (pdbar > T(0) && w > T(0) && det > T(0))
        cst = tlog(pdbar) + tlog(w) - T(0.5) * T(K) * log2pi - T(0.5) * tlog(det);
    else
        cst = tneg_inf<T>();
    // gain entry q = r*3 + cc: K[r][cc] = sum_a P[r][a] S^-1[a][cc]
    T Kg[18];
#pragma unroll
    for (int q = 0; q < 18; ++q) {
        const int r = q / 3, cc = q % 3;
        T acc = 0;
        if (cc < K) {
#pragma unroll
            for (int a = 0; a < K; ++a) acc += P[tri(r, a)] * Si[tri(a, cc)];
        }
        Kg[q] = acc;
        dst[kPrepK + q] = acc;
    }
    // Joseph form with the shared products hoisted: with A = P H' (A_bk = P[b][k]) and
    // Q = K S (Q_bk = sum_l K_bl S_lk, S = H P H' + R), the entry (ea, eb), ea >= eb, of
    // (I - K H) P (I - K H)' + K R K' is P_ab - sum_k K_ak A_bk - sum_k A_ak K_bk
    // + sum_k K_ak Q_bk (the last sum is (K (H P H' + R) K')_ab).
    T Q[18];
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            T acc = 0;
            if (k < K) {
#pragma unroll
                for (int l = 0; l < K; ++l) acc += Kg[r * 3 + l] * (l == k ? S[tri(l, k)] : P[tri(l, k)]);
            }
            Q[r * 3 + k] = acc;
        }
#pragma unroll
    for (int ea = 0; ea < 6; ++ea)
#pragma unroll
    for (int eb = 0; eb <= ea; ++eb) {
        const int e = tri(ea, eb);
        T sv = P[e];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const T Kak = Kg[ea * 3 + k], Kbk = Kg[eb * 3 + k];
            sv -= Kak * P[tri(k, eb)];
            sv -= P[tri(ea, k)] * Kbk;
            sv += Kak * Q[eb * 3 + k];
        }
        Pn[e] = sv;
        dst[kPrepCov + e] = sv;
    }
    const bool pdok = posterior_pd(Pn);
    dst[0] = cst;
    dst[1] = pdok ? T(1) : T(0);
#pragma unroll
    for (int q = 0; q < 6; ++q) dst[kPrepSi + q] = Si[q];
}

// log-likelihood exponent term c - 1/2 nu' S^-1 nu for measurement z
template <typename T, int K>
__device__ __forceinline__ T log_term(T c, const T* Si, const T* mu, const T* z) {
    T n0 = z[0] - mu[0], n1 = z[1] - mu[1];
    T q;
    if (K == 2) {
        q = Si[0] * n0 * n0 + T(2) * Si[1] * n0 * n1 + Si[2] * n1 * n1;
    } else {
        T n2 = z[2] - mu[2];
        q = Si[0] * n0 * n0 + Si[2] * n1 * n1 + Si[5] * n2 * n2 +
            T(2) * (Si[1] * n0 * n1 + Si[3] * n0 * n2 + Si[4] * n1 * n2);
    }
    return c - T(0.5) * q;
}

// FP32 likelihood terms in base 2: with c2 = log2(e) c and A = S^-1 scaled by -log2(e)/2
// on the diagonal and -log2(e) off it (packed as S^-1), log2 of a pair's term is
// c2 + sum_a n_a (sum_{b >= a} A_ab n_b), n = z - mean: nine multiply-adds for K = 3
template <int K>
__device__ __forceinline__ float log2_term(float c2, const float* A, const float* mu, const float* z) {
    const float n0 = z[0] - mu[0], n1 = z[1] - mu[1];
    if (K == 2) {
        const float u0 = fmaf(A[1], n1, A[0] * n0);
        return fmaf(n1, A[2] * n1, fmaf(n0, u0, c2));
    }
    const float n2 = z[2] - mu[2];
    const float u0 = fmaf(A[3], n2, fmaf(A[1], n1, A[0] * n0));
    const float u1 = fmaf(A[4], n2, A[2] * n1);
    return fmaf(n2, A[5] * n2, fmaf(n1, u1, fmaf(n0, u0, c2)));
}
constexpr float kLog2e = 1.4426950408889634f, kLn2 = 0.6931471805599453f;
// 2^x by the hardware approximation (max 2 ulp; 0 below the normal range)
__device__ __forceinline__ float exp2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

}  // namespace scphd

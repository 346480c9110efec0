// scphd_kernels.cuh — sm_100a kernels of one SC-PHD filter step.
//
// Frame data flow (cur = parity of the map/cloud buffers holding the prior map):
//   k_predict_parents   (a) parent CV motion with noise, FP64            [N threads]
//   k_cloud_fit         (b) per daughter Gaussian, one warp: regenerate (merged
//                           components) or load (non-detection clouds) the sample
//                           cloud, apply the pending feature prediction, transform
//                           world->disparity, pD per sample, refit mean/cov, write
//                           the candidate non-detection cloud            [N CTAs]
//   k_prep              (c0) per fitted Gaussian: measurement-independent Kalman
//                           terms (S^-1, log-constant, gain, posterior, PD flag) [N x 128]
//   k_likelihood        (c) per (parent, measurement): log-sum-exp over the
//                           parent's Gaussians (the normaliser), then survivors
//                           (w >= min_weight and PD) compacted per parent [N x M/128]
//   k_merge             (d) per parent: survivors sorted by the reference's argmax
//                           order, greedy merge, new map = merged + non-detection
//                           clouds, parent log-likelihood               [N CTAs]
//   k_weights           FP64 log-domain parent weight update + N_eff   [1 CTA]
//   k_resample          (e) FP64 block scan + systematic resampling     [1 CTA]
#pragma once

#include "scphd_device.cuh"

namespace scphd {

struct Params {
    int N, P, Ps, Gcap, Mcap, Scap, K;
    Model model;
    ModelF model_f;   // model's transform constants in FP32
    double kappa, ps, min_weight, min_sep, min_neff;
    double w0, d0, vu0, vv0, vd0, var_d0, var_vu0, var_vv0, var_vd0;
    double cam_std[6], feat_std[3];
    double prior_a[12], prior_b[12];
    uint32_t key0, key1;
    uint32_t rk[20];   // Philox round keys (key0 + r C0, key1 + r C1), precomputed on the host
};

// the model constants a kernel in T reads: the FP32 copy, or the FP64 original
template <typename T> struct ModelOf;
template <> struct ModelOf<float> {
    __device__ static const ModelF& get(const Params& prm) { return prm.model_f; }
    __device__ static float feat_std(const Params& prm, int q) { return prm.model_f.feat_std[q]; }
};
template <> struct ModelOf<double> {
    __device__ static const Model& get(const Params& prm) { return prm.model; }
    __device__ static double feat_std(const Params& prm, int q) { return prm.feat_std[q]; }
};

template <typename T> struct Bufs {
    double* ext;        // N x 12 parent states
    double* ext_tmp;    // N x 12
    double* lw;         // N log-weights
    int* src;           // N: map row that parent p reads
    int* src_tmp;       // N
    T* map[2];          // N*Gcap rows of kRow: weight, mean, packed cov
    int* map_ref[2];    // N*Gcap: >= 0 cloud row; < 0: merged component with sample key -1-ref
    int* map_n[2];      // N map sizes (by row)
    double* map_ext[2]; // N x 12: extrinsic the merged components are sampled with
    T* cloud[2];        // N*Gcap clouds of 7 x Ps (x,y,z,vx,vy,vz,omega)
    T* fit;             // N*Gcap rows of kRow
    T* prep;            // N*Gcap rows of kPrep (gain and posterior, read by the merge)
    T* lik;             // N*Gcap rows of kLikTerms (the likelihood's per-Gaussian terms)
    T* z;               // Mcap x 3 measurements
    T* ell;             // N x Mcap normalisers
    int* surv_r;        // N x Scap survivor ranks
    T* surv_w;          // N x Scap survivor weights
    int* surv_n;        // N
    int* mlist;         // N x Scap: centre index of each merged component, in output order
    T* mtmp;            // N x Scap rows of kRow (merge output indexed by centre)
    int* merged_n;      // N
    double* loglik;     // N
    double* cum;        // N resampling prefix
    double* scal;       // [0] neff
    int* flags;         // [0] resampled
    int* resample_idx;  // N
    unsigned long long* counters;   // 16
    int* fit_n;         // N: Gaussians the last update fitted (prior map size)
};

// Per-filter arguments of one frame's kernels.
struct FrameArgs {
    int cur, M, fixed, has_pred;
    double dt;
    uint32_t pred_frame, sample_frame, frame;
    const double* zu;   // this frame's measurements (FP64, device; zd unused in (u,v) mode)
    const double* zv;
    const double* zd;
};

// Up to kBatchSlots filters of a batch per launch: their constants and buffers as
// one kernel parameter (read-only parameter space, like a single filter's Params;
// 32 x 824 bytes fits the 32 KB parameter limit).  Each frame's per-filter
// arguments are a separate FrameArgs array in global memory.
constexpr int kBatchSlots = 32;
template <typename T> struct SlotTable {
    Params prm[kBatchSlots];
    Bufs<T> b[kBatchSlots];
};
// kernel parameters are limited to 32764 bytes: the table plus two pointers must fit
static_assert(sizeof(SlotTable<double>) + 64 <= 32764, "batch parameter table exceeds the kernel parameter limit");

__device__ __forceinline__ uint32_t tie_key(uint32_t r) {
    // argmax order of phdUpdateMergeKernel (src/kernels.cu:704-739) on equal weights:
    // earliest index within a thread's stride, then bit-reversed thread slot.
    return (__brev(r & 255u) >> 24) << 24 | (r >> 8);
}

// ---------------------------------------------------------------- (prior)
__global__ void k_prior(Params prm, double* ext, double* lw) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= prm.N) return;
    double u[12];
    for (int b = 0; b < 3; ++b) {
        uint32_t w[4];
        philox(0, 0, (uint32_t)p, ctr_word3(0, ST_PRIOR, b), prm.key0, prm.key1, w);
        for (int q = 0; q < 4; ++q) u[4 * b + q] = u01(w[q]);
    }
    for (int q = 0; q < 12; ++q) ext[12 * p + q] = u[q] * (prm.prior_b[q] - prm.prior_a[q]) + prm.prior_a[q];
    lw[p] = -log((double)prm.N);
}

// ---------------------------------------------------------------- (a) predict parents
__device__ inline double wrap_angle(double a) {   // src/device_math.cu:308-318
    const double pi = 3.14159265358979323846;
    double r = fmod(a, 2 * pi);
    if (r > pi) r -= 2 * pi;
    else if (r < -pi) r += 2 * pi;
    return r;
}

__device__ __forceinline__ void predict_parents_body(const Params& prm, double* ext, double dt, uint32_t frame,
                                                     int p) {
    if (p >= prm.N) return;
    double z[8];
    for (int b = 0; b < 2; ++b) {
        uint32_t w[4];
        philox(0, 0, (uint32_t)p, ctr_word3(frame, ST_CAM, b), prm.key0, prm.key1, w);
        Normals<double>::four(w, z + 4 * b);
    }
    double* e = ext + 12 * p;
    for (int q = 0; q < 3; ++q) {   // linearcvmotionmodel3d.cuh:28-40
        double ac = prm.cam_std[q] * z[q], aa = prm.cam_std[3 + q] * z[3 + q];
        e[q] = (e[q] + e[q + 3] * dt) + 0.5 * ac * dt * dt;
        e[q + 3] = e[q + 3] + ac * dt;
        e[6 + q] = (e[6 + q] + e[9 + q] * dt) + 0.5 * aa * dt * dt;
        e[9 + q] = e[9 + q] + aa * dt;
    }
    for (int q = 0; q < 3; ++q) e[6 + q] = wrap_angle(e[6 + q]);
}

__global__ void k_predict_parents(__grid_constant__ const Params prm, double* ext, double dt, uint32_t frame) {
    predict_parents_body(prm, ext, dt, frame, blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------- (b) cloud -> fit
// One CTA per parent; each warp takes every eighth of the parent's daughter Gaussians,
// a whole warp per Gaussian, after a shared tail pass per round (the sample layout
// below).  Covers: predict_features + ps (.cu:154-178, 1144-1150),
// worldToDisparityKernel + computePdKernel (kernels.cu:6-47, 82-99), weight by pD
// (.cu:1602-1609), normalizeWeightsKernel + fitGaussiansKernel (kernels.cu:996-1018,
// 102-438) and the non-detection copy (.cu:1290-1420).
//
// Each sample is generated (merged component: drawn from its stored Gaussian with
// the counter-based stream; non-detection cloud: loaded), predicted, transformed,
// and staged in the warp's shared-memory rows with its weight w'_s = omega_s pD_s as
// r d, r and w', where d = y - shift (shift: the Gaussian's first sample, if finite)
// and r = sqrt(w').  The 29 moments are then summed lane by lane, one product of two
// rows each (lane q owns moment q: S0 = sum r r, S2 = sum w' w', S1 = sum r (r d),
// SS = sum (r d)(r d)'), so no per-lane accumulators live through the sample loop.
// With the reference's normalised weights w'_s / S0, mean = shift + S1/S0 and the
// weighted covariance is (SS/S0 - d d') (1 + S2/S0^2), d = S1/S0 (the (W^2 + SS)/W
// normaliser of kernels.cu:196 with W = 1).  Zero-weight samples do not enter the sums
// (they stage zeros).  When S0 = 0 the reference weights every sample by 1; that fit
// matters only when the mean pD is positive (some sample weight omega = 0, possible
// only with pD = 1), and is computed from the raw samples, drawn a second time for
// it.  A non-detection cloud is
// kept only if W (1 - pD_mean) >= min_weight (nd_weight, the merge's test), which needs
// W >= min_weight: clouds with W >= min_weight are written while streaming (with
// evict-first stores: they are read again only next frame) and the new map references
// only the retained ones.  (About 90 % of written clouds pass the prune at plain_c1
// scale; staging the points to write only those costs more than it saves.)

// y = L z + mean, with L (packed lower, 21) and the mean (6) read from the warp's
// shared line in 16-byte pieces, consumed in packed order (row a, column c)
template <typename T, typename V, int W>
__device__ __forceinline__ void ltz_line(const T* line, const T z[6], T y[6]) {
    const V* v = reinterpret_cast<const V*>(line);
    T e[28];
#pragma unroll
    for (int i = 0; i < 28 / W; ++i) {
        const V q = v[i];
        const T* x = reinterpret_cast<const T*>(&q);
#pragma unroll
        for (int h = 0; h < W; ++h) e[i * W + h] = x[h];
    }
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        T s = T(0);
#pragma unroll
        for (int c = 0; c <= a; ++c) s += e[tri(a, c)] * z[c];
        y[a] = s + e[21 + a];
    }
}
__device__ __forceinline__ void ltz_plus_mean(const float* line, const float z[6], float y[6]) {
    ltz_line<float, float4, 4>(line, z, y);
}
__device__ __forceinline__ void ltz_plus_mean(const double* line, const double z[6], double y[6]) {
    ltz_line<double, double2, 2>(line, z, y);
}

// sum over the samples of a[s] b[s], four partial sums over 4-sample pieces read in
// 16 bytes (row starts are 16-byte aligned): first the nt pieces of the tail rows (ta,
// tb), then pieces i0 .. n4-1 of the main rows (a, b) -- the order of one sweep over
// rows holding all samples, so the sums do not depend on where samples were staged
// FP32: the partial sums run in pairs through sm_100's packed multiply-add (fma.rn.f32x2:
// two independent single-precision fused multiply-adds, each rounded as fma.rn.f32), two
// instructions per piece instead of four, with the same results
__device__ __forceinline__ unsigned long long pack_f32x2(float lo, float hi) {
    unsigned long long d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
    return d;
}
__device__ __forceinline__ float moment_sweep(const float* ta, const float* tb, int nt, const float* a,
                                              const float* b, int i0, int n4) {
    unsigned long long s01 = 0ull, s23 = 0ull;   // (s0, s1) and (s2, s3), both +0.0f
    auto piece = [&](const float4 y, const float4 z) {
        asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(s01) : "l"(pack_f32x2(y.x, y.y)), "l"(pack_f32x2(z.x, z.y)));
        asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(s23) : "l"(pack_f32x2(y.z, y.w)), "l"(pack_f32x2(z.z, z.w)));
    };
    for (int i = 0; i < nt; ++i) piece(reinterpret_cast<const float4*>(ta)[i], reinterpret_cast<const float4*>(tb)[i]);
    for (int i = i0; i < n4; ++i) piece(reinterpret_cast<const float4*>(a)[i], reinterpret_cast<const float4*>(b)[i]);
    float s0, s1, s2, s3;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(s0), "=f"(s1) : "l"(s01));
    asm("mov.b64 {%0, %1}, %2;" : "=f"(s2), "=f"(s3) : "l"(s23));
    return (s0 + s1) + (s2 + s3);
}
__device__ __forceinline__ double moment_sweep(const double* ta, const double* tb, int nt, const double* a,
                                               const double* b, int i0, int n4) {
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    auto piece = [&](const double* y, const double* z) {
        const double2 y0 = reinterpret_cast<const double2*>(y)[0], z0 = reinterpret_cast<const double2*>(z)[0];
        const double2 y1 = reinterpret_cast<const double2*>(y)[1], z1 = reinterpret_cast<const double2*>(z)[1];
        s0 += y0.x * z0.x;
        s1 += y0.y * z0.y;
        s2 += y1.x * z1.x;
        s3 += y1.y * z1.y;
    };
    for (int i = 0; i < nt; ++i) piece(ta + 4 * i, tb + 4 * i);
    for (int i = i0; i < n4; ++i) piece(a + 4 * i, b + 4 * i);
    return (s0 + s1) + (s2 + s3);
}

// Sample layout.  A warp takes its Gaussians (j = warp, warp + 8, ...) in rounds of up
// to 8.  With R = P mod 32 in {4, 8, 16} (P = 100: R = 4), samples [0, R) of the
// round's 32 / R Gaussians fill one tail pass (lane = Gaussian * R + sample) and
// samples [R, P) of each Gaussian fill whole warp passes (lane l: R + 32 t + l); with
// any other R every sample is taken in warp passes.  So a pass has no idle lanes when
// P = 32 m + R, and lanes of one pass share a Gaussian (no divergence) outside the
// tail pass.  Staged rows per warp: 8 main rows of sY values (r d[6], r, w' at sample
// index) and a tail block of 9 R values per Gaussian (the same 8 rows of R samples):
// sY puts the eight rows a lane-per-moment sweep reads at one sample index (16-byte
// pieces) in distinct banks, and the 9 R tail stride does the same for the tail
// pass's stores (lanes of distinct Gaussians, same sample).
template <typename T> __host__ __device__ constexpr int stage_stride(int P4) {
    return sizeof(T) == 4 ? ((P4 % 8 == 4) ? P4 : P4 + 4) : P4 + 2;
}
__host__ __device__ constexpr int fit_tail(int P) {
    return (P % 32 == 4 || P % 32 == 8 || P % 32 == 16) ? P % 32 : 0;
}
// stride of a cloud's rows (x, y, z, vx, vy, vz, weight): P rounded up to 32 bytes
template <typename T> __host__ __device__ constexpr int cloud_stride(int P) {
    return sizeof(T) == 4 ? ((P + 7) & ~7) : ((P + 3) & ~3);
}
constexpr int kFitWarps = 8;
constexpr int kFitRound = 8;     // Gaussians per warp and round
constexpr int kStageRows = 8;    // r d[6], r, w'
constexpr int kTailFloats = 288; // 32 / R Gaussians x 9 R per warp
template <typename T> __host__ __device__ inline size_t cloud_fit_smem_bytes(int P) {
    const int P4 = (P + 3) & ~3;
    return (size_t)kFitWarps * (kStageRows * stage_stride<T>(P4) + kTailFloats) * sizeof(T);
}

// PC > 0: the body for exactly PC samples per feature, whose strides, loop bounds and
// tail split are compile-time constants (immediate address offsets instead of
// per-sample index arithmetic); PC == 0: any P.  kFitP is the specialised count (the
// configurations' particles_per_feature); fit_specialised says whether a filter's
// parameters match it.
constexpr int kFitP = 100;
template <typename T> __host__ __device__ inline bool fit_specialised(const Params& prm) {
    return prm.P == kFitP && prm.Ps == cloud_stride<T>(kFitP);
}
template <typename T, int K, int PC = 0>
__device__ __forceinline__ void cloud_fit_body(const Params& prm, const Bufs<T>& b, int cur, int M, int fixed,
                                               int has_pred, double dt, uint32_t pred_frame, uint32_t sample_frame,
                                               const double* zu, const double* zv, const double* zd, int p,
                                               int c, int split, T* s_stage) {
    if (p == 0 && c == 0 && zu != nullptr) {   // this frame's measurements into the T layout (u, v, d)
        for (int mm = threadIdx.x; mm < M; mm += blockDim.x) {
            b.z[mm * 3 + 0] = (T)zu[mm];
            b.z[mm * 3 + 1] = (T)zv[mm];
            b.z[mm * 3 + 2] = (K == 3 && zd) ? (T)zd[mm] : T(0);
        }
    }
    // the parent's Gaussians are shared by the warps of its `split` blocks: block c's
    // warp w takes j = gw, gw + nwp, ... (gw = c * kFitWarps + w, nwp = split * kFitWarps)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gw = c * kFitWarps + warp, nwp = split * kFitWarps;
    const int row = b.src[p];
    const int G = min(b.map_n[cur][row], prm.Gcap);
    const int P = PC > 0 ? PC : prm.P, Ps = PC > 0 ? cloud_stride<T>(PC) : prm.Ps;
    const int P4 = (P + 3) & ~3;
    const int sY = stage_stride<T>(P4);
    const int R = fit_tail(P);                      // tail samples per Gaussian (0: no tail pass)
    const int TG = R ? 32 / R : kFitRound;          // Gaussians per round
    T* Y = s_stage + (size_t)warp * kStageRows * sY;                                   // main rows
    T* Yt = s_stage + (size_t)kFitWarps * kStageRows * sY + (size_t)warp * kTailFloats;  // tail blocks
    __shared__ T s_shift[kFitWarps * kFitRound * 6];          // per warp and Gaussian of the round
    __shared__ __align__(16) T s_L[kFitWarps * kFitRound * 28];  // Cholesky factor and mean of merged ones
    __shared__ Pose<T> pose_upd, pose_src;
    __shared__ int s_rd, s_wr;
    // mean pD of a Gaussian with n of its P samples in view, n = 0..P (P <= 256): the
    // value n pD / P in FP64, rounded to T, looked up instead of divided per Gaussian
    __shared__ T s_pbar[257];
    for (int i = threadIdx.x; i <= P; i += blockDim.x) s_pbar[i] = (T)((double)i * prm.model.pd / (double)P);
    // the two poses (FP64 rotation terms) by threads of two warps, side by side
    if (threadIdx.x == 32) pose_src = make_pose<T>(b.map_ext[cur] + 12 * row);
    if (threadIdx.x == 0) {
        double zero[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        pose_upd = make_pose<T>(fixed ? zero : b.ext + 12 * p);
        if (c == 0) {
            b.surv_n[p] = 0;
            atomicAdd(&b.counters[4], (unsigned long long)G * (unsigned long long)M);
            atomicAdd(&b.counters[6], (unsigned long long)G * (unsigned long long)M);
            atomicAdd(&b.counters[10], (unsigned long long)G);
        }
        s_rd = 0;
        s_wr = 0;
    }
    __syncthreads();
    const Model& m = prm.model;
    // the transforms' constants in T (the FP32 copy needs no conversion per use)
    const auto& mt = ModelOf<T>::get(prm);
    const T invP = T(1) / T(P);
    const T dtT = (T)dt, half_dt2 = T(0.5) * (T)dt * (T)dt;
    const T min_w = (T)prm.min_weight;
    T* shw = s_shift + warp * kFitRound * 6;
    T* Lw = s_L + warp * kFitRound * 28;
    // moment owned by this lane: rows (ra, rb) of the product Y[ra] * Y[rb]: lane 0
    // S0 = sum r r, lane 1 S2 = sum w' w', lanes 2-7 S1 = sum r (r d), lanes 8-28 SS
    int ra = 6, rb = 6;
    if (lane == 1) ra = rb = 7;
    else if (lane >= 2 && lane < 8) rb = lane - 2;
    else if (lane >= 8 && lane < 29) {
        int e = lane - 8, aa = 0;
        while ((aa + 1) * (aa + 2) / 2 <= e) ++aa;
        ra = aa;
        rb = e - aa * (aa + 1) / 2;
    }
    // one sample s of Gaussian j (entry ref, factor line Lg): the predicted particle X,
    // its measurement y; returns the sample weight omega (1/P for a drawn sample)
    auto sample = [&](int ref, int j, int s, const T* Lg, T (&X)[6], T (&y)[6]) -> T {
        T om;
        if (ref < 0) {   // merged component: draw (.cu:640-690) and map to world (.cu:1222-1286)
            const uint32_t key_i = (uint32_t)(-1 - ref);
            uint32_t w0[4], w1[4];
            philox_rk((uint32_t)s, key_i, (uint32_t)row, ctr_word3(sample_frame, ST_SAMPLE, 0), prm.rk, w0);
            philox_rk((uint32_t)s, key_i, (uint32_t)row, ctr_word3(sample_frame, ST_SAMPLE, 1), prm.rk, w1);
            T z[6];
            Pair<T>::two(w0[0], w0[1], z[0], z[1]);
            Pair<T>::two(w0[2], w0[3], z[2], z[3]);
            Pair<T>::two(w1[0], w1[1], z[4], z[5]);
            T yy[6];
            ltz_plus_mean(Lg, z, yy);   // y = L z + mean
            invert(yy, pose_src, mt, X);
            om = invP;
        } else {         // non-detection cloud carried from the previous frame
            // the previous frame's clouds are only read in this kernel (writes go to
            // the other buffer): read-only loads, free to move ahead of the stores
            const T* cl_in = b.cloud[cur] + (size_t)ref * 7 * Ps;
#pragma unroll
            for (int a2 = 0; a2 < 6; ++a2) X[a2] = __ldg(cl_in + a2 * Ps + s);
            om = __ldg(cl_in + 6 * Ps + s);
        }
        if (has_pred) {   // predict_features with feature noise
            uint32_t w[4];
            philox_rk((uint32_t)s, (uint32_t)j, (uint32_t)p, ctr_word3(pred_frame, ST_FEAT, 0), prm.rk, w);
            T z[4];
            Pair<T>::two(w[0], w[1], z[0], z[1]);
            Pair<T>::two(w[2], w[3], z[2], z[3]);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                T a2 = ModelOf<T>::feat_std(prm, q) * z[q];
                X[q] = X[q] + X[q + 3] * dtT + a2 * half_dt2;
                X[q + 3] = X[q + 3] + a2 * dtT;
            }
        }
        measure(X, pose_upd, mt, y);
        return om;
    };
    // the non-detection cloud candidate: predicted world point, weight 1 - pD
    auto write_nd = [&](int j, int s, const T (&X)[6], T pds) {
        T* cl_out = b.cloud[cur ^ 1] + ((size_t)p * prm.Gcap + j) * 7 * Ps;
#pragma unroll
        for (int a2 = 0; a2 < 6; ++a2) __stcs(cl_out + a2 * Ps + s, X[a2]);
        __stcs(cl_out + 6 * Ps + s, T(1) - pds);
    };
    // staged moment rows of one sample (zero-weight samples and the padding stage zeros)
    auto stage = [&](T* Ys, int stride, const T (&y)[6], const T (&shift)[6], T wp) {
        const T r = wp != T(0) ? weight_root(wp) : T(0);
#pragma unroll
        for (int a2 = 0; a2 < 6; ++a2) Ys[a2 * stride] = wp != T(0) ? r * (y[a2] - shift[a2]) : T(0);
        Ys[6 * stride] = r;
        Ys[7 * stride] = wp;
    };
    const int nW = G > gw ? (G - gw + nwp - 1) / nwp : 0;   // this warp's Gaussians
    for (int k0 = 0; k0 < nW; k0 += TG) {
        const int nR = min(TG, nW - k0);
        // lane k < nR: entry of the round's Gaussian k
        int my_ref = 0;
        T my_W = T(0);
        if (lane < nR) {
            const size_t erow = (size_t)row * prm.Gcap + gw + nwp * (k0 + lane);
            my_ref = b.map_ref[cur][erow];
            my_W = has_pred ? b.map[cur][erow * kRow] * (T)prm.ps : b.map[cur][erow * kRow];
        }
        const unsigned merged = __ballot_sync(0xffffffffu, lane < nR && my_ref < 0);
        const unsigned writes = __ballot_sync(0xffffffffu, lane < nR && my_W >= min_w);
        if (lane == 0) {
            atomicAdd(&s_rd, nR - __popc(merged));
            atomicAdd(&s_wr, __popc(writes));
        }
        // Cholesky factor (21, stored in the map row) and mean (6) of the round's merged
        // Gaussians: every load issued before the first store (the previous frame's map
        // is only read in this kernel), lane e holding element e of each
        T lv[kFitRound];
#pragma unroll
        for (int k = 0; k < kFitRound; ++k) {
            lv[k] = T(0);
            if ((merged >> k) & 1u) {
                const T* ent = b.map[cur] + ((size_t)row * prm.Gcap + gw + nwp * (k0 + k)) * kRow;
                if (lane < 21) lv[k] = __ldg(ent + 7 + lane);
                else if (lane < 27) lv[k] = __ldg(ent + 1 + lane - 21);
            }
        }
#pragma unroll
        for (int k = 0; k < kFitRound; ++k)
            if (((merged >> k) & 1u) && lane < 28) Lw[k * 28 + lane] = lv[k];
        __syncwarp();
        // tail pass: samples [0, R) of the round's Gaussians; lane gi * R (sample 0)
        // gives its Gaussian's shift
        int t_in = 0;
        bool t_any = false;
        if (R) {
            const int gi = lane / R, s = lane - gi * R;
            const bool valid = gi < nR;
            const int ref = __shfl_sync(0xffffffffu, my_ref, gi & 31);
            const bool wnd = __shfl_sync(0xffffffffu, my_W, gi & 31) >= min_w;
            const int j = gw + nwp * (k0 + gi);
            T X[6], y[6], om = 0;
            if (valid) {
                om = sample(ref, j, s, Lw + gi * 28, X, y);
            } else {
#pragma unroll
                for (int a2 = 0; a2 < 6; ++a2) { X[a2] = 0; y[a2] = 0; }
            }
            const bool inr = valid && in_range(y, mt);
            const T pds = inr ? (T)mt.pd : T(0);
            if (valid && wnd) write_nd(j, s, X, pds);
            const T wp = om * pds;
            T shift[6];
#pragma unroll
            for (int a2 = 0; a2 < 6; ++a2) {
                const T v = __shfl_sync(0xffffffffu, y[a2], lane - s);
                shift[a2] = isfinite(v) ? v : T(0);
            }
            if (valid && s == 0) {
#pragma unroll
                for (int a2 = 0; a2 < 6; ++a2) shw[gi * 6 + a2] = shift[a2];
            }
            stage(Yt + gi * 9 * R + s, R, y, shift, wp);
            const unsigned gm = (R == 32 ? 0xffffffffu : ((1u << R) - 1u)) << (gi * R & 31);
            t_in = __popc(__ballot_sync(0xffffffffu, inr) & gm);
            t_any = (__ballot_sync(0xffffffffu, wp != T(0)) & gm) != 0u;
        }
        __syncwarp();
        for (int k = 0; k < nR; ++k) {
            const int j = gw + nwp * (k0 + k);
            const int ref = __shfl_sync(0xffffffffu, my_ref, k);
            const T W = __shfl_sync(0xffffffffu, my_W, k);
            const bool wnd = W >= min_w;
            const T* Lg = Lw + k * 28;
            const T* Ytk = Yt + k * 9 * R;
            T shift[6];
            if (R) {
#pragma unroll
                for (int a2 = 0; a2 < 6; ++a2) shift[a2] = shw[k * 6 + a2];
            }
            int n_in = R ? __shfl_sync(0xffffffffu, t_in, (k * R) & 31) : 0;
            bool any = R ? __shfl_sync(0xffffffffu, (int)t_any, (k * R) & 31) != 0 : false;
            // warp passes over samples [R, P4): moment rows, non-detection clouds
            for (int s0 = R; s0 < P4; s0 += 32) {
                const int s = s0 + lane;
                const bool valid = s < P;
                T X[6], y[6], om = 0;
                if (valid) {
                    om = sample(ref, j, s, Lg, X, y);
                } else {
#pragma unroll
                    for (int a2 = 0; a2 < 6; ++a2) { X[a2] = 0; y[a2] = 0; }
                }
                const bool inr = valid && in_range(y, mt);
                const T pds = inr ? (T)mt.pd : T(0);
                n_in += __popc(__ballot_sync(0xffffffffu, inr));
                if (valid && wnd) write_nd(j, s, X, pds);
                const T wp = om * pds;
                any |= __any_sync(0xffffffffu, wp != T(0));
                if (!R && s0 == 0) {   // shift: the Gaussian's first sample, if finite, else 0
#pragma unroll
                    for (int a2 = 0; a2 < 6; ++a2) {
                        const T v = __shfl_sync(0xffffffffu, y[a2], 0);
                        shift[a2] = isfinite(v) ? v : T(0);
                    }
                    if (lane < 6) {   // static indices: the shift stays in registers
#pragma unroll
                        for (int a2 = 0; a2 < 6; ++a2)
                            if (lane == a2) shw[k * 6 + a2] = shift[a2];
                    }
                }
                if (s < P4) stage(Y + s, sY, y, shift, wp);
            }
            const T pbar = s_pbar[n_in];
            const bool raw = !any && n_in > 0 && m.pd > 0.0;
            if (raw) {
                // the fallback fit (below) needs the raw samples: rare, so they are drawn
                // again, every sample in warp passes, y itself staged in the main rows
                __syncwarp();
                for (int s0 = 0; s0 < P4; s0 += 32) {
                    const int s = s0 + lane;
                    T X[6], y[6];
                    if (s < P) {
                        sample(ref, j, s, Lg, X, y);
                    } else {
#pragma unroll
                        for (int a2 = 0; a2 < 6; ++a2) y[a2] = 0;
                    }
                    if (s < P4) {
#pragma unroll
                        for (int a2 = 0; a2 < 6; ++a2) Y[a2 * sY + s] = y[a2];
                    }
                }
            }
            __syncwarp();
            const T* sh = shw + k * 6;
            // fitted row element `lane` (W, pD, mean[6], packed cov[21]), written from registers
            T fv = lane == 0 ? W : pbar;
            if (any) {
                // lane q < 29: moment q over the samples, four partial sums
                const T mom = lane < 29 ? moment_sweep(Ytk + ra * R, Ytk + rb * R, R / 4, Y + ra * sY, Y + rb * sY,
                                                       R / 4, P4 / 4)
                                        : T(0);
                const T S0 = __shfl_sync(0xffffffffu, mom, 0), S2 = __shfl_sync(0xffffffffu, mom, 1);
                const T inv = T(1) / S0, scale = T(1) + S2 * inv * inv;
                // lanes 2-7 hold S1 (the mean offsets), lanes 8-28 hold SS
                const T dl = (lane >= 2 && lane < 8) ? mom * inv : T(0);
                T da = 0, db = 0;
                T dvals[6];
#pragma unroll
                for (int a2 = 0; a2 < 6; ++a2) dvals[a2] = __shfl_sync(0xffffffffu, dl, 2 + a2);
#pragma unroll
                for (int a2 = 0; a2 < 6; ++a2) {
                    if (ra == a2) da = dvals[a2];
                    if (rb == a2) db = dvals[a2];
                }
                if (lane >= 2 && lane < 8) fv = sh[lane - 2] + dl;
                if (lane >= 8) fv = (mom * inv - da * db) * scale;
            } else if (pbar > T(0)) {
                // every sample weighted 1 (exp(LOG0 - LOG0)): unnormalised mean (sum of the
                // samples) and covariance x (P + P)/P over the valid samples (raw rows)
                T mu = 0;
                if (lane < 6) {
                    for (int s = 0; s < P; ++s) mu += Y[lane * sY + s];
                }
                T mus[6];
#pragma unroll
                for (int a2 = 0; a2 < 6; ++a2) mus[a2] = __shfl_sync(0xffffffffu, mu, a2);
                T cva = 0;
                if (lane >= 8 && lane < 29) {
                    T ma = 0, mb = 0;
#pragma unroll
                    for (int a2 = 0; a2 < 6; ++a2) {
                        if (ra == a2) ma = mus[a2];
                        if (rb == a2) mb = mus[a2];
                    }
                    for (int s = 0; s < P; ++s) cva += (Y[ra * sY + s] - ma) * (Y[rb * sY + s] - mb);
                }
                const T scale = (T(P) * T(P) + T(P)) / T(P);
                const T mu_e = __shfl_sync(0xffffffffu, mu, (lane - 2) & 31);   // mean element lane - 2
                if (lane >= 2 && lane < 8) fv = mu_e;
                if (lane >= 8) fv = cva * scale;
                if (lane == 0) atomicAdd(&b.counters[14], 1ull);
            } else {   // entirely out of view: never used downstream (its log-constant is -inf)
                if (lane >= 2 && lane < 8) fv = sh[lane - 2];
                if (lane >= 8) fv = T(0);
            }
            T* fr = b.fit + ((size_t)p * prm.Gcap + j) * kRow;
            if (lane < 29) fr[lane] = fv;
            __syncwarp();   // the sweep's reads of the rows end before the next Gaussian's staging
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd(&b.counters[8], (unsigned long long)s_rd);
        atomicAdd(&b.counters[9], (unsigned long long)s_wr);
    }
}


// grid: `split` blocks per parent (block x: parent x / split, part x % split)
template <typename T, int K, int PC = 0>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2)
    k_cloud_fit(__grid_constant__ const Params prm, __grid_constant__ const Bufs<T> b, int cur, int M, int fixed,
                int has_pred, double dt, uint32_t pred_frame, uint32_t sample_frame, const double* zu,
                const double* zv, const double* zd, int split) {
    extern __shared__ __align__(16) unsigned char dsm_fit[];
    const int p = blockIdx.x / split;
    cloud_fit_body<T, K, PC>(prm, b, cur, M, fixed, has_pred, dt, pred_frame, sample_frame, zu, zv, zd, p,
                             blockIdx.x - p * split, split, reinterpret_cast<T*>(dsm_fit));
}

template <typename T, int K, int PC = 0>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2)
    k_cloud_fit_batch(const __grid_constant__ SlotTable<T> tab, const FrameArgs* fas, const int2* map, int split) {
    extern __shared__ __align__(16) unsigned char dsm_fit[];
    const int q = blockIdx.x / split;
    const int2 fp = map[q];
    const FrameArgs fa = fas[fp.x];
    cloud_fit_body<T, K, PC>(tab.prm[fp.x], tab.b[fp.x], fa.cur, fa.M, fa.fixed, fa.has_pred, fa.dt, fa.pred_frame,
                             fa.sample_frame, fa.zu, fa.zv, fa.zd, fp.y, blockIdx.x - q * split, split,
                             reinterpret_cast<T*>(dsm_fit));
}

// ---------------------------------------------------------------- (c0) Kalman terms
// Measurement-independent Kalman terms of every fitted Gaussian (kalman_prep: S, S^-1,
// log-constant, gain, Joseph posterior and its PD test; src/kernels.cu:506-598), one
// thread per Gaussian, in a launch of its own between the cloud fit and the likelihood
// (each thread runs one long dependent chain; here the warps of many parents hide each
// other's latency).  Each thread reads its fitted row in 16-byte pieces and writes its
// rows into shared memory (odd strides: no bank conflicts); the block then copies the
// rows of its Gaussians -- contiguous in global memory -- out with coalesced stores:
//   prep row (kPrep): the gain and posterior covariance the merge reads per survivor;
//   likelihood row (kLikTerms): log-constant (-inf when the posterior is not PD), PD
//   flag, packed S^-1, mean (u, v, d) -- the k_likelihood terms, read in 16-byte pieces;
//   in FP32 in base 2 (log2(e) c, S^-1 scaled for log2_term).
constexpr int kLikTerms = 12;   // log-constant, PD flag, S^-1 (6), mean (3), pad: 16-byte pieces
constexpr int kPrepThreads = 128;
constexpr int kPrepStride = kPrep + 1, kLikStride = kLikTerms + 1;
template <typename T> __host__ __device__ inline size_t prep_smem_bytes() {
    return (size_t)kPrepThreads * (kPrepStride + kLikStride) * sizeof(T);
}

__device__ __forceinline__ void load_row29(const float* fr, float v[29]) {   // fitted row: 16-byte pieces
    const float4* q = reinterpret_cast<const float4*>(fr);
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        const float4 x = q[i];
        v[4 * i] = x.x; v[4 * i + 1] = x.y; v[4 * i + 2] = x.z; v[4 * i + 3] = x.w;
    }
    v[28] = fr[28];
}
__device__ __forceinline__ void load_row29(const double* fr, double v[29]) {
    const double2* q = reinterpret_cast<const double2*>(fr);
#pragma unroll
    for (int i = 0; i < 14; ++i) {
        const double2 x = q[i];
        v[2 * i] = x.x; v[2 * i + 1] = x.y;
    }
    v[28] = fr[28];
}

template <typename T, int K>
__device__ __forceinline__ void prep_body(const Params& prm, const Bufs<T>& b, int cur, int p, T* smem) {
    const int G = min(b.map_n[cur][b.src[p]], prm.Gcap);
    T* s_prep = smem;                                     // kPrepThreads rows of kPrepStride
    T* s_lik = smem + (size_t)kPrepThreads * kPrepStride;  // kPrepThreads rows of kLikStride
    for (int j0 = 0; j0 < G; j0 += kPrepThreads) {
        const int n = min(kPrepThreads, G - j0);
        if ((int)threadIdx.x < n) {
            T v[29];
            load_row29(b.fit + ((size_t)p * prm.Gcap + j0 + threadIdx.x) * kRow, v);
            T Pn[21];
            T* d = s_prep + (size_t)threadIdx.x * kPrepStride;
            kalman_prep<T, K>(v[0], v[1], v + 8, prm.model, Pn, d);
            d[kPrep - 1] = T(0);
            T* l = s_lik + (size_t)threadIdx.x * kLikStride;
            // a non-PD posterior's log-constant is staged as -inf (its weight is LOG0 before
            // the normaliser, kernels.cu:597-598), so the normaliser pass needs no test
            l[0] = (d[0] > tneg_inf<T>() && d[1] != T(0)) ? d[0] : tneg_inf<T>();
            l[1] = d[1];
#pragma unroll
            for (int i = 0; i < 6; ++i) l[2 + i] = d[kPrepSi + i];
            if constexpr (sizeof(T) == 4) {   // base-2 form (log2_term): c2 and the scaled S^-1
                l[0] = l[0] * kLog2e;
#pragma unroll
                for (int i = 0; i < 6; ++i) {
                    const bool diag = K == 3 ? (i == 0 || i == 2 || i == 5) : (i == 0 || i == 2);
                    l[2 + i] = l[2 + i] * (diag ? -0.5f * kLog2e : -kLog2e);
                }
            }
#pragma unroll
            for (int a = 0; a < 3; ++a) l[8 + a] = v[2 + a];
            l[11] = T(0);
        }
        __syncthreads();
        T* gp = b.prep + ((size_t)p * prm.Gcap + j0) * kPrep;
        for (int e = threadIdx.x; e < n * kPrep; e += kPrepThreads) gp[e] = s_prep[(e / kPrep) * kPrepStride + e % kPrep];
        T* gl = b.lik + ((size_t)p * prm.Gcap + j0) * kLikTerms;
        for (int e = threadIdx.x; e < n * kLikTerms; e += kPrepThreads)
            gl[e] = s_lik[(e / kLikTerms) * kLikStride + e % kLikTerms];
        __syncthreads();
    }
}

template <typename T, int K>
__global__ void __launch_bounds__(kPrepThreads) k_prep(__grid_constant__ const Params prm,
                                                       __grid_constant__ const Bufs<T> b, int cur) {
    extern __shared__ __align__(16) unsigned char dsm_prep[];
    prep_body<T, K>(prm, b, cur, blockIdx.x, reinterpret_cast<T*>(dsm_prep));
}

template <typename T, int K>
__global__ void __launch_bounds__(kPrepThreads)
    k_prep_batch(const __grid_constant__ SlotTable<T> tab, const FrameArgs* fas, const int2* map) {
    extern __shared__ __align__(16) unsigned char dsm_prep[];
    const int2 fp = map[blockIdx.x];
    prep_body<T, K>(tab.prm[fp.x], tab.b[fp.x], fas[fp.x].cur, fp.y, reinterpret_cast<T*>(dsm_prep));
}

// ---------------------------------------------------------------- (c) likelihood
// Normaliser ell_{p,m} = logsumexp_j(log w_{j,m}) (+) log(M w0 + kappa)
// (.cu:1729-1768) and survivor compaction: w_{j,m} = exp(log w - ell) >= min_weight
// with a PD posterior (updateKernel, kernels.cu:622-657), births likewise.
// One thread per measurement; a block covers the frame's measurements (a multiple
// of 32 threads, up to 1024; more measurements take more blocks) and stages the
// parent's Gaussian terms once in shared memory for both passes.  Since ell >= bpc =
// log(M w0 + kappa) (the sum inside the log holds exp(0) = 1 around its larger term),
// a pair with log w < bpc + log(min_weight) - 1 can never reach min_weight; the first
// pass remembers the pairs above that bound (up to kLikCand per measurement) and the
// survivor pass evaluates only those (all pairs again if the list overflowed).
constexpr int kLikCand = 16;   // candidate survivors remembered per measurement
template <typename T> __host__ __device__ inline size_t likelihood_smem_bytes(int Gcap, int block) {
    return (size_t)Gcap * kLikTerms * sizeof(T) + (size_t)block * kLikCand * sizeof(int);
}
__host__ __device__ inline int likelihood_block(int M) {
    const int r = (M + 31) / 32 * 32;
    return r < 32 ? 32 : (r > 1024 ? 1024 : r);
}

__device__ __forceinline__ void load_terms(const float* src, float* t) {
    const float4* v = reinterpret_cast<const float4*>(src);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float4 q = v[i];
        t[4 * i] = q.x; t[4 * i + 1] = q.y; t[4 * i + 2] = q.z; t[4 * i + 3] = q.w;
    }
}
__device__ __forceinline__ void load_terms(const double* src, double* t) {
    const double2* v = reinterpret_cast<const double2*>(src);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const double2 q = v[i];
        t[2 * i] = q.x; t[2 * i + 1] = q.y;
    }
}
__device__ __forceinline__ void store_terms(float* dst, const float* t) {
    float4* v = reinterpret_cast<float4*>(dst);
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] = make_float4(t[4 * i], t[4 * i + 1], t[4 * i + 2], t[4 * i + 3]);
}
__device__ __forceinline__ void store_terms(double* dst, const double* t) {
    double2* v = reinterpret_cast<double2*>(dst);
#pragma unroll
    for (int i = 0; i < 6; ++i) v[i] = make_double2(t[2 * i], t[2 * i + 1]);
}

template <typename T, int K>
__device__ __forceinline__ void likelihood_body(const Params& prm, const Bufs<T>& b, int cur, int M, int p,
                                                int mblock, T* s_terms) {
    const int m = mblock * blockDim.x + threadIdx.x;
    const int G = min(b.map_n[cur][b.src[p]], prm.Gcap);
    // per Gaussian: c (-inf for a non-PD posterior), pD flag, S^-1, mean, pad -- the
    // compact rows k_prep wrote, copied into shared memory in 16-byte pieces
    T cm = tneg_inf<T>();
    for (int jj = threadIdx.x; jj < G; jj += blockDim.x) {
        T t[kLikTerms];
        load_terms(b.lik + ((size_t)p * prm.Gcap + jj) * kLikTerms, t);
        cm = t[0] > cm ? t[0] : cm;
        store_terms(s_terms + (size_t)jj * kLikTerms, t);
    }
    T zm[3] = {0, 0, 0};
    if (m < M) {
#pragma unroll
        for (int a2 = 0; a2 < K; ++a2) zm[a2] = b.z[m * 3 + a2];
    }
    // the pair terms' base: log2 in FP32 (log2_term on the rows k_prep scaled), ln in FP64;
    // sc = the factor from ln to that base, ic its inverse
    constexpr bool kB2 = sizeof(T) == 4;
    const T sc = kB2 ? T(kLog2e) : T(1), ic = kB2 ? T(kLn2) : T(1);
    auto pair_term = [&](const T* t) -> T {
        if constexpr (kB2) return log2_term<K>(t[0], t + 2, t + 8, zm);
        else return log_term<T, K>(t[0], t + 2, t + 8, zm);
    };
    auto exp_w = [&](T x) -> T {   // base^x for the normaliser sums and survivor weights
        if constexpr (kB2) return exp2_approx(x);
        else return texp_sum(x);
    };
    const T bpc = (T)log((double)M * prm.w0 + prm.kappa);   // ln of the birth + clutter term
    const T bpc_w = bpc * sc;
    const T cand_min = (bpc + (T)log(prm.min_weight) - T(1)) * sc;
    int* s_cand = reinterpret_cast<int*>(s_terms + (size_t)prm.Gcap * kLikTerms);   // [slot][thread]
    int n_cand = 0;
    // largest log-constant of the parent: lt_j <= c_j, since the quadratic form is >= 0
    __shared__ T s_cm[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T v = __shfl_xor_sync(0xffffffffu, cm, o);
        cm = v > cm ? v : cm;
    }
    if ((threadIdx.x & 31) == 0) s_cm[threadIdx.x >> 5] = cm;
    __syncthreads();
    for (int w2 = 0; w2 < (int)(blockDim.x >> 5); ++w2) cm = s_cm[w2] > cm ? s_cm[w2] : cm;
    // FP32: the sum is taken around the fixed shift s0 = max(c_max, bpc) when no term
    // that matters can underflow there (every term within ~20 of bpc is within 80 of s0);
    // otherwise (a log-constant far above bpc), and always in FP64, by an online
    // log-sum-exp around the running maximum, whose dominant term is exp(0) = 1 exactly:
    // a weight near 1 then rounds as in the FP64 oracle, and the merge order of nearly
    // tied weights with it.  (FP32 values are in base 2 here, the limits scaled alike.)
    const T s0 = cm > bpc_w ? cm : bpc_w;
    const bool fixed_shift = kB2 && !(cm - bpc_w > T(60) * sc);
    T mx = tneg_inf<T>(), acc = 0;
    if (m < M) {
        if (fixed_shift) {
            for (int k = 0; k < G; ++k) {
                T t[kLikTerms];
                load_terms(s_terms + (size_t)k * kLikTerms, t);
                const T lt = pair_term(t);   // -inf for a non-PD posterior
                acc += exp_w(lt - s0);
                if (lt >= cand_min) {
                    if (n_cand < kLikCand) s_cand[n_cand * blockDim.x + threadIdx.x] = k;
                    ++n_cand;
                }
            }
        } else {
            for (int k = 0; k < G; ++k) {
                T t[kLikTerms];
                load_terms(s_terms + (size_t)k * kLikTerms, t);
                const T c = t[0];
                if (!(c > tneg_inf<T>())) continue;
                const T lt = pair_term(t);
                if (lt > mx) { acc = acc * exp_w(mx - lt) + T(1); mx = lt; }   // online log-sum-exp
                else acc += exp_w(lt - mx);
                if (lt >= cand_min) {
                    if (n_cand < kLikCand) s_cand[n_cand * blockDim.x + threadIdx.x] = k;
                    ++n_cand;
                }
            }
        }
    }
    // the normaliser in the working base (ell_w), stored as ln: (sum_j base^lt_j) (+) bpc
    auto log_b = [&](T x) -> T {   // accurate log in the working base
        if constexpr (kB2) return log2f(x);
        else return tlog(x);
    };
    auto exp_b = [&](T x) -> T {   // accurate base^x
        if constexpr (kB2) return exp2f(x);
        else return texp(x);
    };
    T ell_w = bpc_w;
    if (m < M && fixed_shift) {
        ell_w = s0 + log_b(acc + exp_b(bpc_w - s0));
    } else if (m < M && mx > tneg_inf<T>()) {
        // evaluated around the larger of the two
        T big = mx > bpc_w ? mx : bpc_w;
        ell_w = big + log_b(acc * exp_b(mx - big) + exp_b(bpc_w - big));
    }
    const T ell = kB2 ? ell_w * ic : ell_w;
    if (m < M) b.ell[(size_t)p * prm.Mcap + m] = ell;
    // survivors among the candidates (or all pairs, if the list overflowed)
    const T minw = (T)prm.min_weight;
    const unsigned lane = threadIdx.x & 31;
    if (m < M) {
        const bool all = n_cand > kLikCand;
        const int nk = all ? G : n_cand;
        for (int q = 0; q < nk; ++q) {
            const int k = all ? q : s_cand[q * blockDim.x + threadIdx.x];
            T t[kLikTerms];
            load_terms(s_terms + (size_t)k * kLikTerms, t);
            const T c = t[0];
            if (!(c > tneg_inf<T>() && t[1] > T(0))) continue;
            const T w = exp_w(pair_term(t) - ell_w);
            if (w >= minw) {
                const int slot = atomicAdd(&b.surv_n[p], 1);
                if (slot < prm.Scap) {
                    b.surv_r[(size_t)p * prm.Scap + slot] = m * G + k;
                    b.surv_w[(size_t)p * prm.Scap + slot] = w;
                } else {
                    atomicAdd(&b.counters[1], 1ull);
                }
            }
        }
    }
    // birth term of measurement m (always PD)
    bool keep = false;
    T wb = 0;
    if (m < M) {
        wb = texp((T)log(prm.w0) - ell);
        keep = wb >= minw;
    }
    unsigned mask = __ballot_sync(0xffffffffu, keep);
    if (mask) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&b.surv_n[p], __popc(mask));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (keep) {
            int slot = base + __popc(mask & ((1u << lane) - 1u));
            if (slot < prm.Scap) {
                b.surv_r[(size_t)p * prm.Scap + slot] = G * M + m;
                b.surv_w[(size_t)p * prm.Scap + slot] = wb;
            } else {
                atomicAdd(&b.counters[1], 1ull);
            }
        }
    }
}

template <typename T, int K>
__global__ void __launch_bounds__(1024) k_likelihood(__grid_constant__ const Params prm,
                                                     __grid_constant__ const Bufs<T> b, int cur, int M) {
    extern __shared__ __align__(16) unsigned char dsm_lik[];
    likelihood_body<T, K>(prm, b, cur, M, blockIdx.x, blockIdx.y, reinterpret_cast<T*>(dsm_lik));
}

// map entry: (filter, parent, measurement block); blocks past a filter's M exit
template <typename T, int K>
__global__ void __launch_bounds__(1024)
    k_likelihood_batch(const __grid_constant__ SlotTable<T> tab, const FrameArgs* fas, const int4* map) {
    extern __shared__ __align__(16) unsigned char dsm_lik[];
    const int4 e = map[blockIdx.x];
    const int M = fas[e.x].M;
    if (e.z * (int)blockDim.x >= M) return;
    likelihood_body<T, K>(tab.prm[e.x], tab.b[e.x], fas[e.x].cur, M, e.y, e.z, reinterpret_cast<T*>(dsm_lik));
}

// ---------------------------------------------------------------- (d) merge
// Posterior components of one parent (detections and births) by survivor rank r: the
// mean, from the fitted row, the Kalman gain and the measurement (a birth's from the
// birth template); bcov holds the birth covariance, the detections' covariances are
// their Gaussians' posteriors in the prep rows.
template <typename T, int K> struct KalmanSource {
    const T* fit;   // parent's fitted rows
    const T* prep;  // parent's prep rows
    const T* z;     // measurements
    int G, M;
    T bmean[6], bcov[21];   // birth template (mean[0..K) replaced by z)
    __device__ void mean(int r, T mu[6]) const {
        if (r < G * M) {
            int mm = r / G, j = r - mm * G;
            const T* fr = fit + (size_t)j * kRow;
            const T* Kg = prep + (size_t)j * kPrep + kPrepK;
            T nu[3];
#pragma unroll
            for (int a = 0; a < K; ++a) nu[a] = z[mm * 3 + a] - fr[2 + a];
#pragma unroll
            for (int a = 0; a < 6; ++a) {
                T s = fr[2 + a];
#pragma unroll
                for (int c = 0; c < K; ++c) s += nu[c] * Kg[a * 3 + c];
                mu[a] = s;
            }
        } else {
            int mm = r - G * M;
#pragma unroll
            for (int a = 0; a < 6; ++a) mu[a] = bmean[a];
#pragma unroll
            for (int a = 0; a < K; ++a) mu[a] = z[mm * 3 + a];
        }
    }
};

// Survivor views of the greedy merge: index i is a survivor's position in the sorted
// order.  ListView reads a caller's rows in place; KalmanView reads the survivors'
// means and covariance-row indices staged in shared memory by the merge kernel
// (cj[i] = the posterior's Gaussian, -1 = a birth) and the covariances from the
// parent's prep rows.
template <typename T> struct ListView {
    static constexpr bool kSelfAbsorbs = false;   // caller's rows: the self-distance is evaluated
    const T* rows;
    const int* s_r;
    __device__ void mean(int i, T mu[6]) const {
        const T* r = rows + (size_t)s_r[i] * kRow + 1;
#pragma unroll
        for (int a = 0; a < 6; ++a) mu[a] = r[a];
    }
    __device__ const T* cov(int i) const { return rows + (size_t)s_r[i] * kRow + 7; }
};
template <typename T> struct KalmanView {
    // every component has a PD covariance (posteriors passed the PD test, births are
    // diagonal), so a centre's distance to itself is exactly 0 < min_separation
    static constexpr bool kSelfAbsorbs = true;
    const T* mu;      // S x 6
    const int* cj;    // S
    const T* covs;    // Gaussian j's covariance at covs + j * kPrep
    const T* bcov;    // birth covariance (21, shared memory)
    __device__ void mean(int i, T m[6]) const {
#pragma unroll
        for (int a = 0; a < 6; ++a) m[a] = mu[i * 6 + a];
    }
    __device__ const T* cov(int i) const {
        const int j = cj[i];
        return j >= 0 ? covs + (size_t)j * kPrep : bcov;
    }
};

// Order of the greedy merge's argmax (and of the map-capacity cut): by weight rounded
// to single precision, higher first; equal keys by the index tie key.  Exact ties are
// common (every birth of an unexplained measurement has weight w0 / (M w0 + kappa)), and
// FP64 weights that differ only in their last bits (a Gaussian term 1e-15 of a
// normaliser) are ordered differently by any two implementations of the FP64 sums; with
// single-precision keys both count as ties.  In FP32 mode the key is the weight itself.
__device__ __forceinline__ float order_key(float w) { return w; }
__device__ __forceinline__ float order_key(double w) { return __double2float_rn(w); }
template <typename T> __device__ __forceinline__ bool merge_before(T wa, uint32_t ka, T wb, uint32_t kb) {
    const float fa = order_key(wa), fb = order_key(wb);
    return fa > fb || (fa == fb && ka < kb);
}

// Bitonic sort of n_pad (a power of two) items in shared arrays, ordered by
// Items::before.  The comparator network is the textbook one (for k = 2, 4, ..:
// for j = k/2 .. 1: items i and i^j swap when the later should come first, in the
// direction of bit k of i).  When the block splits the items into one chunk of 32 R
// items per warp (R = 1..8), every stage whose partners lie in the same chunk runs in
// registers (j < 32: shuffles across lanes; 32 <= j < 32 R: within a thread), and only
// the stages with j >= 32 R go through shared memory, each behind a barrier; otherwise
// every stage does.  Both give the network's result.  Starts and ends with a barrier.
template <typename T> struct SurvItems {   // (weight, tie key, rank) by merge_before
    T* w;
    uint32_t* key;
    int* r;
    struct Item { T w; uint32_t key; int r; };
    __device__ Item load(int i) const { return Item{w[i], key[i], r[i]}; }
    __device__ void store(int i, const Item& x) const { w[i] = x.w; key[i] = x.key; r[i] = x.r; }
    __device__ static bool before(const Item& a, const Item& b) { return merge_before(a.w, a.key, b.w, b.key); }
    __device__ static Item shfl(const Item& x, int m) {
        return Item{__shfl_xor_sync(0xffffffffu, x.w, m), __shfl_xor_sync(0xffffffffu, x.key, m),
                    __shfl_xor_sync(0xffffffffu, x.r, m)};
    }
};
struct KeyItems {   // (key, value) by ascending key
    uint32_t* key;
    int* val;
    struct Item { uint32_t key; int val; };
    __device__ Item load(int i) const { return Item{key[i], val[i]}; }
    __device__ void store(int i, const Item& x) const { key[i] = x.key; val[i] = x.val; }
    __device__ static bool before(const Item& a, const Item& b) { return a.key < b.key; }
    __device__ static Item shfl(const Item& x, int m) {
        return Item{__shfl_xor_sync(0xffffffffu, x.key, m), __shfl_xor_sync(0xffffffffu, x.val, m)};
    }
};

// FP32 survivors as one 64-bit key each, sorted descending: the weight's bits (a
// non-negative float orders as its bit pattern) above the complement of the tie key,
// so that the order is merge_before's; padding slots hold 0 and sort last.  Half the
// shuffles and a single compare per exchange against SurvItems.
struct PackedSurvItems {
    unsigned long long* k;
    typedef unsigned long long Item;
    __device__ Item load(int i) const { return k[i]; }
    __device__ void store(int i, const Item& x) const { k[i] = x; }
    __device__ static bool before(const Item& a, const Item& b) { return a > b; }
    __device__ static Item shfl(const Item& x, int m) { return __shfl_xor_sync(0xffffffffu, x, m); }
};
__device__ __forceinline__ unsigned long long pack_survivor(float w, uint32_t r) {
    return ((unsigned long long)__float_as_uint(w) << 32) | (uint32_t)~tie_key(r);
}
__device__ __forceinline__ uint32_t untie_key(uint32_t t) {   // inverse of tie_key
    return ((t & 0xffffffu) << 8) | (__brev(t >> 24) >> 24);
}

// one shared-memory stage (k, j) over all pairs
template <typename Items>
__device__ __forceinline__ void bitonic_smem_stage(const Items& it, int n_pad, int k, int jj) {
    for (int i = threadIdx.x; i < n_pad; i += blockDim.x) {
        const int ixj = i ^ jj;
        if (ixj > i) {
            const bool up = (i & k) == 0;
            const typename Items::Item lo = it.load(i), hi = it.load(ixj);
            if (Items::before(hi, lo) == up) {
                it.store(i, hi);
                it.store(ixj, lo);
            }
        }
    }
}

// stage (k, j) with 32 <= j < 32 R: pairs (r, r | D) of one thread, D = j / 32
template <int R, int D, typename Items>
__device__ __forceinline__ void bitonic_thread_stage(typename Items::Item (&x)[R], int base, int lane, int k) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
        if ((r & D) == 0 && (r | D) < R) {
            const bool up = ((base + r * 32 + lane) & k) == 0;
            if (Items::before(x[r | D], x[r]) == up) {
                const typename Items::Item t = x[r];
                x[r] = x[r | D];
                x[r | D] = t;
            }
        }
    }
}

// stages (k, j0), (k, j0/2), .., (k, 1), all inside the warp's chunk
template <int R, typename Items>
__device__ __forceinline__ void bitonic_local(typename Items::Item (&x)[R], int base, int lane, int k, int j0) {
    for (int jj = j0; jj > 0; jj >>= 1) {
        if (jj >= 32) {
            const int d = jj >> 5;
            if (d == 4) bitonic_thread_stage<R, 4, Items>(x, base, lane, k);
            else if (d == 2) bitonic_thread_stage<R, 2, Items>(x, base, lane, k);
            else bitonic_thread_stage<R, 1, Items>(x, base, lane, k);
        } else {
            const bool lower = (lane & jj) == 0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const bool up = ((base + r * 32 + lane) & k) == 0;
                const typename Items::Item q = Items::shfl(x[r], jj);
                const bool sw = lower ? (Items::before(q, x[r]) == up) : (Items::before(x[r], q) == up);
                if (sw) x[r] = q;
            }
        }
    }
}

template <int R, typename Items>
__device__ void bitonic_sort_chunks(const Items& it, int n_pad) {
    const int lane = threadIdx.x & 31;
    const int CH = 32 * R, base = (threadIdx.x >> 5) * CH;
    typename Items::Item x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = it.load(base + r * 32 + lane);
    for (int k = 2; k <= CH; k <<= 1) bitonic_local<R, Items>(x, base, lane, k, k >> 1);
#pragma unroll
    for (int r = 0; r < R; ++r) it.store(base + r * 32 + lane, x[r]);
    for (int k = 2 * CH; k <= n_pad; k <<= 1) {
        for (int jj = k >> 1; jj >= CH; jj >>= 1) {
            __syncthreads();
            bitonic_smem_stage(it, n_pad, k, jj);
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R; ++r) x[r] = it.load(base + r * 32 + lane);
        bitonic_local<R, Items>(x, base, lane, k, CH >> 1);
#pragma unroll
        for (int r = 0; r < R; ++r) it.store(base + r * 32 + lane, x[r]);
    }
}

template <typename Items>
__device__ void block_bitonic_sort(const Items& it, int n_pad) {
    __syncthreads();
    const int nw = blockDim.x >> 5;
    const int ch = n_pad / nw;
    if (ch * nw == n_pad && ch >= 32 && ch <= 256) {
        if (ch == 32) bitonic_sort_chunks<1>(it, n_pad);
        else if (ch == 64) bitonic_sort_chunks<2>(it, n_pad);
        else if (ch == 128) bitonic_sort_chunks<4>(it, n_pad);
        else bitonic_sort_chunks<8>(it, n_pad);
    } else {
        for (int k = 2; k <= n_pad; k <<= 1)
            for (int jj = k >> 1; jj > 0; jj >>= 1) {
                bitonic_smem_stage(it, n_pad, k, jj);
                __syncthreads();
            }
    }
    __syncthreads();
}

// In-place sort of (w, key, r) by merge_before over n_pad (power of 2) slots.
template <typename T>
__device__ void sort_survivors(T* s_w, uint32_t* s_key, int* s_r, int n_pad) {
    block_bitonic_sort(SurvItems<T>{s_w, s_key, s_r}, n_pad);
}

// Block-wide exclusive scan of int flags; returns the total.  Starts with a barrier:
// callers write data in any pattern, each thread then scans a contiguous chunk.
__device__ int block_exclusive_scan(int* data, int n, int* s_tmp) {
    __syncthreads();
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int lo = threadIdx.x * per, hi = min(n, lo + per);
    int run = 0;
    for (int i = lo; i < hi; ++i) { int v = data[i]; data[i] = run; run += v; }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int v = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) s_tmp[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int w = 0; w < nw; ++w) { int t = s_tmp[w]; s_tmp[w] = acc; acc += t; }
        s_tmp[nw] = acc;
    }
    __syncthreads();
    const int off = s_tmp[warp] + v - run;
    for (int i = lo; i < hi; ++i) data[i] += off;
    const int total = s_tmp[nw];
    __syncthreads();
    return total;
}

// lock-free union-find on shared memory: roots only change by CAS from a self
// loop, the larger root is attached under the smaller, so every component's root
// is its smallest index
__device__ __forceinline__ int uf_find(int* uf, int x) {
    int p = uf[x];
    while (p != x) {
        int gp = uf[p];
        if (gp != p) uf[x] = gp;   // path halving; only ever points closer to the root
        x = p;
        p = uf[x];
    }
    return x;
}
__device__ __forceinline__ void uf_unite(int* uf, int a, int b) {
    while (true) {
        a = uf_find(uf, a);
        b = uf_find(uf, b);
        if (a == b) return;
        if (a < b) { int t = a; a = b; b = t; }
        if (atomicCAS(&uf[a], a, b) == a) return;
    }
}

// Shared-memory working set of the merge (per CTA); sizes are derived from the
// survivor capacity S and map capacity G by merge_smem_bytes().
template <typename T> struct MergeScratch {
    float* pf;            // S x 6: mean[0..3), cov diagonal [0..3) (prefilter data)
    uint8_t* flag;        // S: merged
    uint8_t* is_center;   // S
    int* lab;             // S: union-find parent, then the component's root
    int* cidx;            // S: component index of a root; later the queue of large components
    int* start;           // S + 1: member range of each component in perm
    int* fill;            // S
    int* perm;            // cap: survivors grouped by component (first: survivors in u order)
    uint32_t* masks;      // (blockDim/32) x nchunk member masks
    int nchunk;
};

constexpr int kSmallComp = 8;       // components up to this size are merged by one thread
constexpr int kMergeThreads = 256;   // threads of a parent's merge block (8 warps)

__host__ __device__ inline int next_pow2(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

// sort capacity (survivors, then map entries), in elements
__host__ __device__ inline int merge_sort_cap(int S, int G) {
    int a = next_pow2(S), b = S + G;
    return a > b ? a : b;
}

// Survivor staging of the filter's merge (KalmanView) in front of the scratch: means
// (S x 6), the birth covariance (21) and covariance-row indices (S).  A caller's rows
// (ListView) are read in place and stage nothing.  (Staging the G posterior
// covariances as well was measured slower: the copy costs more than the reads save.)
template <typename T> __host__ __device__ inline size_t merge_stage_bytes(int S, bool stage) {
    return stage ? (((6 * (size_t)S + 21) * sizeof(T) + 4 * (size_t)S + 15) & ~(size_t)15) : 0;
}
template <typename T> inline size_t merge_smem_bytes(int S, int G, int nwarps, bool stage) {
    const size_t cap = merge_sort_cap(S, G), nchunk = (S + 31) / 32;
    const size_t pf = 6 * (size_t)S * sizeof(float), pos = (size_t)(S + G) * 4;   // pos aliases pf
    return merge_stage_bytes<T>(S, stage) + cap * (sizeof(T) + 8) + (pf > pos ? pf : pos) + 3 * (size_t)S * 4 +
           cap * 4 + (size_t)(S + 1) * 4 + (size_t)nwarps * nchunk * 4 + 2 * (size_t)S + 64;
}
template <typename T>
__device__ inline void carve_merge_smem(unsigned char* smem, int S, int G, bool stage, T*& s_w, uint32_t*& s_key,
                                        int*& s_r, int*& s_pos, MergeScratch<T>& ms) {
    const int cap = merge_sort_cap(S, G);
    s_w = reinterpret_cast<T*>(smem + merge_stage_bytes<T>(S, stage));
    s_key = reinterpret_cast<uint32_t*>(s_w + cap);
    s_r = reinterpret_cast<int*>(s_key + cap);
    ms.pf = reinterpret_cast<float*>(s_r + cap);
    s_pos = reinterpret_cast<int*>(ms.pf);   // positions are used only once the prefilter rows are dead
    ms.lab = reinterpret_cast<int*>(ms.pf + (6 * S > S + G ? 6 * S : S + G));
    ms.cidx = ms.lab + S;
    ms.fill = ms.cidx + S;
    ms.perm = ms.fill + S;
    ms.start = ms.perm + cap;
    ms.nchunk = (S + 31) / 32;
    ms.masks = reinterpret_cast<uint32_t*>(ms.start + S + 1);
    ms.flag = reinterpret_cast<uint8_t*>(ms.masks + (blockDim.x / 32) * ms.nchunk);
    ms.is_center = ms.flag + S;
}

__device__ __forceinline__ bool could_merge_f(const float* a, const float* b, float min_sep, float margin) {
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float d = a[k] - b[k];
        ok = ok && (d * d <= min_sep * (a[3 + k] + b[3 + k]) * margin);
    }
    return ok;
}

// Moment-matched merge of the members (ascending survivor indices mem[k] for the set
// bits k of mbits) into centre c, written to sparse[c]; reference order of the sums
// (kernels.cu:770-843): weights and weighted means, then covariances about the mean.
template <typename T, typename View>
__device__ void merge_members_thread(const View& v, const T* s_w, const int* mem, uint32_t mbits, int c, const T* cmu,
                                     const T* ccov, T* sparse) {
    T W = 0, acc[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t mb = mbits; mb; mb &= mb - 1) {
        int i = mem[__ffs(mb) - 1];
        T w = s_w[i], mu[6];
        if (i == c) {   // the centre's mean is already at hand (same values)
#pragma unroll
            for (int a = 0; a < 6; ++a) mu[a] = cmu[a];
        } else {
            v.mean(i, mu);
        }
        W += w;
#pragma unroll
        for (int a = 0; a < 6; ++a) acc[a] += w * mu[a];
    }
    T row[28];
    row[0] = W;
    const T iW = T(1) / W;
#pragma unroll
    for (int a = 0; a < 6; ++a) row[1 + a] = div_by(acc[a], W, iW);
    T cv[21];
#pragma unroll
    for (int e = 0; e < 21; ++e) cv[e] = 0;
    for (uint32_t mb = mbits; mb; mb &= mb - 1) {
        int i = mem[__ffs(mb) - 1];
        T w = s_w[i], mu[6], d[6];
        if (i == c) {
#pragma unroll
            for (int a = 0; a < 6; ++a) mu[a] = cmu[a];
        } else {
            v.mean(i, mu);
        }
        const T* sc = v.cov(i);
#pragma unroll
        for (int a = 0; a < 6; ++a) d[a] = row[1 + a] - mu[a];
#pragma unroll
        for (int a = 0; a < 6; ++a)
#pragma unroll
            for (int bb = 0; bb <= a; ++bb) cv[tri(a, bb)] += w * (sc[tri(a, bb)] + d[a] * d[bb]);
    }
#pragma unroll
    for (int e = 0; e < 21; ++e) row[7 + e] = div_by(cv[e], W, iW);
    T L[21];
    const bool pd = chol6(row + 7, L);
    if (!pd) {   // "bad hack, just keep the max feature" (kernels.cu:855-862)
        row[0] = s_w[c];
#pragma unroll
        for (int a = 0; a < 6; ++a) row[1 + a] = cmu[a];
#pragma unroll
        for (int e = 0; e < 21; ++e) row[7 + e] = ccov[e];
    }
    row28_store(sparse + (size_t)c * kRow, row);
}

// Order-preserving integer key of a non-negative weight's order key (the bits of the
// weight rounded to single precision).
template <typename T> __device__ __forceinline__ uint64_t weight_key(T w) {
    return (uint64_t)__float_as_uint(order_key(w));
}

// Exact k-th largest key among the entries with w >= 0 (k <= their count), by an
// MSB-first radix select over the key's four 8-bit digits.  Block-wide call.
template <typename T>
__device__ uint64_t select_kth_largest(const T* w, int n, int k) {
    __shared__ int s_hist[256];
    __shared__ uint64_t s_prefix;
    __shared__ int s_k;
    const int passes = 4;
    uint64_t prefix = 0, mask = 0;
    if (threadIdx.x == 0) s_k = k;
    for (int d = passes - 1; d >= 0; --d) {
        for (int b = threadIdx.x; b < 256; b += blockDim.x) s_hist[b] = 0;
        __syncthreads();
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            const T v = w[e];
            if (!(v >= T(0))) continue;
            const uint64_t key = weight_key(v);
            if ((key & mask) == prefix) atomicAdd(&s_hist[(key >> (8 * d)) & 255], 1);
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            // the bin holding the k-th largest: counts from the top bin down, lane l owning
            // bins 255-8l .. 248-8l; the first lane whose running total reaches k walks its 8
            const int lane = threadIdx.x;
            int c[8], sum = 0;
#pragma unroll
            for (int q = 0; q < 8; ++q) { c[q] = s_hist[255 - 8 * lane - q]; sum += c[q]; }
            int incl = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            const int kk = s_k;
            const unsigned hit = __ballot_sync(0xffffffffu, incl >= kk);
            const int owner = hit ? __ffs(hit) - 1 : 31;
            if (lane == owner) {
                int rem = kk - (incl - sum), b = 255 - 8 * lane;
                for (int q = 0; q < 8; ++q, --b) {
                    if (b == 0 || c[q] >= rem) break;
                    rem -= c[q];
                }
                s_k = rem;
                s_prefix = prefix | ((uint64_t)b << (8 * d));
            }
        }
        __syncthreads();
        prefix = s_prefix;
        mask |= (uint64_t)255 << (8 * d);
    }
    return prefix;
}

// In-place bitonic sort of (key, payload) ascending by key over n_pad (power of 2) slots.
__device__ void sort_keys(uint32_t* key, int* val, int n_pad) {
    block_bitonic_sort(KeyItems{key, val}, n_pad);
}

// Greedy reduction of phdUpdateMergeKernel (src/kernels.cu:693-866) over n
// survivors already sorted into the reference's argmax order: the next centre is
// the first unmerged survivor, every unmerged survivor within squared Mahalanobis
// distance < min_sep of it (covariance sum) is absorbed, the moment-matched result
// is kept if PD, else the centre.  Since x' A^-1 x >= x_k^2 / A_kk for SPD A, two
// survivors failing the diagonal bound on u, v or d (with a safety margin) can
// never merge; the greedy sequence therefore decomposes exactly over the connected
// components of the "may merge" graph.  Components are listed with their members in
// sorted order; one thread runs the greedy loop of a small component, one warp that
// of a large one.  Merged rows are written to sparse[centre index]; returns the
// index of the first centre that absorbed nothing (the reference's loop ends there),
// or n.  Block-wide call.
template <typename T, typename View>
__device__ int merge_components(const View& v, const T* s_w, const int* s_r, int n, MergeScratch<T> ms,
                                uint32_t* ukey, T min_sep, T* sparse, int* member_out,
                                unsigned long long* counters) {
    __shared__ int s_ncomp, s_take, s_nlarge, s_take_large, s_stop, s_evals;
    __shared__ int s_tmp[40];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float fsep = (float)min_sep, fmargin = 1.01f;
    for (int i = tid; i < n; i += blockDim.x) {
        T mu[6];
        v.mean(i, mu);
        const T* cv = v.cov(i);
        float* pf = ms.pf + i * 6;
        pf[0] = (float)mu[0]; pf[1] = (float)mu[1]; pf[2] = (float)mu[2];
        pf[3] = (float)cv[0]; pf[4] = (float)cv[2]; pf[5] = (float)cv[5];
        ms.flag[i] = 0;
        ms.is_center[i] = 0;
        ms.lab[i] = i;
    }
    if (tid == 0) { s_ncomp = 0; s_take = 0; s_nlarge = 0; s_take_large = 0; s_stop = n; s_evals = 0; }
    __syncthreads();
    // "may merge" edges -> union-find.  |du| <= sqrt(sep*margin*(Suu_i + max Suu)) is
    // necessary for the bound on u, so with the survivors in u order each one scans
    // forward only over that window.
    __shared__ float s_maxsuu;
    {
        float mx = 0.f;
        for (int i = tid; i < n; i += blockDim.x) {
            mx = fmaxf(mx, ms.pf[i * 6 + 3]);
            const float u = ms.pf[i * 6 + 0];
            uint32_t bits = __float_as_uint(u);
            ukey[i] = (bits & 0x80000000u) ? ~bits : (bits | 0x80000000u);   // orderable float key
            ms.perm[i] = i;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (tid == 0) s_maxsuu = 0.f;
        __syncthreads();
        if (lane == 0) atomicMax(reinterpret_cast<int*>(&s_maxsuu), __float_as_int(mx));   // mx >= 0
        const int np2 = next_pow2(n);
        for (int i = n + tid; i < np2; i += blockDim.x) { ukey[i] = 0xffffffffu; ms.perm[i] = 0x7fffffff; }
        __syncthreads();
        sort_keys(ukey, ms.perm, np2);
    }
    const float maxsuu = s_maxsuu;
    for (int q = tid; q < n; q += blockDim.x) {
        const int i = ms.perm[q];
        float a[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) a[k] = ms.pf[i * 6 + k];
        const float reach = sqrtf(fsep * fmargin * (a[3] + maxsuu)) * 1.0001f;
        for (int q2 = q + 1; q2 < n; ++q2) {
            const int j = ms.perm[q2];
            const float* bj = ms.pf + j * 6;
            if (bj[0] - a[0] > reach) break;
            if (could_merge_f(a, bj, fsep, fmargin)) uf_unite(ms.lab, i, j);
        }
    }
    __syncthreads();
    for (int i = tid; i < n; i += blockDim.x) {
        if (uf_find(ms.lab, i) == i) {
            int c = atomicAdd(&s_ncomp, 1);
            ms.cidx[i] = c;
            ms.start[c] = 0;
            ms.fill[c] = 0;
        }
    }
    __syncthreads();
    for (int i = tid; i < n; i += blockDim.x) ms.lab[i] = uf_find(ms.lab, i);
    __syncthreads();
    const int ncomp = s_ncomp;
    for (int i = tid; i < n; i += blockDim.x) atomicAdd(&ms.start[ms.cidx[ms.lab[i]]], 1);
    __syncthreads();
    block_exclusive_scan(ms.start, ncomp, s_tmp);
    if (tid == 0) ms.start[ncomp] = n;
    __syncthreads();
    // members of each component in ascending order (chunks in order, ranks by lane)
    if (warp == 0) {
        for (int base = 0; base < n; base += 32) {
            const int i = base + lane;
            const bool valid = i < n;
            const unsigned vmask = __ballot_sync(0xffffffffu, valid);
            if (valid) {
                const int c = ms.cidx[ms.lab[i]];
                const unsigned grp = __match_any_sync(vmask, c);
                const int leader = __ffs(grp) - 1;
                const int rank = __popc(grp & ((1u << lane) - 1u));
                int off = 0;
                if (lane == leader) {
                    off = ms.fill[c];
                    ms.fill[c] = off + __popc(grp);
                }
                off = __shfl_sync(grp, off, leader);
                ms.perm[ms.start[c] + off + rank] = i;
            }
            __syncwarp();
        }
    }
    __syncthreads();
    int evals = 0;
    // small components: one thread each; large ones are queued for the warps
    while (true) {
        const int c = atomicAdd(&s_take, 1);
        if (c >= ncomp) break;
        const int s0 = ms.start[c], cnt = ms.start[c + 1] - s0;
        if (cnt > kSmallComp) {
            ms.cidx[atomicAdd(&s_nlarge, 1)] = c;   // roots' indices are no longer needed
            continue;
        }
        const int* mem = ms.perm + s0;
        uint32_t done = 0;
        while (true) {
            const int k0 = __ffs(~done) - 1;
            if (k0 < 0 || k0 >= cnt) break;
            const int cc = mem[k0];
            T cmu[6], ccov[21];
            v.mean(cc, cmu);
            const T* cp = v.cov(cc);
#pragma unroll
            for (int q = 0; q < 21; ++q) ccov[q] = cp[q];
            uint32_t mbits = 0;
            for (int k = k0; k < cnt; ++k) {
                if ((done >> k) & 1u) continue;
                const int i = mem[k];
                if (View::kSelfAbsorbs && k == k0) {   // distance to itself: 0
                    mbits |= 1u << k;
                    continue;
                }
                if (!could_merge_f(ms.pf + cc * 6, ms.pf + i * 6, fsep, fmargin)) continue;
                ++evals;
                T mu[6];
                v.mean(i, mu);
                if (mahal6(cmu, ccov, mu, v.cov(i)) < min_sep) mbits |= 1u << k;
            }
            if (!mbits) {   // merged weight 0: the reference's loop ends (kernels.cu:783-784)
                atomicMin(&s_stop, cc);
                break;
            }
            merge_members_thread(v, s_w, mem, mbits, cc, cmu, ccov, sparse);
            ms.is_center[cc] = 1;
            if (member_out)
                for (uint32_t mb = mbits; mb; mb &= mb - 1) member_out[s_r[mem[__ffs(mb) - 1]]] = cc;
            done |= mbits;
        }
    }
    __syncthreads();
    // large components: one warp each, lanes over the member range
    uint32_t* masks = ms.masks + (size_t)warp * ms.nchunk;
    while (true) {
        int q = 0;
        if (lane == 0) q = atomicAdd(&s_take_large, 1);
        q = __shfl_sync(0xffffffffu, q, 0);
        if (q >= s_nlarge) break;
        const int c = ms.cidx[q];
        const int s0 = ms.start[c], cnt = ms.start[c + 1] - s0;
        const int* mem = ms.perm + s0;
        const int nch = (cnt + 31) >> 5;
        int next = 0;
        while (true) {
            int k0 = -1;
            for (int ch = next >> 5; ch < nch; ++ch) {
                const int k = ch * 32 + lane;
                const bool pred = k >= next && k < cnt && !ms.flag[mem[k]];
                const unsigned bal = __ballot_sync(0xffffffffu, pred);
                if (bal) { k0 = ch * 32 + __ffs(bal) - 1; break; }
            }
            if (k0 < 0) break;
            next = k0 + 1;
            const int cc = mem[k0];
            T cmu[6], ccov[21];
            v.mean(cc, cmu);
            const T* cp = v.cov(cc);
#pragma unroll
            for (int qq = 0; qq < 21; ++qq) ccov[qq] = cp[qq];
            bool any = false;
            for (int ch = k0 >> 5; ch < nch; ++ch) {
                const int k = ch * 32 + lane;
                bool m = false;
                if (k >= k0 && k < cnt) {
                    const int i = mem[k];
                    if (!ms.flag[i] && could_merge_f(ms.pf + cc * 6, ms.pf + i * 6, fsep, fmargin)) {
                        ++evals;
                        T mu[6];
                        v.mean(i, mu);
                        m = mahal6(cmu, ccov, mu, v.cov(i)) < min_sep;
                    }
                }
                const unsigned bal = __ballot_sync(0xffffffffu, m);
                if (lane == 0) masks[ch] = bal;
                any = any || bal;
            }
            __syncwarp();
            if (!any) {
                if (lane == 0) atomicMin(&s_stop, cc);
                break;
            }
            // weight and mean (lane a < 6 owns mean[a]), members in ascending order
            T accw = 0, accm = 0;
            for (int ch = k0 >> 5; ch < nch; ++ch) {
                for (unsigned mk = masks[ch]; mk; mk &= mk - 1) {
                    const int i = mem[ch * 32 + __ffs(mk) - 1];
                    T w = s_w[i], mu[6];
                    v.mean(i, mu);
                    accw += w;
                    T sel = mu[0];
#pragma unroll
                    for (int a = 1; a < 6; ++a) sel = (lane == a) ? mu[a] : sel;
                    if (lane < 6) accm += w * sel;
                }
            }
            const T W = accw;
            const T my_mean = (lane < 6) ? accm / W : T(0);
            T mean[6];
#pragma unroll
            for (int a = 0; a < 6; ++a) mean[a] = __shfl_sync(0xffffffffu, my_mean, a);
            int ea = 0;
            while ((ea + 1) * (ea + 2) / 2 <= lane && ea < 5) ++ea;
            const int eb = lane - ea * (ea + 1) / 2;
            T accc = 0;
            for (int ch = k0 >> 5; ch < nch; ++ch) {
                const unsigned mk0 = masks[ch];
                const int k = ch * 32 + lane;
                if (mk0 & (1u << lane)) {
                    const int i = mem[k];
                    ms.flag[i] = 1;
                    if (member_out) member_out[s_r[i]] = cc;
                }
                for (unsigned mk = mk0; mk; mk &= mk - 1) {
                    const int i = mem[ch * 32 + __ffs(mk) - 1];
                    if (lane < 21) {
                        T w = s_w[i], mu[6];
                        v.mean(i, mu);
                        const T* cv = v.cov(i);
                        accc += w * (cv[lane] + (mean[ea] - mu[ea]) * (mean[eb] - mu[eb]));
                    }
                }
            }
            const T my_cov = (lane < 21) ? accc / W : T(0);
            T row[28];
            row[0] = W;
#pragma unroll
            for (int a = 0; a < 6; ++a) row[1 + a] = mean[a];
#pragma unroll
            for (int qq = 0; qq < 21; ++qq) row[7 + qq] = __shfl_sync(0xffffffffu, my_cov, qq);
            T L[21];
            const bool pd = chol6(row + 7, L);
            T* o = sparse + (size_t)cc * kRow;
            if (lane < 28) {
                T v = pd ? row[0] : s_w[cc];
#pragma unroll
                for (int qq = 1; qq < 28; ++qq)
                    if (lane == qq) v = pd ? row[qq] : (qq < 7 ? cmu[qq - 1] : ccov[qq - 7]);
                o[lane] = v;
            }
            if (lane == 0) ms.is_center[cc] = 1;
            __syncwarp();
        }
    }
    atomicAdd(&s_evals, evals);
    __syncthreads();
    if (tid == 0 && counters) atomicAdd(&counters[12], (unsigned long long)s_evals);
    return s_stop;
}

template <typename T, int K>
__device__ __forceinline__ void merge_body(const Params& prm, const Bufs<T>& b, int cur, int M, int fixed, int p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int tid = threadIdx.x;
    const int G = min(b.map_n[cur][b.src[p]], prm.Gcap);
    const int n_all_surv = b.surv_n[p];
    const int n = min(n_all_surv, prm.Scap);
    const int n_pad = next_pow2(n);
    T* s_w;
    uint32_t* s_key;
    int* s_r;
    int* s_pos;
    MergeScratch<T> ms;
    carve_merge_smem<T>(smem, prm.Scap, prm.Gcap, true, s_w, s_key, s_r, s_pos, ms);
    __shared__ int s_tmp[40];
    // FP32: packed sort keys in the survivor staging area (free until the survivors are
    // staged; 8 n_pad <= 16 Scap bytes fit in its 28 Scap); FP64: (weight, tie key, rank)
    unsigned long long* s_pk = reinterpret_cast<unsigned long long*>(smem);
    for (int i = tid; i < n_pad; i += blockDim.x) {
        if (sizeof(T) == 4) {
            s_pk[i] = i < n ? pack_survivor((float)b.surv_w[(size_t)p * prm.Scap + i],
                                            (uint32_t)b.surv_r[(size_t)p * prm.Scap + i])
                            : 0ull;
        } else if (i < n) {
            s_w[i] = b.surv_w[(size_t)p * prm.Scap + i];
            s_r[i] = b.surv_r[(size_t)p * prm.Scap + i];
            s_key[i] = tie_key((uint32_t)s_r[i]);
        } else {
            s_w[i] = T(-1);
            s_key[i] = 0xffffffffu;
            s_r[i] = 0x7fffffff;
        }
    }
    // parent log-likelihood: sum_m ell + sum_j w_j (.cu:1813-1849), FP64, in an order
    // that does not depend on the block's width (128 or 256 threads, stage kernel or
    // fused): 256 lane partials, a butterfly within each group of 32, the 8 group
    // totals in order
    __shared__ double s_part[256];
    for (int v = tid; v < 256; v += blockDim.x) {
        double part = 0;
        for (int mm = v; mm < M; mm += 256) part += (double)b.ell[(size_t)p * prm.Mcap + mm];
        for (int j = v; j < G; j += 256) part += (double)b.fit[((size_t)p * prm.Gcap + j) * kRow];
        s_part[v] = part;
    }
    __syncthreads();
    if (tid < 32) {
        double t = 0;
        for (int grp = 0; grp < 8; ++grp) {
            double part = s_part[grp * 32 + tid];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
            t += part;
        }
        if (tid == 0) b.loglik[p] = t;
    }
    if (sizeof(T) == 4) {
        block_bitonic_sort(PackedSurvItems{s_pk}, n_pad);
        for (int i = tid; i < n_pad; i += blockDim.x) {
            const unsigned long long v = s_pk[i];
            s_w[i] = i < n ? (T)__uint_as_float((uint32_t)(v >> 32)) : T(-1);
            s_r[i] = i < n ? (int)untie_key(~(uint32_t)v) : 0x7fffffff;
        }
        __syncthreads();   // the staging below reuses the key area
    } else {
        sort_survivors(s_w, s_key, s_r, n_pad);
    }
    KalmanSource<T, K> src;
    src.fit = b.fit + (size_t)p * prm.Gcap * kRow;
    src.prep = b.prep + (size_t)p * prm.Gcap * kPrep;
    src.z = b.z;
    src.G = G;
    src.M = M;
    src.bmean[0] = 0; src.bmean[1] = 0;
    src.bmean[2] = (T)prm.d0; src.bmean[3] = (T)prm.vu0; src.bmean[4] = (T)prm.vv0; src.bmean[5] = (T)prm.vd0;
    for (int i = 0; i < 21; ++i) src.bcov[i] = 0;
    src.bcov[tri(0, 0)] = (T)prm.model.var[0];
    src.bcov[tri(1, 1)] = (T)prm.model.var[1];
    src.bcov[tri(2, 2)] = (K == 3) ? (T)prm.model.var[2] : (T)prm.var_d0;
    src.bcov[tri(3, 3)] = (T)prm.var_vu0;
    src.bcov[tri(4, 4)] = (T)prm.var_vv0;
    src.bcov[tri(5, 5)] = (T)prm.var_vd0;
    // survivors' means and covariance rows staged once (each is read several times)
    KalmanView<T> view;
    {
        T* st_mu = reinterpret_cast<T*>(smem);
        T* st_bcov = st_mu + 6 * prm.Scap;
        int* st_cj = reinterpret_cast<int*>(st_bcov + 21);
        for (int i = tid; i < n; i += blockDim.x) {
            const int r = s_r[i];
            T mu[6];
            src.mean(r, mu);
#pragma unroll
            for (int a = 0; a < 6; ++a) st_mu[i * 6 + a] = mu[a];
            st_cj[i] = r < G * M ? r % G : -1;
        }
        if (tid < 21) st_bcov[tid] = src.bcov[tid];
        view.covs = src.prep + kPrepCov;
        view.mu = st_mu;
        view.cj = st_cj;
        view.bcov = st_bcov;
        __syncthreads();
    }
    T* sparse = b.mtmp + (size_t)p * prm.Scap * kRow;
    const int stop = merge_components<T>(view, s_w, s_r, n, ms, s_key, (T)prm.min_sep, sparse, nullptr, b.counters);
    // merged list in centre order (centres after a stop are dropped, as the reference's loop ends there)
    for (int i = tid; i < n; i += blockDim.x) s_pos[i] = (i < stop && ms.is_center[i]) ? 1 : 0;
    __syncthreads();
    const int n_out = block_exclusive_scan(s_pos, n, s_tmp);
    // merged component e (output order) is the row sparse[centre_of[e]]; the member
    // lists are dead once the merge has run, so their slots hold centre_of
    int* centre_of = ms.perm;
    for (int i = tid; i < n; i += blockDim.x)
        if (i < stop && ms.is_center[i]) centre_of[s_pos[i]] = i;
    __syncthreads();
    for (int e = tid; e < n_out; e += blockDim.x) b.mlist[(size_t)p * prm.Scap + e] = centre_of[e];
    // new map: merged components then retained non-detection clouds (.cu:1923-2058);
    // entries e < n_out are merged, e >= n_out are the Gaussians j = e - n_out
    const T minw = (T)prm.min_weight;
    const int n_all = n_out + G;
    int n_valid_part = 0;
    for (int e = tid; e < n_all; e += blockDim.x) {
        T w;
        if (e < n_out) {
            w = sparse[(size_t)centre_of[e] * kRow];
        } else {
            const T* fr = b.fit + ((size_t)p * prm.Gcap + (e - n_out)) * kRow;
            const T wnd = nd_weight(fr[0], fr[1]);
            w = (wnd >= minw) ? wnd : T(-1);   // -1: not retained
        }
        s_w[e] = w;
        n_valid_part += w >= T(0);
    }
    __shared__ int s_nvalid;
    if (tid == 0) s_nvalid = 0;
    __syncthreads();
    atomicAdd(&s_nvalid, n_valid_part);
    __syncthreads();
    const bool cut = s_nvalid > prm.Gcap;
    // keep: retained, and when over capacity among the Gcap largest (ties by entry order)
    if (!cut) {
        for (int e = tid; e < n_all; e += blockDim.x) s_pos[e] = s_w[e] >= T(0);
        __syncthreads();
    } else {
        const uint64_t thr = select_kth_largest(s_w, n_all, prm.Gcap);
        // entries above the threshold, then ties in entry order up to Gcap
        int above = 0;
        for (int e = tid; e < n_all; e += blockDim.x) {
            const T w = s_w[e];
            const uint64_t key = w >= T(0) ? weight_key(w) : 0ull;
            above += key > thr;
            s_pos[e] = (w >= T(0) && key == thr) ? 1 : 0;
        }
        __shared__ int s_above;
        if (tid == 0) s_above = 0;
        __syncthreads();
        atomicAdd(&s_above, above);
        __syncthreads();
        const int ties_keep = prm.Gcap - s_above;
        block_exclusive_scan(s_pos, n_all, s_tmp);   // rank among the ties
        for (int e = tid; e < n_all; e += blockDim.x) {
            const T w = s_w[e];
            const uint64_t key = w >= T(0) ? weight_key(w) : 0ull;
            const bool tie = w >= T(0) && key == thr;
            s_pos[e] = (w >= T(0) && key > thr) || (tie && s_pos[e] < ties_keep);
        }
        __syncthreads();
    }
    const int total = block_exclusive_scan(s_pos, n_all, s_tmp);
    const int wrow = p;   // the new map lives at row p of the other buffer
    T* mo = b.map[cur ^ 1] + (size_t)wrow * prm.Gcap * kRow;
    int* mr = b.map_ref[cur ^ 1] + (size_t)wrow * prm.Gcap;
    for (int e = tid; e < n_all; e += blockDim.x) {
        const int pos = s_pos[e];
        const int nxt = (e + 1 < n_all) ? s_pos[e + 1] : total;
        if (nxt == pos) continue;   // not kept
        if (e < n_out) {   // merged component: weight, mean and the Cholesky factor of its covariance
            T v[28];
            row28_load(sparse + (size_t)centre_of[e] * kRow, v);
            T L[21];
            chol6(v + 7, L);
#pragma unroll
            for (int q = 0; q < 21; ++q) v[7 + q] = L[q];
            row28_store(mo + (size_t)pos * kRow, v);
            mr[pos] = -1 - e;
        } else {
            const int j = e - n_out;
            mo[(size_t)pos * kRow] = s_w[e];
            mr[pos] = p * prm.Gcap + j;
        }
    }
    if (tid == 0) {
        b.merged_n[p] = n_out;
        b.map_n[cur ^ 1][wrow] = min(total, prm.Gcap);
        double* me = b.map_ext[cur ^ 1] + 12 * wrow;
        for (int q = 0; q < 12; ++q) me[q] = fixed ? 0.0 : b.ext[12 * p + q];
        if (cut) atomicAdd(&b.counters[0], 1ull);
        atomicAdd(&b.counters[5], (unsigned long long)n);
        atomicAdd(&b.counters[7], (unsigned long long)n);
        atomicAdd(&b.counters[11], (unsigned long long)n_out);
        atomicMax(&b.counters[13], (unsigned long long)n_all_surv);
        b.fit_n[p] = G;   // prior map size, for the inspection dumps
        b.src[p] = p;     // the new map lives at row p: the indirection is reset
    }
}

template <typename T, int K>
__global__ void __launch_bounds__(kMergeThreads, sizeof(T) == 4 ? 3 : 2) k_merge(__grid_constant__ const Params prm, __grid_constant__ const Bufs<T> b,
                                               int cur, int M, int fixed) {
    merge_body<T, K>(prm, b, cur, M, fixed, blockIdx.x);
}

template <typename T, int K>
__global__ void __launch_bounds__(kMergeThreads, sizeof(T) == 4 ? 3 : 2)
    k_merge_batch(const __grid_constant__ SlotTable<T> tab, const FrameArgs* fas, const int2* map) {
    const int2 fp = map[blockIdx.x];
    const FrameArgs fa = fas[fp.x];
    merge_body<T, K>(tab.prm[fp.x], tab.b[fp.x], fa.cur, fa.M, fa.fixed, fp.y);
}

// ---------------------------------------------------------------- fused update
// The update of one parent -- cloud fit, Kalman terms, likelihood and merge -- run by
// one block, for every parent of a filter (or of a batch group) in one launch: a grid
// of at most the resident capacity takes parents from a work counter until none is
// left.  No block waits for another: a parent's stages read only that parent's rows
// (written to global memory and read back by the same block, from L2), so the grid
// has no stage boundaries and no per-stage tails.  The launch before converts the
// measurements and resets the counters; the filter-level weight update and resampling
// run in the launches after.  Results are those of the stage-by-stage kernels (the
// same bodies on the same inputs; the likelihood's survivor slots may come in another
// order, and the merge sorts them).
constexpr int kFusedThreads = 256;
template <typename T> inline size_t fused_smem_bytes(int P, int Gcap, int Scap) {
    size_t s = cloud_fit_smem_bytes<T>(P);
    const size_t cand[3] = {prep_smem_bytes<T>(), likelihood_smem_bytes<T>(Gcap, kFusedThreads),
                            merge_smem_bytes<T>(Scap, Gcap, kFusedThreads / 32, true)};
    for (size_t c : cand) s = c > s ? c : s;
    return s;
}

template <typename T, int K>
__device__ __forceinline__ void fused_parent(const Params& prm, const Bufs<T>& b, const FrameArgs& fa, int p,
                                             unsigned char* smem) {
    cloud_fit_body<T, K>(prm, b, fa.cur, fa.M, fa.fixed, fa.has_pred, fa.dt, fa.pred_frame, fa.sample_frame, nullptr,
                         nullptr, nullptr, p, 0, 1, reinterpret_cast<T*>(smem));
    __syncthreads();
    prep_body<T, K>(prm, b, fa.cur, p, reinterpret_cast<T*>(smem));
    for (int mb = 0; mb * (int)blockDim.x < fa.M; ++mb) {
        likelihood_body<T, K>(prm, b, fa.cur, fa.M, p, mb, reinterpret_cast<T*>(smem));
        __syncthreads();
    }
    merge_body<T, K>(prm, b, fa.cur, fa.M, fa.fixed, p);
    __syncthreads();
}

template <typename T, int K>
__global__ void __launch_bounds__(kFusedThreads, sizeof(T) == 4 ? 3 : 2)
    k_fused(__grid_constant__ const Params prm, __grid_constant__ const Bufs<T> b, const FrameArgs fa, int* work) {
    extern __shared__ __align__(16) unsigned char dsm_fused[];
    __shared__ int s_item;
    while (true) {
        if (threadIdx.x == 0) s_item = atomicAdd(work, 1);
        __syncthreads();
        const int p = s_item;
        __syncthreads();
        if (p >= prm.N) break;
        fused_parent<T, K>(prm, b, fa, p, dsm_fused);
    }
}

template <typename T, int K>
__global__ void __launch_bounds__(kFusedThreads, sizeof(T) == 4 ? 3 : 2)
    k_fused_batch(const __grid_constant__ SlotTable<T> tab, const FrameArgs* fas, const int2* map, int n_items,
                  int* work) {
    extern __shared__ __align__(16) unsigned char dsm_fused[];
    __shared__ int s_item;
    while (true) {
        if (threadIdx.x == 0) s_item = atomicAdd(work, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= n_items) break;
        const int2 fp = map[it];
        const FrameArgs fa = fas[fp.x];
        fused_parent<T, K>(tab.prm[fp.x], tab.b[fp.x], fa, fp.y, dsm_fused);
    }
}

// The launch before a single filter's fused update: this frame's measurements into the
// T layout (u, v, d), the per-update counters and the work counter to 0.
template <typename T, int K>
__global__ void k_stage_frame(T* z, const double* zu, const double* zv, const double* zd, int M,
                              unsigned long long* counters, int* work) {
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        z[m * 3 + 0] = (T)zu[m];
        z[m * 3 + 1] = (T)zv[m];
        z[m * 3 + 2] = (K == 3 && zd) ? (T)zd[m] : T(0);
    }
    if (threadIdx.x == 0) {
        counters[4] = 0;
        counters[5] = 0;
        *work = 0;
    }
}

// ---------------------------------------------------------------- parent weights
__device__ double block_reduce_sum(double v, double* s_tmp) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) s_tmp[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += s_tmp[i];
    return r;
}
__device__ double block_reduce_max(double v, double* s_tmp) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) s_tmp[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = -INFINITY;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r = fmax(r, s_tmp[i]);
    return r;
}

// log-domain form of .cu:1845-1875: lw += loglik, normalise; N_eff of the result
__device__ __forceinline__ void weights_body(int N, double* lw, const double* loglik, int apply, double* scal,
                                             unsigned long long* counters) {
    if (threadIdx.x == 0 && counters) counters[2] += 1;   // frames updated
    __shared__ double s_tmp[32];
    double mx = -INFINITY;
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        double v = lw[p] + (apply ? loglik[p] : 0.0);
        lw[p] = v;
        mx = fmax(mx, v);
    }
    mx = block_reduce_max(mx, s_tmp);
    double s = 0;
    for (int p = threadIdx.x; p < N; p += blockDim.x) s += exp(lw[p] - mx);
    s = block_reduce_sum(s, s_tmp);
    const double ls = mx + log(s);
    double ss = 0;
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        double v = lw[p] - ls;
        lw[p] = v;
        double w = exp(v);
        ss += w * w;
    }
    ss = block_reduce_sum(ss, s_tmp);
    if (threadIdx.x == 0) scal[0] = 1.0 / (N * ss);   // computeNeff, .cu:2641-2649
}

__global__ void __launch_bounds__(1024) k_weights(int N, double* lw, const double* loglik, int apply, double* scal,
                                                  unsigned long long* counters) {
    weights_body(N, lw, loglik, apply, scal, counters);
}

template <typename T>
__global__ void __launch_bounds__(1024) k_weights_batch(const __grid_constant__ SlotTable<T> tab, const FrameArgs* fas) {
    const int f = blockIdx.x;
    const Bufs<T>& b = tab.b[f];
    weights_body(tab.prm[f].N, b.lw, b.loglik, fas[f].fixed ? 0 : 1, b.scal, b.counters);
}

// ---------------------------------------------------------------- (e) resample
// Systematic resampling (.cu:2660-2702): r_j = r0 + j/N, index = first i with
// cumulative C_i >= r_j (FP64 block scan), over-run -> argmax; parents and map
// rows are gathered through the src indirection, weights reset to 1/N.
__device__ void block_scan_inclusive(double* data, int N, double* s_tmp) {
    // per-thread contiguous chunk, then a scan of the chunk totals
    const int T = blockDim.x;
    const int per = (N + T - 1) / T;
    const int lo = threadIdx.x * per, hi = min(N, lo + per);
    double run = 0;
    for (int i = lo; i < hi; ++i) { run += data[i]; data[i] = run; }
    // warp-level inclusive scan of chunk totals
    double v = run;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        double t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) s_tmp[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double wv = lane < (T >> 5) ? s_tmp[lane] : 0.0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            double t = __shfl_up_sync(0xffffffffu, wv, o);
            if (lane >= o) wv += t;
        }
        s_tmp[lane] = wv;
    }
    __syncthreads();
    double offset = (v - run) + (warp > 0 ? s_tmp[warp - 1] : 0.0);
    for (int i = lo; i < hi; ++i) data[i] += offset;
    __syncthreads();
}

// gather_ext = false: the parent states are left for k_gather_parents / k_copy_parents
// (the single filter's path: the 96-byte rows are moved by the whole GPU, not one block)
__device__ __forceinline__ void resample_body(const Params& prm, double* lw, double* ext, double* ext_tmp, int* src,
                                              int* src_tmp, double* cum, double* scal, int* flags, int* idx_out,
                                              uint32_t frame, int force, double r0_override,
                                              unsigned long long* counters, bool gather_ext = true) {
    __shared__ double s_tmp[32];
    __shared__ double s_r0;
    __shared__ int s_amax;
    const int N = prm.N;
    double ss = 0;
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        double w = exp(lw[p]);
        cum[p] = w;
        ss += w * w;
    }
    ss = block_reduce_sum(ss, s_tmp);
    const double neff = 1.0 / (N * ss);   // computeNeff, .cu:2641-2649
    if (threadIdx.x == 0) scal[0] = neff;
    if (!force && !(neff < prm.min_neff)) {   // .cu:2656-2657
        if (threadIdx.x == 0) flags[0] = 0;
        return;
    }
    __syncthreads();
    {   // argmax of the weights, first index on ties (the over-run fallback of .cu:2683-2693),
        // as a block reduction: strided scans, then warps, then one warp over the warps
        __shared__ double s_bw[32];
        __shared__ int s_bi[32];
        double best = -1;
        int bi = -1;
        for (int p = threadIdx.x; p < N; p += blockDim.x)
            if (cum[p] > best) { best = cum[p]; bi = p; }   // NaN never wins, as in a serial scan
        auto better = [](double w, int i, double bw, int bj) {
            return i >= 0 && (bj < 0 || w > bw || (w == bw && i < bj));
        };
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ow = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (better(ow, oi, best, bi)) { best = ow; bi = oi; }
        }
        const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
        if (lane == 0) { s_bw[threadIdx.x >> 5] = best; s_bi[threadIdx.x >> 5] = bi; }
        __syncthreads();
        if (threadIdx.x < 32) {
            best = lane < nw ? s_bw[lane] : -1.0;
            bi = lane < nw ? s_bi[lane] : -1;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ow = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (better(ow, oi, best, bi)) { best = ow; bi = oi; }
            }
            if (threadIdx.x == 0) s_amax = bi < 0 ? 0 : bi;
        }
    }
    if (threadIdx.x == 0) {
        if (r0_override >= 0) {
            s_r0 = r0_override * (1.0 / N);
        } else {
            uint32_t w[4];
            philox(0, 0, 0, ctr_word3(frame, ST_RESAMPLE, 0), prm.key0, prm.key1, w);
            s_r0 = u01(w[0]) * (1.0 / N);
        }
    }
    __syncthreads();
    block_scan_inclusive(cum, N, s_tmp);
    const double r0 = s_r0, h = 1.0 / N;
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        double r = r0 + j * h;
        int lo = 0, hi = N;   // first i with cum[i] >= r
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (cum[mid] >= r) hi = mid; else lo = mid + 1;
        }
        int i = lo < N ? lo : s_amax;
        i = i < 0 ? 0 : (i >= N ? N - 1 : i);
        idx_out[j] = i;
        if (gather_ext)
            for (int q = 0; q < 12; ++q) ext_tmp[12 * j + q] = ext[12 * i + q];
        src_tmp[j] = src[i];
    }
    __syncthreads();
    const double lw0 = -log((double)N);
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        if (gather_ext)
            for (int q = 0; q < 12; ++q) ext[12 * j + q] = ext_tmp[12 * j + q];
        src[j] = src_tmp[j];
        lw[j] = lw0;
    }
    if (threadIdx.x == 0) {
        flags[0] = 1;
        if (counters) atomicAdd(&counters[3], 1ull);
    }
}

__global__ void __launch_bounds__(1024) k_resample(__grid_constant__ const Params prm, double* lw, double* ext,
                                                   double* ext_tmp, int* src, int* src_tmp, double* cum, double* scal,
                                                   int* flags, int* idx_out, uint32_t frame, int force,
                                                   double r0_override, unsigned long long* counters, int gather_ext) {
    resample_body(prm, lw, ext, ext_tmp, src, src_tmp, cum, scal, flags, idx_out, frame, force, r0_override, counters,
                  gather_ext != 0);
}

// The resampled parents' states, for a k_resample launch with gather_ext = 0: one thread
// per state value, ext_tmp[j] = ext[idx[j]], then ext = ext_tmp (when flags[0] says the
// step resampled; otherwise both return at once)
__global__ void k_gather_parents(const int* flags, const int* idx, const double* ext, double* ext_tmp, int N) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (!flags[0] || e >= 12 * N) return;
    const int j = e / 12;
    ext_tmp[e] = ext[12 * idx[j] + (e - 12 * j)];
}
__global__ void k_copy_parents(const int* flags, const double* ext_tmp, double* ext, int N) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (!flags[0] || e >= 12 * N) return;
    ext[e] = ext_tmp[e];
}

template <typename T>
__global__ void __launch_bounds__(1024) k_resample_batch(const __grid_constant__ SlotTable<T> tab, const FrameArgs* fas) {
    const int f = blockIdx.x;
    const Bufs<T>& b = tab.b[f];
    resample_body(tab.prm[f], b.lw, b.ext, b.ext_tmp, b.src, b.src_tmp, b.cum, b.scal, b.flags, b.resample_idx,
                  fas[f].frame, 0, -1.0, b.counters);
}

// map entry: (filter, first parent of a 256-parent block).  The first block of each
// filter also resets its per-update counters and converts its frame's measurements
// into the T layout (u, v, d) for the fused update; block 0 resets the group's work
// counter (may be null).
template <typename T>
__global__ void k_predict_parents_batch(const __grid_constant__ SlotTable<T> tab, const FrameArgs* fas, const int2* map,
                                        int* work) {
    const int2 fp = map[blockIdx.x];
    const Bufs<T>& b = tab.b[fp.x];
    const FrameArgs& fa = fas[fp.x];
    if (fp.y == 0) {
        if (threadIdx.x == 0) {   // counters of "the last update" start at 0
            b.counters[4] = 0;
            b.counters[5] = 0;
        }
        if (fa.zu != nullptr) {
            const int K = tab.prm[fp.x].K;
            for (int m = threadIdx.x; m < fa.M; m += blockDim.x) {
                b.z[m * 3 + 0] = (T)fa.zu[m];
                b.z[m * 3 + 1] = (T)fa.zv[m];
                b.z[m * 3 + 2] = (K == 3 && fa.zd) ? (T)fa.zd[m] : T(0);
            }
        }
    }
    if (work != nullptr && blockIdx.x == 0 && threadIdx.x == 0) *work = 0;
    predict_parents_body(tab.prm[fp.x], b.ext, fa.dt, fa.frame, fp.y + threadIdx.x);
}

// ---------------------------------------------------------------- cloud materialisation
// Write the Euclidean cloud of every entry of the maps into dst (rows p*Gcap + j),
// optionally applying a pending feature prediction (the path of predict() called
// twice without an update, and the cloud dump of scphd_get_map_clouds).
template <typename T>
__global__ void __launch_bounds__(256) k_materialize(Params prm, Bufs<T> b, int cur, T* dst, T* dst_map,
                                                     int* dst_ref, int* dst_n, int has_pred, double dt,
                                                     uint32_t pred_frame, uint32_t sample_frame, int only_p) {
    const int p = only_p >= 0 ? only_p : blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = b.src[p];
    const int G = min(b.map_n[cur][row], prm.Gcap);
    __shared__ Pose<T> pose_src;
    if (threadIdx.x == 0) pose_src = make_pose<T>(b.map_ext[cur] + 12 * row);
    __syncthreads();
    const auto& m = ModelOf<T>::get(prm);   // the constants the cloud fit regenerates samples with
    const int P = prm.P, Ps = prm.Ps;
    for (int j = warp; j < G; j += blockDim.x >> 5) {
        const size_t erow = (size_t)row * prm.Gcap + j;
        const T* ent = b.map[cur] + erow * kRow;
        const int ref = b.map_ref[cur][erow];
        T W = ent[0];
        const T* L = ent + 7;   // merged component: Cholesky factor stored in the map row
        T* cl = dst + ((size_t)(only_p >= 0 ? 0 : p) * prm.Gcap + j) * 7 * Ps;
        for (int s = lane; s < P; s += 32) {
            T X[6], om;
            if (ref < 0) {
                uint32_t w0[4], w1[4];
                const uint32_t key_i = (uint32_t)(-1 - ref);
                philox((uint32_t)s, key_i, (uint32_t)row, ctr_word3(sample_frame, ST_SAMPLE, 0), prm.key0, prm.key1, w0);
                philox((uint32_t)s, key_i, (uint32_t)row, ctr_word3(sample_frame, ST_SAMPLE, 1), prm.key0, prm.key1, w1);
                T z[6];
                Pair<T>::two(w0[0], w0[1], z[0], z[1]);
                Pair<T>::two(w0[2], w0[3], z[2], z[3]);
                Pair<T>::two(w1[0], w1[1], z[4], z[5]);
                T y[6];
                for (int a = 0; a < 6; ++a) {
                    T v = 0;
                    for (int c = 0; c <= a; ++c) v += L[tri(a, c)] * z[c];
                    y[a] = v + ent[1 + a];
                }
                invert(y, pose_src, m, X);
                om = T(1) / T(P);
            } else {
                const T* sc = b.cloud[cur] + (size_t)ref * 7 * Ps;
                for (int a = 0; a < 6; ++a) X[a] = sc[a * Ps + s];
                om = sc[6 * Ps + s];
            }
            if (has_pred) {
                uint32_t w[4];
                philox((uint32_t)s, (uint32_t)j, (uint32_t)p, ctr_word3(pred_frame, ST_FEAT, 0), prm.key0, prm.key1, w);
                T z[4];
                Pair<T>::two(w[0], w[1], z[0], z[1]);
                Pair<T>::two(w[2], w[3], z[2], z[3]);
                const T dtT = (T)dt, half_dt2 = T(0.5) * (T)dt * (T)dt;
                for (int q = 0; q < 3; ++q) {
                    T a = ModelOf<T>::feat_std(prm, q) * z[q];
                    X[q] = X[q] + X[q + 3] * dtT + a * half_dt2;
                    X[q + 3] = X[q + 3] + a * dtT;
                }
            }
            for (int a = 0; a < 6; ++a) cl[a * Ps + s] = X[a];
            cl[6 * Ps + s] = om;
        }
        if (dst_map != nullptr && lane == 0) {
            T* o = dst_map + ((size_t)p * prm.Gcap + j) * kRow;
            o[0] = has_pred ? W * (T)prm.ps : W;
            dst_ref[(size_t)p * prm.Gcap + j] = p * prm.Gcap + j;
        }
    }
    if (dst_n != nullptr && threadIdx.x == 0) dst_n[p] = G;
}

// ---------------------------------------------------------------- stand-alone merge
// phdUpdateMergeKernel on an explicit component list (rows of kRow) with prune flags;
// shared memory as merge_smem_bytes<T>(n_all + 1, 0, 4, false).
template <typename T>
__global__ void __launch_bounds__(128) k_merge_list(const T* rows, const uint8_t* flags_in, int n_all,
                                                    T min_sep, T* sparse, T* out, int* n_out_p, int* member_of) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_n, s_tmp[40];
    if (threadIdx.x == 0) {
        int n = 0;
        for (int i = 0; i < n_all; ++i) n += !flags_in[i];
        s_n = n;
    }
    __syncthreads();
    const int n = s_n;
    const int n_pad = next_pow2(n);
    T* s_w;
    uint32_t* s_key;
    int* s_r;
    int* s_pos;
    MergeScratch<T> ms;
    carve_merge_smem<T>(smem, n_all + 1, 0, false, s_w, s_key, s_r, s_pos, ms);
    if (threadIdx.x == 0) {
        int k = 0;
        for (int i = 0; i < n_all; ++i)
            if (!flags_in[i]) {
                s_w[k] = rows[(size_t)i * kRow];
                s_r[k] = i;
                s_key[k] = tie_key((uint32_t)i);
                ++k;
            }
        for (; k < n_pad; ++k) { s_w[k] = T(-1); s_key[k] = 0xffffffffu; s_r[k] = 0x7fffffff; }
    }
    __syncthreads();
    sort_survivors(s_w, s_key, s_r, n_pad);
    ListView<T> view{rows, s_r};
    const int stop = merge_components<T>(view, s_w, s_r, n, ms, s_key, min_sep, sparse, member_of, nullptr);
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_pos[i] = (i < stop && ms.is_center[i]) ? 1 : 0;
    __syncthreads();
    const int n_out = block_exclusive_scan(s_pos, n, s_tmp);
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (i < stop && ms.is_center[i])
            for (int q = 0; q < 28; ++q) out[(size_t)s_pos[i] * kRow + q] = sparse[(size_t)i * kRow + q];
    __syncthreads();
    // membership: centre index -> output row
    if (member_of)
        for (int i = threadIdx.x; i < n_all; i += blockDim.x) {
            int c = member_of[i];
            member_of[i] = (c >= 0 && c < stop) ? s_pos[c] : -1;
        }
    if (threadIdx.x == 0) *n_out_p = n_out;
}

}  // namespace scphd

// scphd_kernels.cuh — sm_100a kernels of one SC-PHD filter step.
//
// Frame data flow (cur = parity of the map/cloud buffers holding the prior map):
//   k_predict_parents   (a) parent CV motion with noise, FP64            [N threads]
//   k_cloud_fit         (b) per daughter Gaussian, one warp: regenerate (merged
//                           components) or load (non-detection clouds) the sample
//                           cloud, apply the pending feature prediction, transform
//                           world->disparity, pD per sample, refit mean/cov, write
//                           the retained non-detection cloud and the Gaussian's
//                           measurement-independent Kalman terms        [N CTAs]
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
    double kappa, ps, min_weight, min_sep, min_neff;
    double w0, d0, vu0, vv0, vd0, var_d0, var_vu0, var_vv0, var_vd0;
    double cam_std[6], feat_std[3];
    double prior_a[12], prior_b[12];
    uint32_t key0, key1;
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
    T* prep;            // N*Gcap rows of kPrep
    T* z;               // Mcap x 3 measurements
    T* ell;             // N x Mcap normalisers
    int* surv_r;        // N x Scap survivor ranks
    T* surv_w;          // N x Scap survivor weights
    int* surv_n;        // N
    T* merged;          // N x Scap rows of kRow (merge output, in order)
    int* merged_n;      // N
    double* loglik;     // N
    double* cum;        // N resampling prefix
    double* scal;       // [0] neff
    int* flags;         // [0] resampled
    int* resample_idx;  // N
    unsigned long long* counters;   // 8
};

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

__global__ void k_predict_parents(Params prm, double* ext, double dt, uint32_t frame) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
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

// ---------------------------------------------------------------- (b) cloud -> fit
// One CTA per parent, one warp per daughter Gaussian; lane l owns samples
// l, l+32, ... (NS per lane).  Covers: predict_features + ps (.cu:154-178,
// 1144-1150), worldToDisparityKernel + computePdKernel (kernels.cu:6-47, 82-99),
// weight by pD (.cu:1602-1609), normalizeWeightsKernel + fitGaussiansKernel
// (kernels.cu:996-1018, 102-438) and the non-detection copy (.cu:1290-1420).
template <typename T, int K, int NS>
__global__ void __launch_bounds__(256) k_cloud_fit(Params prm, Bufs<T> b, int cur, int M, int fixed,
                                                   int has_pred, double dt, uint32_t pred_frame,
                                                   uint32_t sample_frame) {
    const int p = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = b.src[p];
    const int G = b.map_n[cur][row];
    __shared__ Pose<T> pose_upd, pose_src;
    if (threadIdx.x == 0) {
        double zero[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        pose_upd = make_pose<T>(fixed ? zero : b.ext + 12 * p);
        pose_src = make_pose<T>(b.map_ext[cur] + 12 * row);
        b.surv_n[p] = 0;
        atomicAdd(&b.counters[4], (unsigned long long)G * (unsigned long long)M);
    }
    __syncthreads();
    const Model& m = prm.model;
    const int P = prm.P, Ps = prm.Ps;
    const T invP = T(1) / T(P);
    for (int j = warp; j < G; j += blockDim.x >> 5) {
        const size_t erow = (size_t)row * prm.Gcap + j;
        const T* ent = b.map[cur] + erow * kRow;
        const int ref = b.map_ref[cur][erow];
        T W = ent[0];
        T X[NS][6], om[NS];
        if (ref < 0) {   // merged component: regenerate its sample cloud (.cu:640-690 + :1222-1286)
            T L[21];
            chol6(ent + 7, L);
            const uint32_t key_i = (uint32_t)(-1 - ref);
#pragma unroll
            for (int t = 0; t < NS; ++t) {
                const int s = lane + 32 * t;
                if (s < P) {
                    uint32_t w0[4], w1[4];
                    philox((uint32_t)s, key_i, (uint32_t)row, ctr_word3(sample_frame, ST_SAMPLE, 0), prm.key0, prm.key1, w0);
                    philox((uint32_t)s, key_i, (uint32_t)row, ctr_word3(sample_frame, ST_SAMPLE, 1), prm.key0, prm.key1, w1);
                    T z[8];
                    Normals<T>::four(w0, z);
                    Normals<T>::four(w1, z + 4);
                    T y[6];
#pragma unroll
                    for (int a = 0; a < 6; ++a) {
                        T v = 0;
#pragma unroll
                        for (int c = 0; c <= a; ++c) v += L[tri(a, c)] * z[c];
                        y[a] = v + ent[1 + a];
                    }
                    invert(y, pose_src, m, X[t]);
                    om[t] = invP;
                } else {
#pragma unroll
                    for (int a = 0; a < 6; ++a) X[t][a] = 0;
                    om[t] = 0;
                }
            }
        } else {         // non-detection cloud carried from the previous frame
            const T* cl = b.cloud[cur] + (size_t)ref * 7 * Ps;
#pragma unroll
            for (int t = 0; t < NS; ++t) {
                const int s = lane + 32 * t;
                if (s < P) {
#pragma unroll
                    for (int a = 0; a < 6; ++a) X[t][a] = cl[a * Ps + s];
                    om[t] = cl[6 * Ps + s];
                } else {
#pragma unroll
                    for (int a = 0; a < 6; ++a) X[t][a] = 0;
                    om[t] = 0;
                }
            }
        }
        if (has_pred) {   // predict_features with feature noise, then w *= ps
            W *= (T)prm.ps;
            const T dtT = (T)dt, half_dt2 = T(0.5) * (T)dt * (T)dt;
#pragma unroll
            for (int t = 0; t < NS; ++t) {
                const int s = lane + 32 * t;
                if (s < P) {
                    uint32_t w[4];
                    philox((uint32_t)s, (uint32_t)j, (uint32_t)p, ctr_word3(pred_frame, ST_FEAT, 0), prm.key0, prm.key1, w);
                    T z[4];
                    Normals<T>::four(w, z);
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        T a = (T)prm.feat_std[q] * z[q];
                        X[t][q] = X[t][q] + X[t][q + 3] * dtT + a * half_dt2;
                        X[t][q + 3] = X[t][q + 3] + a * dtT;
                    }
                }
            }
        }
        // world -> disparity, pD per sample, weight by pD
        T y[NS][6], pds[NS];
        T sum_om = 0;
        int n_in = 0;
#pragma unroll
        for (int t = 0; t < NS; ++t) {
            const int s = lane + 32 * t;
            bool valid = s < P;
            if (valid) {
                measure(X[t], pose_upd, m, y[t]);
            } else {
#pragma unroll
                for (int a = 0; a < 6; ++a) y[t][a] = 0;
            }
            bool inr = valid && in_range(y[t], m);
            pds[t] = inr ? (T)m.pd : T(0);
            n_in += __popc(__ballot_sync(0xffffffffu, inr));
            om[t] *= pds[t];
            sum_om += om[t];
        }
        sum_om = warp_sum(sum_om);
        // normalise: exp(safeLog(w) - safeLog(sum)) -> w/sum, 0, or 1 when the sum is 0
        T wsum = 0, wsq = 0, mu[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int t = 0; t < NS; ++t) {
            const int s = lane + 32 * t;
            T w = (s < P) ? ((sum_om > T(0)) ? om[t] / sum_om : T(1)) : T(0);
            om[t] = w;
            wsum += w;
            wsq += w * w;
            if (w != T(0)) {
#pragma unroll
                for (int a = 0; a < 6; ++a) mu[a] += y[t][a] * w;
            }
        }
        wsum = warp_sum(wsum);
        wsq = warp_sum(wsq);
#pragma unroll
        for (int a = 0; a < 6; ++a) mu[a] = warp_sum(mu[a]);
        const T covscale = (wsum * wsum + wsq) / wsum;   // 1 / cov_normalizer (kernels.cu:196)
        T cv[21];
#pragma unroll
        for (int i = 0; i < 21; ++i) cv[i] = 0;
#pragma unroll
        for (int t = 0; t < NS; ++t) {
            if (om[t] == T(0)) continue;
            T dv[6];
#pragma unroll
            for (int a = 0; a < 6; ++a) dv[a] = y[t][a] - mu[a];
#pragma unroll
            for (int a = 0; a < 6; ++a)
#pragma unroll
                for (int c = 0; c <= a; ++c) cv[tri(a, c)] += dv[a] * dv[c] * om[t];
        }
#pragma unroll
        for (int i = 0; i < 21; ++i) cv[i] = warp_sum(cv[i]) * covscale;
        const T pbar = (T)((double)n_in * m.pd / (double)P);
        T* fr = b.fit + ((size_t)p * prm.Gcap + j) * kRow;
        if (lane == 0) {
            fr[0] = W;
            fr[1] = pbar;
#pragma unroll
            for (int a = 0; a < 6; ++a) fr[2 + a] = mu[a];
#pragma unroll
            for (int i = 0; i < 21; ++i) fr[8 + i] = cv[i];
        }
        __syncwarp();
        if (lane == 0) {
            T rowbuf[kRow];
            rowbuf[0] = W; rowbuf[1] = pbar;
            for (int a = 0; a < 6; ++a) rowbuf[2 + a] = mu[a];
            for (int i = 0; i < 21; ++i) rowbuf[8 + i] = cv[i];
            T pr[kPrep];
            kalman_prep<T, K>(rowbuf, m, pr);
            T* dst = b.prep + ((size_t)p * prm.Gcap + j) * kPrep;
            for (int i = 0; i < kPrep - 1; ++i) dst[i] = pr[i];
        }
        // retained non-detection cloud: predicted world samples, weights 1 - pD
        const T wnd = W * (T(1) - pbar);
        if (wnd >= (T)prm.min_weight) {
            T* cl = b.cloud[cur ^ 1] + ((size_t)p * prm.Gcap + j) * 7 * Ps;
#pragma unroll
            for (int t = 0; t < NS; ++t) {
                const int s = lane + 32 * t;
                if (s < P) {
#pragma unroll
                    for (int a = 0; a < 6; ++a) cl[a * Ps + s] = X[t][a];
                    cl[6 * Ps + s] = T(1) - pds[t];
                }
            }
        }
    }
}

// ---------------------------------------------------------------- (c) likelihood
// Normaliser ell_{p,m} = logsumexp_j(log w_{j,m}) (+) log(M w0 + kappa)
// (.cu:1729-1768) and survivor compaction: w_{j,m} = exp(log w - ell) >= min_weight
// with a PD posterior (updateKernel, kernels.cu:622-657), births likewise.
template <typename T, int K>
__global__ void __launch_bounds__(128) k_likelihood(Params prm, Bufs<T> b, int cur, int M) {
    const int p = blockIdx.x;
    const int m = blockIdx.y * blockDim.x + threadIdx.x;
    const int G = b.map_n[cur][b.src[p]];
    __shared__ T s_c[128], s_pd[128], s_si[128][6], s_mu[128][3];
    T zm[3] = {0, 0, 0};
    if (m < M) {
#pragma unroll
        for (int a = 0; a < K; ++a) zm[a] = b.z[m * 3 + a];
    }
    const T bpc = (T)log((double)M * prm.w0 + prm.kappa);
    T mx = tneg_inf<T>(), acc = 0;
    for (int j0 = 0; j0 < G; j0 += 128) {
        const int jj = j0 + threadIdx.x;
        if (jj < G) {
            const T* pr = b.prep + ((size_t)p * prm.Gcap + jj) * kPrep;
            const T* fr = b.fit + ((size_t)p * prm.Gcap + jj) * kRow;
            s_c[threadIdx.x] = pr[0];
            s_pd[threadIdx.x] = pr[1];
#pragma unroll
            for (int i = 0; i < 6; ++i) s_si[threadIdx.x][i] = pr[kPrepSi + i];
#pragma unroll
            for (int a = 0; a < 3; ++a) s_mu[threadIdx.x][a] = fr[2 + a];
        }
        __syncthreads();
        const int cnt = min(128, G - j0);
        if (m < M) {
            for (int k = 0; k < cnt; ++k) {
                T c = s_c[k];
                // non-PD posteriors carry weight LOG0 before the normaliser (kernels.cu:597-598)
                if (!(c > tneg_inf<T>()) || s_pd[k] == T(0)) continue;
                T lt = log_term<T, K>(c, s_si[k], s_mu[k], zm);
                if (lt > mx) { acc = acc * texp(mx - lt) + T(1); mx = lt; }
                else acc += texp(lt - mx);
            }
        }
        __syncthreads();
    }
    T ell = bpc;
    if (m < M && mx > tneg_inf<T>()) {
        // (sum_j exp(lt_j)) (+) bpc, evaluated around the larger of the two
        T big = mx > bpc ? mx : bpc;
        ell = big + tlog(acc * texp(mx - big) + texp(bpc - big));
    }
    if (m < M) b.ell[(size_t)p * prm.Mcap + m] = ell;
    // survivors
    const T minw = (T)prm.min_weight;
    const unsigned lane = threadIdx.x & 31;
    for (int j0 = 0; j0 < G; j0 += 128) {
        const int jj = j0 + threadIdx.x;
        if (jj < G) {
            const T* pr = b.prep + ((size_t)p * prm.Gcap + jj) * kPrep;
            const T* fr = b.fit + ((size_t)p * prm.Gcap + jj) * kRow;
            s_c[threadIdx.x] = pr[0];
            s_pd[threadIdx.x] = pr[1];
#pragma unroll
            for (int i = 0; i < 6; ++i) s_si[threadIdx.x][i] = pr[kPrepSi + i];
#pragma unroll
            for (int a = 0; a < 3; ++a) s_mu[threadIdx.x][a] = fr[2 + a];
        }
        __syncthreads();
        const int cnt = min(128, G - j0);
        for (int k = 0; k < cnt; ++k) {
            bool keep = false;
            T w = 0;
            if (m < M) {
                T c = s_c[k];
                if (c > tneg_inf<T>() && s_pd[k] > T(0)) {
                    w = texp(log_term<T, K>(c, s_si[k], s_mu[k], zm) - ell);
                    keep = w >= minw;
                }
            }
            unsigned mask = __ballot_sync(0xffffffffu, keep);
            if (mask) {
                int base = 0;
                if (lane == 0) base = atomicAdd(&b.surv_n[p], __popc(mask));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (keep) {
                    int slot = base + __popc(mask & ((1u << lane) - 1u));
                    if (slot < prm.Scap) {
                        b.surv_r[(size_t)p * prm.Scap + slot] = m * G + (j0 + k);
                        b.surv_w[(size_t)p * prm.Scap + slot] = w;
                    } else {
                        atomicAdd(&b.counters[1], 1ull);
                    }
                }
            }
        }
        __syncthreads();
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

// ---------------------------------------------------------------- (d) merge
// Component sources for the merge loop: posterior components of one parent
// (detections and births), or an explicit list.
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
    __device__ const T* cov(int r) const {
        if (r < G * M) {
            int j = r % G;
            return prep + (size_t)j * kPrep + kPrepCov;
        }
        return bcov;
    }
};

template <typename T> struct ListSource {
    const T* rows;   // n rows of kRow
    __device__ void mean(int r, T mu[6]) const {
#pragma unroll
        for (int a = 0; a < 6; ++a) mu[a] = rows[(size_t)r * kRow + 1 + a];
    }
    __device__ const T* cov(int r) const { return rows + (size_t)r * kRow + 7; }
};

template <typename T> __device__ __forceinline__ bool merge_before(T wa, uint32_t ka, T wb, uint32_t kb) {
    return wa > wb || (wa == wb && ka < kb);
}

// In-place bitonic sort of (w, key, r) by merge_before over n_pad (power of 2) slots.
template <typename T>
__device__ void sort_survivors(T* s_w, uint32_t* s_key, int* s_r, int n_pad) {
    for (int k = 2; k <= n_pad; k <<= 1) {
        for (int jj = k >> 1; jj > 0; jj >>= 1) {
            for (int i = threadIdx.x; i < n_pad; i += blockDim.x) {
                int ixj = i ^ jj;
                if (ixj > i) {
                    bool up = (i & k) == 0;
                    bool before = merge_before(s_w[ixj], s_key[ixj], s_w[i], s_key[i]);
                    if (before == up) {
                        T tw = s_w[i]; s_w[i] = s_w[ixj]; s_w[ixj] = tw;
                        uint32_t tk = s_key[i]; s_key[i] = s_key[ixj]; s_key[ixj] = tk;
                        int tr = s_r[i]; s_r[i] = s_r[ixj]; s_r[ixj] = tr;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Greedy reduction of phdUpdateMergeKernel (src/kernels.cu:693-866) over n sorted
// survivors: the next centre is the first unmerged one in sorted order (the
// reference's argmax sequence), every unmerged survivor within squared
// Mahalanobis distance < min_sep of the centre (covariance sum) is absorbed, the
// moment-matched result is kept if PD, else the centre.  A diagonal bound
// (x' A^-1 x >= x_k^2 / A_kk for SPD A) skips the full distance for pairs that
// cannot merge; pairs within a safety margin of the bound are evaluated fully.
// Outputs rows of kRow to out[0..), returns the count.  Block-wide call.
template <typename T, typename Src>
__device__ int merge_loop(const Src& src, const T* s_w, const int* s_r, int n, T* s_pf, uint8_t* s_flag,
                          T min_sep, T margin, T* out, int out_cap, int* member_out) {
    __shared__ int s_center, s_nmem;
    __shared__ T s_cmu[6], s_ccov[21];
    __shared__ T s_acc[28];
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    // prefilter data: mean[0..3) and cov diagonal [0..3) per survivor
    for (int i = tid; i < n; i += blockDim.x) {
        T mu[6];
        src.mean(s_r[i], mu);
        const T* cv = src.cov(s_r[i]);
        s_pf[i * 6 + 0] = mu[0]; s_pf[i * 6 + 1] = mu[1]; s_pf[i * 6 + 2] = mu[2];
        s_pf[i * 6 + 3] = cv[0]; s_pf[i * 6 + 4] = cv[2]; s_pf[i * 6 + 5] = cv[5];
        s_flag[i] = 0;
    }
    __syncthreads();
    int next = 0, n_out = 0;
    while (true) {
        if (tid == 0) {
            while (next < n && s_flag[next]) ++next;
            s_center = next < n ? next : -1;
            s_nmem = 0;
            if (next < n) {
                T mu[6];
                src.mean(s_r[next], mu);
                const T* cv = src.cov(s_r[next]);
                for (int a = 0; a < 6; ++a) s_cmu[a] = mu[a];
                for (int i = 0; i < 21; ++i) s_ccov[i] = cv[i];
            }
        }
        __syncthreads();
        const int c = s_center;
        if (c < 0) break;
        // mark members (flag 2)
        for (int i = tid; i < n; i += blockDim.x) {
            if (s_flag[i]) continue;
            bool cand = true;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                T d = s_cmu[k] - s_pf[i * 6 + k];
                T a = s_ccov[tri(k, k)] + s_pf[i * 6 + 3 + k];
                cand = cand && (d * d <= min_sep * a * margin);
            }
            if (!cand) continue;
            T mu[6];
            src.mean(s_r[i], mu);
            T dist = mahal6(s_cmu, s_ccov, mu, src.cov(s_r[i]));
            if (dist < min_sep) {
                s_flag[i] = 2;
                atomicAdd(&s_nmem, 1);
            }
        }
        __syncthreads();
        // no member (not even the centre itself, e.g. a NaN distance): the reference's
        // merged weight is 0 and its loop ends (kernels.cu:783-784)
        if (s_nmem == 0) break;
        if (warp == 0) {
            // pass 1: weight and mean, members in index order
            T accw = 0, accm = 0;   // lane a < 6 accumulates mean[a]
            for (int base = 0; base < n; base += 32) {
                int i = base + lane;
                unsigned mask = __ballot_sync(0xffffffffu, i < n && s_flag[i] == 2);
                while (mask) {
                    int l = __ffs(mask) - 1;
                    mask &= mask - 1;
                    int ii = base + l;
                    T w = s_w[ii];
                    T mu[6];
                    src.mean(s_r[ii], mu);
                    accw += w;
                    if (lane < 6) accm += w * mu[lane];
                }
            }
            T W = accw;
            T mean_l = (lane < 6) ? accm / W : T(0);
            if (lane < 6) s_acc[1 + lane] = mean_l;
            __syncwarp();
            T mean[6];
#pragma unroll
            for (int a = 0; a < 6; ++a) mean[a] = s_acc[1 + a];
            // pass 2: covariance (lane e < 21 owns packed entry e)
            int ea = 0, eb = 0;
            if (lane < 21) { ea = 0; while ((ea + 1) * (ea + 2) / 2 <= lane) ++ea; eb = lane - ea * (ea + 1) / 2; }
            T accc = 0;
            for (int base = 0; base < n; base += 32) {
                int i = base + lane;
                unsigned mask = __ballot_sync(0xffffffffu, i < n && s_flag[i] == 2);
                while (mask) {
                    int l = __ffs(mask) - 1;
                    mask &= mask - 1;
                    int ii = base + l;
                    T w = s_w[ii];
                    if (lane < 21) {
                        T mu[6];
                        src.mean(s_r[ii], mu);
                        const T* cv = src.cov(s_r[ii]);
                        T da = mean[ea] - mu[ea], db = mean[eb] - mu[eb];
                        accc += w * (cv[lane] + da * db);
                    }
                }
                if (i < n && s_flag[i] == 2) {
                    s_flag[i] = 1;
                    if (member_out) member_out[s_r[i]] = n_out;
                }
            }
            if (lane < 21) s_acc[7 + lane] = accc / W;
            __syncwarp();
            if (lane == 0) {
                T row[kRow];
                row[0] = W;
                for (int a = 0; a < 6; ++a) row[1 + a] = mean[a];
                for (int i = 0; i < 21; ++i) row[7 + i] = s_acc[7 + i];
                T L[21];
                bool pd = chol6(row + 7, L);
                T* o = out + (size_t)n_out * kRow;
                if (n_out < out_cap) {
                    if (pd) {
                        for (int i = 0; i < 28; ++i) o[i] = row[i];
                    } else {   // "bad hack, just keep the max feature" (kernels.cu:855-862)
                        o[0] = s_w[c];
                        for (int a = 0; a < 6; ++a) o[1 + a] = s_cmu[a];
                        for (int i = 0; i < 21; ++i) o[7 + i] = s_ccov[i];
                    }
                }
            }
        }
        ++n_out;
        __syncthreads();
    }
    return n_out;
}

template <typename T, int K>
__global__ void __launch_bounds__(128) k_merge(Params prm, Bufs<T> b, int cur, int M, int fixed) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int p = blockIdx.x;
    const int tid = threadIdx.x;
    const int G = b.map_n[cur][b.src[p]];
    const int n = min(b.surv_n[p], prm.Scap);
    int n_pad = 1;
    while (n_pad < n) n_pad <<= 1;
    T* s_w = reinterpret_cast<T*>(smem);
    uint32_t* s_key = reinterpret_cast<uint32_t*>(s_w + 2 * prm.Scap);
    int* s_r = reinterpret_cast<int*>(s_key + 2 * prm.Scap);
    T* s_pf = reinterpret_cast<T*>(s_r + 2 * prm.Scap);
    uint8_t* s_flag = reinterpret_cast<uint8_t*>(s_pf + 6 * prm.Scap);
    for (int i = tid; i < n_pad; i += blockDim.x) {
        if (i < n) {
            s_w[i] = b.surv_w[(size_t)p * prm.Scap + i];
            s_r[i] = b.surv_r[(size_t)p * prm.Scap + i];
            s_key[i] = tie_key((uint32_t)s_r[i]);
        } else {
            s_w[i] = T(-1);
            s_key[i] = 0xffffffffu;
            s_r[i] = 0x7fffffff;
        }
    }
    // parent log-likelihood: sum_m ell + sum_j w_j (.cu:1813-1849), FP64
    __shared__ double s_red[4];
    double part = 0;
    for (int mm = tid; mm < M; mm += blockDim.x) part += (double)b.ell[(size_t)p * prm.Mcap + mm];
    for (int j = tid; j < G; j += blockDim.x) part += (double)b.fit[((size_t)p * prm.Gcap + j) * kRow];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((tid & 31) == 0) s_red[tid >> 5] = part;
    __syncthreads();
    if (tid == 0) b.loglik[p] = s_red[0] + s_red[1] + s_red[2] + s_red[3];
    sort_survivors(s_w, s_key, s_r, n_pad);
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
    T* out = b.merged + (size_t)p * prm.Scap * kRow;
    const T margin = sizeof(T) == 4 ? T(1.05) : T(1.000001);
    int n_out = merge_loop<T>(src, s_w, s_r, n, s_pf, s_flag, (T)prm.min_sep, margin, out, prm.Scap, nullptr);
    // new map: merged components then retained non-detection clouds (.cu:1923-2058)
    __shared__ int s_nnd, s_total;
    __syncthreads();
    if (tid == 0) {
        int nnd = 0;
        for (int j = 0; j < G; ++j) {
            const T* fr = b.fit + ((size_t)p * prm.Gcap + j) * kRow;
            T wnd = fr[0] * (T(1) - fr[1]);
            nnd += wnd >= (T)prm.min_weight;
        }
        s_nnd = nnd;
        s_total = n_out + nnd;
        b.merged_n[p] = n_out;
    }
    __syncthreads();
    const int total = s_total;
    T thr = T(-1);   // keep every entry with weight > thr, and ties in order, up to Gcap
    int n_ties_keep = 0x7fffffff;
    if (total > prm.Gcap) {
        // weight threshold: the Gcap-th largest weight among all entries
        if (tid == 0) {
            atomicAdd(&b.counters[0], 1ull);
        }
        __shared__ T s_thr;
        __shared__ int s_tie;
        if (tid == 0) {
            // bisection over the weight value
            T lo = 0, hi = 0;
            for (int i = 0; i < n_out; ++i) hi = max(hi, out[(size_t)i * kRow]);
            for (int j = 0; j < G; ++j) {
                const T* fr = b.fit + ((size_t)p * prm.Gcap + j) * kRow;
                T wnd = fr[0] * (T(1) - fr[1]);
                if (wnd >= (T)prm.min_weight) hi = max(hi, wnd);
            }
            for (int it = 0; it < 60; ++it) {
                T mid = (lo + hi) / 2;
                int cnt = 0;
                for (int i = 0; i < n_out; ++i) cnt += out[(size_t)i * kRow] > mid;
                for (int j = 0; j < G; ++j) {
                    const T* fr = b.fit + ((size_t)p * prm.Gcap + j) * kRow;
                    T wnd = fr[0] * (T(1) - fr[1]);
                    cnt += (wnd >= (T)prm.min_weight) && wnd > mid;
                }
                if (cnt >= prm.Gcap) lo = mid; else hi = mid;
            }
            int above = 0;
            for (int i = 0; i < n_out; ++i) above += out[(size_t)i * kRow] > hi;
            for (int j = 0; j < G; ++j) {
                const T* fr = b.fit + ((size_t)p * prm.Gcap + j) * kRow;
                T wnd = fr[0] * (T(1) - fr[1]);
                above += (wnd >= (T)prm.min_weight) && wnd > hi;
            }
            s_thr = hi;
            s_tie = prm.Gcap - above;
        }
        __syncthreads();
        thr = s_thr;
        n_ties_keep = s_tie;
    }
    const int wrow = p;   // the new map lives at row p of the other buffer
    if (tid == 0) {
        int k = 0, ties = 0;
        T* mo = b.map[cur ^ 1] + (size_t)wrow * prm.Gcap * kRow;
        int* mr = b.map_ref[cur ^ 1] + (size_t)wrow * prm.Gcap;
        for (int i = 0; i < n_out && k < prm.Gcap; ++i) {
            T w = out[(size_t)i * kRow];
            bool keep = total <= prm.Gcap || w > thr || (w == thr && ties++ < n_ties_keep);
            if (!keep) continue;
            for (int q = 0; q < 28; ++q) mo[(size_t)k * kRow + q] = out[(size_t)i * kRow + q];
            mr[k] = -1 - i;
            ++k;
        }
        for (int j = 0; j < G && k < prm.Gcap; ++j) {
            const T* fr = b.fit + ((size_t)p * prm.Gcap + j) * kRow;
            T wnd = fr[0] * (T(1) - fr[1]);
            if (!(wnd >= (T)prm.min_weight)) continue;
            bool keep = total <= prm.Gcap || wnd > thr || (wnd == thr && ties++ < n_ties_keep);
            if (!keep) continue;
            mo[(size_t)k * kRow] = wnd;
            mr[k] = p * prm.Gcap + j;
            ++k;
        }
        b.map_n[cur ^ 1][wrow] = k;
        double* me = b.map_ext[cur ^ 1] + 12 * wrow;
        for (int q = 0; q < 12; ++q) me[q] = fixed ? 0.0 : b.ext[12 * p + q];
        atomicAdd(&b.counters[5], (unsigned long long)n);
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
__global__ void __launch_bounds__(1024) k_weights(int N, double* lw, const double* loglik, int apply,
                                                  double* scal) {
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

__global__ void __launch_bounds__(1024) k_resample(Params prm, double* lw, double* ext, double* ext_tmp,
                                                   int* src, int* src_tmp, double* cum, double* scal,
                                                   int* flags, int* idx_out, uint32_t frame, int force,
                                                   double r0_override, unsigned long long* counters) {
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
    if (threadIdx.x == 0) {
        double best = -1;
        int bi = -1;
        for (int p = 0; p < N; ++p)
            if (cum[p] > best) { best = cum[p]; bi = p; }
        s_amax = bi < 0 ? 0 : bi;
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
        for (int q = 0; q < 12; ++q) ext_tmp[12 * j + q] = ext[12 * i + q];
        src_tmp[j] = src[i];
    }
    __syncthreads();
    const double lw0 = -log((double)N);
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        for (int q = 0; q < 12; ++q) ext[12 * j + q] = ext_tmp[12 * j + q];
        src[j] = src_tmp[j];
        lw[j] = lw0;
    }
    if (threadIdx.x == 0) {
        flags[0] = 1;
        if (counters) atomicAdd(&counters[3], 1ull);
    }
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
    const int G = b.map_n[cur][row];
    __shared__ Pose<T> pose_src;
    if (threadIdx.x == 0) pose_src = make_pose<T>(b.map_ext[cur] + 12 * row);
    __syncthreads();
    const Model& m = prm.model;
    const int P = prm.P, Ps = prm.Ps;
    for (int j = warp; j < G; j += blockDim.x >> 5) {
        const size_t erow = (size_t)row * prm.Gcap + j;
        const T* ent = b.map[cur] + erow * kRow;
        const int ref = b.map_ref[cur][erow];
        T W = ent[0];
        T L[21];
        if (ref < 0) chol6(ent + 7, L);
        T* cl = dst + ((size_t)(only_p >= 0 ? 0 : p) * prm.Gcap + j) * 7 * Ps;
        for (int s = lane; s < P; s += 32) {
            T X[6], om;
            if (ref < 0) {
                uint32_t w0[4], w1[4];
                const uint32_t key_i = (uint32_t)(-1 - ref);
                philox((uint32_t)s, key_i, (uint32_t)row, ctr_word3(sample_frame, ST_SAMPLE, 0), prm.key0, prm.key1, w0);
                philox((uint32_t)s, key_i, (uint32_t)row, ctr_word3(sample_frame, ST_SAMPLE, 1), prm.key0, prm.key1, w1);
                T z[8];
                Normals<T>::four(w0, z);
                Normals<T>::four(w1, z + 4);
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
                Normals<T>::four(w, z);
                const T dtT = (T)dt, half_dt2 = T(0.5) * (T)dt * (T)dt;
                for (int q = 0; q < 3; ++q) {
                    T a = (T)prm.feat_std[q] * z[q];
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
template <typename T>
__global__ void __launch_bounds__(128) k_merge_list(const T* rows, const uint8_t* flags_in, int n_all,
                                                    T min_sep, T* out, int* n_out_p, int* member_of) {
    extern __shared__ __align__(16) unsigned char smem[];
    // survivors = unflagged inputs, sorted by the argmax order
    __shared__ int s_n;
    if (threadIdx.x == 0) {
        int n = 0;
        for (int i = 0; i < n_all; ++i) n += !flags_in[i];
        s_n = n;
    }
    __syncthreads();
    const int n = s_n;
    int n_pad = 1;
    while (n_pad < n) n_pad <<= 1;
    T* s_w = reinterpret_cast<T*>(smem);
    uint32_t* s_key = reinterpret_cast<uint32_t*>(s_w + 2 * n_all + 2);
    int* s_r = reinterpret_cast<int*>(s_key + 2 * n_all + 2);
    T* s_pf = reinterpret_cast<T*>(s_r + 2 * n_all + 2);
    uint8_t* s_flag = reinterpret_cast<uint8_t*>(s_pf + 6 * n_all + 6);
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
    ListSource<T> src{rows};
    const T margin = sizeof(T) == 4 ? T(1.05) : T(1.000001);
    // membership: rerun the marking through a per-survivor record of the output row
    int n_out = merge_loop<T>(src, s_w, s_r, n, s_pf, s_flag, min_sep, margin, out, n_all, member_of);
    if (threadIdx.x == 0) *n_out_p = n_out;
}

}  // namespace scphd

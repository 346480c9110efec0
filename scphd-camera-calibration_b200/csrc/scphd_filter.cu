// scphd_filter.cu — host orchestration and C ABI (include/scphd.h) of the B200
// SC-PHD calibration filter.  One handle owns one CUDA stream and one device
// arena sized from the configuration at scphd_create; the step API issues
// kernels only (no allocation, no host synchronisation except where a call
// returns device data to the host).
#include "scphd.h"
#include "scphd_kernels.cuh"

#include <atomic>
#include <cmath>
#include <algorithm>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace scphd;

namespace {

thread_local std::string g_err;
std::atomic<long long> g_launches{0};

scphd_status fail(scphd_status s, const std::string& msg) {
    g_err = msg;
    return s;
}

#define CUDA_TRY(expr)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (expr);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(SCPHD_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define LAUNCHED()                                                                              \
    do {                                                                                        \
        g_launches.fetch_add(1, std::memory_order_relaxed);                                     \
        cudaError_t e_ = cudaGetLastError();                                                    \
        if (e_ != cudaSuccess) return fail(SCPHD_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
    } while (0)

int round_up(int x, int m) { return (x + m - 1) / m * m; }

// The dynamic shared-memory limit is an attribute of the kernel function, shared by
// every filter, batch and call in the process: it is raised to the device's whole
// opt-in budget (less the kernel's static shared memory), so that no later setting
// for a smaller launch can undercut a larger one.  The limit does not change the
// occupancy of a launch, which follows the bytes that launch asks for.
cudaError_t allow_dynamic_smem(const void* fn) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    return e;
}

struct Arena {
    char* base = nullptr;
    size_t used = 0, cap = 0;
    template <typename X> X* take(size_t n) {
        size_t off = (used + 255) & ~(size_t)255;
        used = off + n * sizeof(X);
        return base ? reinterpret_cast<X*>(base + off) : nullptr;
    }
};

}  // namespace

// error text for the other translation units of the library (not exported)
__attribute__((visibility("hidden"))) scphd_status scphd_fail_internal(scphd_status st, const char* msg) {
    return fail(st, msg);
}

struct scphd_filter {
    scphd_config cfg;
    Params prm;
    cudaStream_t stream = nullptr;
    cudaEvent_t stage_ev = nullptr;
    double* h_stage = nullptr;   // pinned staging of one frame's measurements (3 x Mcap)
    double* d_stage = nullptr;
    int cur = 0;
    uint32_t frame = 0;
    bool pending = false;
    double pending_dt = 0;
    uint32_t pending_frame = 0;
    uint32_t sample_frame[2] = {0, 0};
    int last_M = 0;
    cudaStream_t own_stream = nullptr;   // the handle's stream while the filter is in a batch
    void* batch = nullptr;               // the batch this filter belongs to, if any
    // Launch shapes of the stage kernels that leave every result unchanged, tuned on the
    // first updates that have measurements: threads per merge block, and whether the
    // likelihood runs one block over all of a parent's measurements or 128-thread blocks.
    // Each shape runs twice, the update is timed with events, the fastest is kept.
    struct Shape { int merge_threads; int lik_full; };
    static constexpr int kShapes = 4;
    const Shape shapes[kShapes] = {{kMergeThreads, 1}, {128, 1}, {kMergeThreads, 0}, {128, 0}};
    // The fused update (one launch for the cloud fit, Kalman terms, likelihood and merge
    // of every parent) runs only on request (scphd_set_fused): measured slower than the
    // stage kernels on every workload here.
    int fused_mode = 0;    // 0: stage kernels, 1: fused kernel
    int fused_grid = 0;    // blocks of the fused kernel (the resident capacity); 0 = unavailable
    size_t fused_smem = 0;
    bool tuning = true;
    int tune_trials = 0;
    int tune_pending = -1;
    double tune_ms[kShapes] = {0, 0, 0, 0};
    int chosen = 0;
    cudaEvent_t tune_ev[2] = {nullptr, nullptr};
    // Blocks per parent of the cloud fit (the parent's Gaussians dealt out over the warps
    // of all its blocks): 1, 2 or 4, tuned by the cloud-fit launch's own event time (each
    // twice) on the updates with measurements after the first kFitTuneAfter, when the maps
    // have grown (the best split depends on the Gaussians per parent), or fixed by
    // scphd_set_fit_split.  Every split computes the same values.
    static constexpr int kFitSplits = 3, kFitTuneAfter = 16;
    const int fit_splits[kFitSplits] = {1, 2, 4};
    bool fit_tuning = true;
    int fit_seen = 0;   // updates with measurements so far
    int fit_trials = 0, fit_pending = -1, fit_chosen = 0;
    double fit_ms[kFitSplits] = {0, 0, 0};
    cudaEvent_t fit_ev[2] = {nullptr, nullptr};
    // whether the next update takes the fused path (profiling times the stage kernels
    // one by one)
    bool fused_next() const { return fused_mode == 1 && !profiling && fused_grid > 0; }
    // the shape for the next update, and whether it is timed
    int pick_shape(bool can_time, bool& timed) {
        timed = tuning && can_time;
        return timed ? tune_trials % kShapes : chosen;
    }
    // fold in the last timed update (waits for it)
    scphd_status tune_collect() {
        if (fit_pending >= 0) {
            CUDA_TRY(cudaEventSynchronize(fit_ev[1]));
            float ms = 0;
            CUDA_TRY(cudaEventElapsedTime(&ms, fit_ev[0], fit_ev[1]));
            fit_ms[fit_pending] += ms;
            fit_pending = -1;
            if (++fit_trials >= 2 * kFitSplits) {
                fit_tuning = false;
                for (int k = 1; k < kFitSplits; ++k)
                    if (fit_ms[k] < fit_ms[fit_chosen]) fit_chosen = k;
            }
        }
        if (tune_pending < 0) return SCPHD_OK;
        CUDA_TRY(cudaEventSynchronize(tune_ev[1]));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, tune_ev[0], tune_ev[1]));
        tune_ms[tune_pending] += ms;
        tune_pending = -1;
        if (++tune_trials >= 2 * kShapes) {
            tuning = false;
            for (int k = 1; k < kShapes; ++k)
                if (tune_ms[k] < tune_ms[chosen]) chosen = k;
        }
        return SCPHD_OK;
    }
    // opt-in per-stage event timing
    bool profiling = false;
    struct Mark { int stage; cudaEvent_t a, b; };
    std::vector<Mark> marks;
    std::vector<cudaEvent_t> event_pool;
    size_t pool_next = 0;
    double stage_ms[8] = {0};
    long long stage_n[8] = {0};
    cudaEvent_t take_event() {
        if (pool_next >= event_pool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            event_pool.push_back(e);
        }
        return event_pool[pool_next++];
    }
    // begin/end of one stage's launch on the stream (no-ops unless profiling)
    int stage_begin(int stage) {
        if (!profiling) return -1;
        if (marks.size() > 8192) flush_marks();
        Mark m{stage, take_event(), take_event()};
        cudaEventRecord(m.a, stream);
        marks.push_back(m);
        return (int)marks.size() - 1;
    }
    void stage_end(int h) {
        if (h < 0) return;
        cudaEventRecord(marks[h].b, stream);
    }
    void flush_marks() {
        cudaStreamSynchronize(stream);
        for (const Mark& m : marks) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, m.a, m.b) == cudaSuccess) {
                stage_ms[m.stage] += ms;
                stage_n[m.stage] += 1;
            }
        }
        marks.clear();
        pool_next = 0;
    }
    virtual ~scphd_filter() {
        for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
        for (cudaEvent_t e : tune_ev)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : fit_ev)
            if (e) cudaEventDestroy(e);
    }
    virtual scphd_status init() = 0;
    virtual scphd_status predict(double dt) = 0;
    virtual scphd_status update_staged(int M, int fixed) = 0;
    virtual scphd_status resample(int32_t* resampled, bool read_back) = 0;
    virtual scphd_status get_particles(double* st, double* lw) = 0;
    virtual scphd_status get_particles_async(double* st, double* lw) = 0;
    virtual scphd_status get_map_sizes(int32_t* sizes) = 0;
    virtual scphd_status get_map_weights(int p, double* w) = 0;
    virtual scphd_status get_map_clouds(int p, double* xyz, double* om) = 0;
    virtual scphd_status get_mixture(int which, int p, double* out, int32_t* count) = 0;
    virtual scphd_status get_normalizers(double* ell, double* ll) = 0;
    virtual scphd_status get_resample_indices(int32_t* idx) = 0;
    virtual scphd_status set_state(const double* st, const double* lw, const int32_t* sizes, const double* w,
                                   const double* xyz, const double* om) = 0;
    virtual scphd_status get_counters(int64_t* c) = 0;
    virtual scphd_status check() = 0;
};

namespace {

__global__ void k_iota(int* a, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

__global__ void k_reset_src(int* src, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) src[i] = i;
}

template <typename T> class Filter final : public scphd_filter {
public:
    Bufs<T> b{};
    void* arena_ptr = nullptr;
    T* dump = nullptr;        // Gcap x 7 x Ps cloud dump scratch
    size_t merge_smem = 0;
    size_t fit_smem = 0;

    ~Filter() override {
        if (stream) cudaStreamSynchronize(stream);
        if (arena_ptr) cudaFree(arena_ptr);
        if (h_stage) cudaFreeHost(h_stage);
        if (stage_ev) cudaEventDestroy(stage_ev);
        if (stream) cudaStreamDestroy(stream);
    }

    void carve(Arena& a) {
        const size_t N = prm.N, G = prm.Gcap, S = prm.Scap, Mc = prm.Mcap, Ps = prm.Ps;
        b.ext = a.take<double>(N * 12);
        b.ext_tmp = a.take<double>(N * 12);
        b.lw = a.take<double>(N);
        b.src = a.take<int>(N);
        b.src_tmp = a.take<int>(N);
        for (int k = 0; k < 2; ++k) {
            b.map[k] = a.take<T>(N * G * kRow);
            b.map_ref[k] = a.take<int>(N * G);
            b.map_n[k] = a.take<int>(N);
            b.map_ext[k] = a.take<double>(N * 12);
            b.cloud[k] = a.take<T>(N * G * 7 * Ps);
        }
        b.fit = a.take<T>(N * G * kRow);
        b.prep = a.take<T>(N * G * kPrep);
        b.lik = a.take<T>(N * G * kLikTerms);
        b.z = a.take<T>(Mc * 3);
        b.ell = a.take<T>(N * Mc);
        b.surv_r = a.take<int>(N * S);
        b.surv_w = a.take<T>(N * S);
        b.surv_n = a.take<int>(N);
        b.mlist = a.take<int>(N * S);
        b.mtmp = a.take<T>(N * S * kRow);
        b.merged_n = a.take<int>(N);
        b.loglik = a.take<double>(N);
        b.cum = a.take<double>(N);
        b.scal = a.take<double>(4);
        b.flags = a.take<int>(4);
        b.resample_idx = a.take<int>(N);
        b.counters = a.take<unsigned long long>(16);
        dump = a.take<T>(G * 7 * Ps);
        b.fit_n = a.take<int>(N);
        d_stage = a.take<double>(Mc * 3);
    }

    scphd_status init() override {
        CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreate(&tune_ev[0]));
        CUDA_TRY(cudaEventCreate(&tune_ev[1]));
        CUDA_TRY(cudaEventCreate(&fit_ev[0]));
        CUDA_TRY(cudaEventCreate(&fit_ev[1]));
        CUDA_TRY(cudaEventCreateWithFlags(&stage_ev, cudaEventDisableTiming));
        CUDA_TRY(cudaMallocHost(&h_stage, sizeof(double) * 3 * prm.Mcap));
        Arena probe;
        carve(probe);
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, probe.used);
        if (e != cudaSuccess)
            return fail(SCPHD_ERR_CAPACITY, "device arena of " + std::to_string(probe.used) +
                                                " bytes: " + cudaGetErrorString(e));
        arena_ptr = p;
        Arena a;
        a.base = static_cast<char*>(p);
        a.cap = probe.used;
        carve(a);
        CUDA_TRY(cudaMemsetAsync(p, 0, probe.used, stream));
        merge_smem = merge_smem_bytes<T>(prm.Scap, prm.Gcap, kMergeThreads / 32, true);
        fit_smem = cloud_fit_smem_bytes<T>(prm.P);
        // with the kernel's static shared memory (20 KB at most), within 227 KB per block:
        // every particles_per_feature up to 256 fits (FP64 at 256: 147 KB of sample rows)
        if (fit_smem > 200 * 1024)
            return fail(SCPHD_ERR_CAPACITY, "particles_per_feature needs " + std::to_string(fit_smem) +
                                                " bytes of shared memory per cloud-fit block (limit 200 KB)");
        if (merge_smem > 227 * 1024)
            return fail(SCPHD_ERR_CAPACITY, "max_survivors/max_gaussians need " + std::to_string(merge_smem) +
                                                " bytes of shared memory per merge block (limit 227 KB)");
        const void* fused_fn = prm.K == 2 ? (const void*)k_fused<T, 2> : (const void*)k_fused<T, 3>;
        if (prm.K == 2) {
            CUDA_TRY(allow_dynamic_smem((const void*)k_merge<T, 2>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_cloud_fit<T, 2>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_cloud_fit<T, 2, kFitP>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_likelihood<T, 2>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_prep<T, 2>));
        } else {
            CUDA_TRY(allow_dynamic_smem((const void*)k_merge<T, 3>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_cloud_fit<T, 3>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_cloud_fit<T, 3, kFitP>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_likelihood<T, 3>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_prep<T, 3>));
        }
        fused_smem = fused_smem_bytes<T>(prm.P, prm.Gcap, prm.Scap);
        fused_grid = 0;
        if (fused_smem <= 220 * 1024) {   // else the stage kernels only
            CUDA_TRY(allow_dynamic_smem(fused_fn));
            int dev = 0, nsm = 0, occ = 0;
            CUDA_TRY(cudaGetDevice(&dev));
            CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fused_fn, kFusedThreads, fused_smem));
            fused_grid = std::min(prm.N, nsm * occ);
        }
        const int N = prm.N;
        k_prior<<<(N + 255) / 256, 256, 0, stream>>>(prm, b.ext, b.lw);
        LAUNCHED();
        k_iota<<<(N + 255) / 256, 256, 0, stream>>>(b.src, N);
        LAUNCHED();
        CUDA_TRY(cudaStreamSynchronize(stream));
        return SCPHD_OK;
    }

    scphd_status materialize_pending() {
        const int N = prm.N;
        k_materialize<T><<<N, 256, 0, stream>>>(prm, b, cur, b.cloud[cur ^ 1], b.map[cur ^ 1], b.map_ref[cur ^ 1],
                                                 b.map_n[cur ^ 1], 1, pending_dt, pending_frame, sample_frame[cur], -1);
        LAUNCHED();
        cur ^= 1;
        k_reset_src<<<(N + 255) / 256, 256, 0, stream>>>(b.src, N);
        LAUNCHED();
        pending = false;
        return SCPHD_OK;
    }

    scphd_status predict(double dt) override {
        if (pending) {
            scphd_status s = materialize_pending();
            if (s != SCPHD_OK) return s;
        }
        frame++;
        if (frame >= (1u << 20)) return fail(SCPHD_ERR_CAPACITY, "frame counter exhausted (2^20 frames)");
        const int N = prm.N;
        int h = stage_begin(0);
        k_predict_parents<<<(N + 255) / 256, 256, 0, stream>>>(prm, b.ext, dt, frame);
        LAUNCHED();
        stage_end(h);
        pending = true;
        pending_dt = dt;
        pending_frame = frame;
        return SCPHD_OK;
    }

    template <int K> scphd_status update_k(int M, int fixed) {
        const int N = prm.N;
        {
            const scphd_status ts = tune_collect();
            if (ts != SCPHD_OK) return ts;
        }
        bool timed = false;
        const Shape sh = shapes[pick_shape(M > 0, timed)];
        if (timed) CUDA_TRY(cudaEventRecord(tune_ev[0], stream));
        if (fused_next()) {
            k_stage_frame<T, K><<<1, 256, 0, stream>>>(b.z, M > 0 ? d_stage : nullptr, M > 0 ? d_stage + M : nullptr,
                                                       M > 0 ? d_stage + 2 * M : nullptr, M, b.counters, b.flags + 2);
            LAUNCHED();
            const FrameArgs fa{cur, M, fixed, pending ? 1 : 0, pending_dt, pending_frame, sample_frame[cur], frame,
                               nullptr, nullptr, nullptr};
            k_fused<T, K><<<fused_grid, kFusedThreads, fused_smem, stream>>>(prm, b, fa, b.flags + 2);
            LAUNCHED();
        } else {
            CUDA_TRY(cudaMemsetAsync(b.counters + 4, 0, 2 * sizeof(unsigned long long), stream));
            int h = stage_begin(1);
            const double* zs[3] = {M > 0 ? d_stage : nullptr, M > 0 ? d_stage + M : nullptr,
                                   M > 0 ? d_stage + 2 * M : nullptr};
            const bool fit_timed = fit_tuning && M > 0 && fit_seen >= kFitTuneAfter;
            if (M > 0) ++fit_seen;
            const int fs = fit_timed ? fit_trials % kFitSplits : fit_chosen, split = fit_splits[fs];
            if (fit_timed) CUDA_TRY(cudaEventRecord(fit_ev[0], stream));
            if (fit_specialised<T>(prm))
                k_cloud_fit<T, K, kFitP><<<N * split, 256, fit_smem, stream>>>(
                    prm, b, cur, M, fixed, pending ? 1 : 0, pending_dt, pending_frame, sample_frame[cur], zs[0], zs[1],
                    zs[2], split);
            else
                k_cloud_fit<T, K><<<N * split, 256, fit_smem, stream>>>(prm, b, cur, M, fixed, pending ? 1 : 0,
                                                                        pending_dt, pending_frame, sample_frame[cur],
                                                                        zs[0], zs[1], zs[2], split);
            LAUNCHED();
            if (fit_timed) {
                CUDA_TRY(cudaEventRecord(fit_ev[1], stream));
                fit_pending = fs;
            }
            stage_end(h);
            h = stage_begin(6);
            k_prep<T, K><<<N, kPrepThreads, prep_smem_bytes<T>(), stream>>>(prm, b, cur);
            LAUNCHED();
            stage_end(h);
            if (M > 0) {
                const int bs = sh.lik_full ? likelihood_block(M) : 128;
                dim3 grid(N, (M + bs - 1) / bs);
                h = stage_begin(2);
                k_likelihood<T, K><<<grid, bs, likelihood_smem_bytes<T>(prm.Gcap, bs), stream>>>(prm, b, cur, M);
                LAUNCHED();
                stage_end(h);
            }
            h = stage_begin(3);
            k_merge<T, K><<<N, sh.merge_threads, merge_smem, stream>>>(prm, b, cur, M, fixed);
            LAUNCHED();
            stage_end(h);
        }
        pending = false;
        if (timed) {
            CUDA_TRY(cudaEventRecord(tune_ev[1], stream));
            tune_pending = tune_trials % kShapes;
        }
        int h = stage_begin(4);
        k_weights<<<1, 1024, 0, stream>>>(N, b.lw, b.loglik, fixed ? 0 : 1, b.scal, b.counters);
        LAUNCHED();
        stage_end(h);
        return SCPHD_OK;
    }

    // one update: the kernels convert the staged measurements, record the fitted
    // counts, reset the src indirection and count the frame themselves
    scphd_status update_staged(int M, int fixed) override {
        scphd_status s = prm.K == 2 ? update_k<2>(M, fixed) : update_k<3>(M, fixed);
        if (s != SCPHD_OK) return s;
        cur ^= 1;
        sample_frame[cur] = frame;
        last_M = M;
        return SCPHD_OK;
    }

    scphd_status resample(int32_t* resampled, bool read_back) override {
        int h = stage_begin(5);
        k_resample<<<1, 1024, 0, stream>>>(prm, b.lw, b.ext, b.ext_tmp, b.src, b.src_tmp, b.cum, b.scal, b.flags,
                                           b.resample_idx, frame, 0, -1.0, b.counters, 0);
        LAUNCHED();
        const int ng = (12 * prm.N + 255) / 256;
        k_gather_parents<<<ng, 256, 0, stream>>>(b.flags, b.resample_idx, b.ext, b.ext_tmp, prm.N);
        LAUNCHED();
        k_copy_parents<<<ng, 256, 0, stream>>>(b.flags, b.ext_tmp, b.ext, prm.N);
        LAUNCHED();
        stage_end(h);
        if (read_back) {
            int f = 0;
            CUDA_TRY(cudaMemcpyAsync(&f, b.flags, sizeof(int), cudaMemcpyDeviceToHost, stream));
            CUDA_TRY(cudaStreamSynchronize(stream));
            if (resampled) *resampled = f;
        }
        return SCPHD_OK;
    }

    scphd_status get_particles(double* st, double* lw) override {
        const scphd_status s = get_particles_async(st, lw);
        if (s != SCPHD_OK) return s;
        CUDA_TRY(cudaStreamSynchronize(stream));
        return SCPHD_OK;
    }
    scphd_status get_particles_async(double* st, double* lw) override {
        if (st) CUDA_TRY(cudaMemcpyAsync(st, b.ext, sizeof(double) * 12 * prm.N, cudaMemcpyDeviceToHost, stream));
        if (lw) CUDA_TRY(cudaMemcpyAsync(lw, b.lw, sizeof(double) * prm.N, cudaMemcpyDeviceToHost, stream));
        return SCPHD_OK;
    }

    scphd_status host_rows(std::vector<int>& src, std::vector<int>& n) {
        src.resize(prm.N);
        n.resize(prm.N);
        CUDA_TRY(cudaMemcpyAsync(src.data(), b.src, sizeof(int) * prm.N, cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaMemcpyAsync(n.data(), b.map_n[cur], sizeof(int) * prm.N, cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return SCPHD_OK;
    }

    scphd_status get_map_sizes(int32_t* sizes) override {
        std::vector<int> src, n;
        scphd_status s = host_rows(src, n);
        if (s != SCPHD_OK) return s;
        for (int p = 0; p < prm.N; ++p) sizes[p] = n[src[p]];
        return SCPHD_OK;
    }

    scphd_status get_map_weights(int p, double* w) override {
        std::vector<int> src, n;
        scphd_status s = host_rows(src, n);
        if (s != SCPHD_OK) return s;
        const int row = src[p], G = n[row];
        std::vector<T> rows((size_t)G * kRow);
        if (G) {
            CUDA_TRY(cudaMemcpyAsync(rows.data(), b.map[cur] + (size_t)row * prm.Gcap * kRow, sizeof(T) * G * kRow,
                                     cudaMemcpyDeviceToHost, stream));
            CUDA_TRY(cudaStreamSynchronize(stream));
        }
        const T ps = pending ? (T)prm.ps : T(1);
        for (int j = 0; j < G; ++j) w[j] = (double)(rows[(size_t)j * kRow] * ps);
        return SCPHD_OK;
    }

    scphd_status get_map_clouds(int p, double* xyz, double* om) override {
        std::vector<int> src, n;
        scphd_status s = host_rows(src, n);
        if (s != SCPHD_OK) return s;
        const int G = n[src[p]], P = prm.P, Ps = prm.Ps;
        if (G == 0) return SCPHD_OK;
        k_materialize<T><<<1, 256, 0, stream>>>(prm, b, cur, dump, nullptr, nullptr, nullptr, pending ? 1 : 0,
                                                 pending_dt, pending_frame, sample_frame[cur], p);
        LAUNCHED();
        std::vector<T> h((size_t)G * 7 * Ps);
        CUDA_TRY(cudaMemcpyAsync(h.data(), dump, sizeof(T) * h.size(), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        for (int j = 0; j < G; ++j)
            for (int s2 = 0; s2 < P; ++s2) {
                for (int a = 0; a < 6; ++a)
                    if (xyz) xyz[((size_t)j * 6 + a) * P + s2] = (double)h[((size_t)j * 7 + a) * Ps + s2];
                if (om) om[(size_t)j * P + s2] = (double)h[((size_t)j * 7 + 6) * Ps + s2];
            }
        return SCPHD_OK;
    }

    scphd_status get_mixture(int which, int p, double* out, int32_t* count) override {
        int cnt = 0;
        const T* base;
        int width;
        if (which == SCPHD_MIX_FITTED) {
            CUDA_TRY(cudaMemcpyAsync(&cnt, b.fit_n + p, sizeof(int), cudaMemcpyDeviceToHost, stream));
            base = b.fit + (size_t)p * prm.Gcap * kRow;
            width = 29;
        } else if (which == SCPHD_MIX_MERGED) {
            // merged rows stay where the merge wrote them, listed in output order
            CUDA_TRY(cudaMemcpyAsync(&cnt, b.merged_n + p, sizeof(int), cudaMemcpyDeviceToHost, stream));
            CUDA_TRY(cudaStreamSynchronize(stream));
            if (count) *count = cnt;
            if (!out || cnt == 0) return SCPHD_OK;
            std::vector<int> list(cnt);
            std::vector<T> rows((size_t)prm.Scap * kRow);
            CUDA_TRY(cudaMemcpyAsync(list.data(), b.mlist + (size_t)p * prm.Scap, sizeof(int) * cnt,
                                     cudaMemcpyDeviceToHost, stream));
            CUDA_TRY(cudaMemcpyAsync(rows.data(), b.mtmp + (size_t)p * prm.Scap * kRow, sizeof(T) * rows.size(),
                                     cudaMemcpyDeviceToHost, stream));
            CUDA_TRY(cudaStreamSynchronize(stream));
            for (int i = 0; i < cnt; ++i) {
                if (list[i] < 0 || list[i] >= prm.Scap) return fail(SCPHD_ERR_INVALID, "corrupt merged list");
                for (int q = 0; q < 28; ++q) out[(size_t)i * 28 + q] = (double)rows[(size_t)list[i] * kRow + q];
            }
            return SCPHD_OK;
        } else {
            return fail(SCPHD_ERR_INVALID, "unknown mixture selector");
        }
        CUDA_TRY(cudaStreamSynchronize(stream));
        if (count) *count = cnt;
        if (!out || cnt == 0) return SCPHD_OK;
        std::vector<T> rows((size_t)cnt * kRow);
        CUDA_TRY(cudaMemcpyAsync(rows.data(), base, sizeof(T) * rows.size(), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        for (int i = 0; i < cnt; ++i)
            for (int q = 0; q < width; ++q) out[(size_t)i * width + q] = (double)rows[(size_t)i * kRow + q];
        return SCPHD_OK;
    }

    scphd_status get_normalizers(double* ell, double* ll) override {
        if (ell && last_M > 0) {
            std::vector<T> h((size_t)prm.N * prm.Mcap);
            CUDA_TRY(cudaMemcpyAsync(h.data(), b.ell, sizeof(T) * h.size(), cudaMemcpyDeviceToHost, stream));
            CUDA_TRY(cudaStreamSynchronize(stream));
            for (int p = 0; p < prm.N; ++p)
                for (int m = 0; m < last_M; ++m) ell[(size_t)p * last_M + m] = (double)h[(size_t)p * prm.Mcap + m];
        }
        if (ll) {
            CUDA_TRY(cudaMemcpyAsync(ll, b.loglik, sizeof(double) * prm.N, cudaMemcpyDeviceToHost, stream));
            CUDA_TRY(cudaStreamSynchronize(stream));
        }
        return SCPHD_OK;
    }

    scphd_status get_resample_indices(int32_t* idx) override {
        CUDA_TRY(cudaMemcpyAsync(idx, b.resample_idx, sizeof(int) * prm.N, cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return SCPHD_OK;
    }

    scphd_status set_state(const double* st, const double* lw, const int32_t* sizes, const double* w,
                           const double* xyz, const double* om) override {
        const int N = prm.N, G = prm.Gcap, P = prm.P, Ps = prm.Ps;
        for (int p = 0; p < N; ++p)
            if (sizes[p] < 0 || sizes[p] > G) return fail(SCPHD_ERR_CAPACITY, "map size exceeds max_gaussians");
        CUDA_TRY(cudaStreamSynchronize(stream));
        std::vector<T> cl((size_t)N * G * 7 * Ps, T(0)), mp((size_t)N * G * kRow, T(0));
        std::vector<int> ref((size_t)N * G, 0), n(N), src(N);
        size_t g = 0;
        for (int p = 0; p < N; ++p) {
            n[p] = sizes[p];
            src[p] = p;
            for (int j = 0; j < sizes[p]; ++j, ++g) {
                size_t r = (size_t)p * G + j;
                mp[r * kRow] = (T)w[g];
                ref[r] = (int)r;
                for (int s2 = 0; s2 < P; ++s2) {
                    for (int a = 0; a < 6; ++a) cl[(r * 7 + a) * Ps + s2] = (T)xyz[(g * 6 + a) * P + s2];
                    cl[(r * 7 + 6) * Ps + s2] = (T)om[g * P + s2];
                }
            }
        }
        CUDA_TRY(cudaMemcpy(b.cloud[cur], cl.data(), sizeof(T) * cl.size(), cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(b.map[cur], mp.data(), sizeof(T) * mp.size(), cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(b.map_ref[cur], ref.data(), sizeof(int) * ref.size(), cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(b.map_n[cur], n.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(b.src, src.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(b.ext, st, sizeof(double) * 12 * N, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(b.lw, lw, sizeof(double) * N, cudaMemcpyHostToDevice));
        pending = false;
        return SCPHD_OK;
    }

    scphd_status get_counters(int64_t* c) override {
        unsigned long long h[16];
        CUDA_TRY(cudaMemcpyAsync(h, b.counters, sizeof(h), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        for (int i = 0; i < 16; ++i) c[i] = (int64_t)h[i];
        return SCPHD_OK;
    }

    scphd_status check() override {
        std::vector<double> lw(prm.N);
        CUDA_TRY(cudaMemcpyAsync(lw.data(), b.lw, sizeof(double) * prm.N, cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        for (double v : lw)
            if (std::isnan(v)) return fail(SCPHD_ERR_NAN, "nan weight detected");
        return SCPHD_OK;
    }
};

scphd_status validate(const scphd_config* c) {
    if (!c) return fail(SCPHD_ERR_INVALID, "null config");
    if (c->n_parents < 1 || c->n_parents > (1 << 20)) return fail(SCPHD_ERR_INVALID, "n_parents out of range");
    if (c->particles_per_feature < 1 || c->particles_per_feature > 256)
        return fail(SCPHD_ERR_INVALID, "particles_per_feature must be in [1, 256]");
    if (c->max_gaussians < 1) return fail(SCPHD_ERR_INVALID, "max_gaussians must be >= 1");
    if (c->max_measurements < 1) return fail(SCPHD_ERR_INVALID, "max_measurements must be >= 1");
    if (c->meas_dim != 2 && c->meas_dim != 3) return fail(SCPHD_ERR_INVALID, "meas_dim must be 2 or 3");
    if (c->precision != SCPHD_FP32 && c->precision != SCPHD_FP64) return fail(SCPHD_ERR_INVALID, "bad precision");
    if ((double)c->max_gaussians * c->max_measurements > 2e9) return fail(SCPHD_ERR_INVALID, "G x M too large");
    if (c->baseline == 0 || c->fy == 0) return fail(SCPHD_ERR_INVALID, "baseline and fy must be non-zero");
    if (!(c->min_separation > 0)) return fail(SCPHD_ERR_INVALID, "min_separation must be > 0");
    if (!(c->min_weight > 0)) return fail(SCPHD_ERR_INVALID, "min_weight must be > 0");
    return SCPHD_OK;
}

Params make_params(const scphd_config& c) {
    Params p{};
    p.N = c.n_parents;
    p.P = c.particles_per_feature;
    p.Gcap = c.max_gaussians;
    p.Mcap = c.max_measurements;
    p.Scap = c.max_survivors > 0 ? c.max_survivors : 4 * c.max_gaussians + c.max_measurements;
    p.K = c.meas_dim;
    p.Ps = c.precision == SCPHD_FP64 ? cloud_stride<double>(c.particles_per_feature)
                                     : cloud_stride<float>(c.particles_per_feature);
    p.model.fx = c.fx; p.model.fy = c.fy; p.model.u0 = c.u0; p.model.v0 = c.v0;
    p.model.B = c.baseline; p.model.pd = c.pd;
    p.model.var[0] = c.std_u * c.std_u;
    p.model.var[1] = c.std_v * c.std_v;
    p.model.var[2] = c.std_d * c.std_d;
    p.kappa = c.kappa; p.ps = c.ps; p.min_weight = c.min_weight; p.min_sep = c.min_separation;
    p.min_neff = c.min_neff;
    p.w0 = c.w0; p.d0 = c.d0; p.vu0 = c.vu0; p.vv0 = c.vv0; p.vd0 = c.vd0;
    p.var_d0 = c.var_d0; p.var_vu0 = c.var_vu0; p.var_vv0 = c.var_vv0; p.var_vd0 = c.var_vd0;
    for (int i = 0; i < 6; ++i) p.cam_std[i] = c.cam_std[i];
    for (int i = 0; i < 3; ++i) p.feat_std[i] = c.feat_std[i];
    p.model_f = {(float)p.model.fx, (float)p.model.fy, (float)p.model.u0, (float)p.model.v0, (float)p.model.B,
                 (float)p.model.pd, {(float)p.feat_std[0], (float)p.feat_std[1], (float)p.feat_std[2]}};
    for (int i = 0; i < 12; ++i) { p.prior_a[i] = c.prior_a[i]; p.prior_b[i] = c.prior_b[i]; }
    p.key0 = (uint32_t)c.seed;
    p.key1 = (uint32_t)(c.seed >> 32);
    for (int r = 0; r < kPhiloxRounds; ++r) {   // Philox round keys
        p.rk[2 * r] = p.key0 + 0x9E3779B9u * (uint32_t)r;
        p.rk[2 * r + 1] = p.key1 + 0xBB67AE85u * (uint32_t)r;
    }
    return p;
}

scphd_status stage_host(scphd_filter* f, const double* u, const double* v, const double* d, int32_t n) {
    if (n < 0) return fail(SCPHD_ERR_INVALID, "negative measurement count");
    if (n > f->prm.Mcap) return fail(SCPHD_ERR_CAPACITY, "more measurements than max_measurements");
    if (n > 0 && (!u || !v)) return fail(SCPHD_ERR_INVALID, "null measurement array");
    if (f->prm.K == 3 && n > 0 && !d) return fail(SCPHD_ERR_INVALID, "meas_dim 3 needs the disparity array");
    if (n == 0) return SCPHD_OK;
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(u[i]) || !std::isfinite(v[i]) || (f->prm.K == 3 && !std::isfinite(d[i])))
            return fail(SCPHD_ERR_INVALID, "non-finite measurement");
    CUDA_TRY(cudaEventSynchronize(f->stage_ev));   // previous copy out of the pinned buffer is done
    std::memcpy(f->h_stage, u, sizeof(double) * n);
    std::memcpy(f->h_stage + n, v, sizeof(double) * n);
    if (d) std::memcpy(f->h_stage + 2 * n, d, sizeof(double) * n);
    CUDA_TRY(cudaMemcpyAsync(f->d_stage, f->h_stage, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, f->stream));
    CUDA_TRY(cudaEventRecord(f->stage_ev, f->stream));
    return SCPHD_OK;
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

void scphd_config_defaults(scphd_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->n_parents = 100;
    c->particles_per_feature = 100;
    c->max_gaussians = 256;
    c->max_measurements = 64;
    c->meas_dim = 2;
    c->precision = SCPHD_FP64;
    c->seed = 0x5C9D0000ull;
    const double mean[12] = {0, -50, -3, 0, 0, 0, 0.3927, 0.1, 0, 0, 0, 0};
    const double sd[12] = {0, 0, 3, 0, 0, 0, 0, 0.1, 0, 0, 0, 0};
    for (int i = 0; i < 12; ++i) { c->prior_a[i] = mean[i] - sd[i]; c->prior_b[i] = mean[i] + sd[i]; }
    const double cam[6] = {0, 0, 0.15, 0, 0.001, 0};
    for (int i = 0; i < 6; ++i) c->cam_std[i] = cam[i];
    c->feat_std[0] = 0.05; c->feat_std[1] = 0.05; c->feat_std[2] = 0.1;
    c->fx = -895.6561; c->fy = -891.2656; c->u0 = 400; c->v0 = 300;
    c->std_u = 5; c->std_v = 5; c->std_d = 1; c->pd = 0.95;
    c->kappa = 10.0001 / (600.0 * 600.0);
    c->baseline = 1;
    c->ps = 0.9; c->min_weight = 1e-4; c->min_separation = 6.0; c->min_neff = 0.75;
    c->w0 = 1e-6; c->d0 = 8; c->vu0 = 0; c->vv0 = 0; c->vd0 = 0;
    c->var_d0 = 2; c->var_vu0 = 6; c->var_vv0 = 6; c->var_vd0 = 0.05;
}

scphd_status scphd_device_bytes(const scphd_config* cfg, int64_t* bytes) {
    if (!bytes) return fail(SCPHD_ERR_INVALID, "null output");
    scphd_status s = validate(cfg);
    if (s != SCPHD_OK) return s;
    Arena probe;
    if (cfg->precision == SCPHD_FP64) {
        Filter<double> f;
        f.prm = make_params(*cfg);
        f.carve(probe);
    } else {
        Filter<float> f;
        f.prm = make_params(*cfg);
        f.carve(probe);
    }
    *bytes = (int64_t)probe.used;
    return SCPHD_OK;
}

scphd_status scphd_create(const scphd_config* cfg, scphd_filter** out) {
    if (!out) return fail(SCPHD_ERR_INVALID, "null output handle");
    *out = nullptr;
    scphd_status s = validate(cfg);
    if (s != SCPHD_OK) return s;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SCPHD_ERR_NO_DEVICE, "no CUDA device");
    if (cfg->device < 0 || cfg->device >= ndev) return fail(SCPHD_ERR_INVALID, "device ordinal out of range");
    CUDA_TRY(cudaSetDevice(cfg->device));
    scphd_filter* f = cfg->precision == SCPHD_FP64 ? static_cast<scphd_filter*>(new Filter<double>())
                                                   : static_cast<scphd_filter*>(new Filter<float>());
    f->cfg = *cfg;
    f->prm = make_params(*cfg);
    s = f->init();
    if (s != SCPHD_OK) {
        delete f;
        return s;
    }
    *out = f;
    return SCPHD_OK;
}

scphd_status scphd_destroy(scphd_filter* f) {
    if (!f) return fail(SCPHD_ERR_INVALID, "null handle");
    if (f->batch) return fail(SCPHD_ERR_INVALID, "filter is in a batch: destroy the batch first");
    cudaSetDevice(f->cfg.device);
    delete f;
    return SCPHD_OK;
}

#define HANDLE(f)                                                  \
    do {                                                           \
        if (!(f)) return fail(SCPHD_ERR_INVALID, "null handle");   \
        CUDA_TRY(cudaSetDevice((f)->cfg.device));                  \
    } while (0)

scphd_status scphd_predict(scphd_filter* f, double dt) {
    HANDLE(f);
    if (!std::isfinite(dt)) return fail(SCPHD_ERR_INVALID, "dt must be finite");
    return f->predict(dt);
}

scphd_status scphd_update(scphd_filter* f, const double* u, const double* v, const double* d, int32_t n,
                          int32_t fixed_camera) {
    HANDLE(f);
    scphd_status s = stage_host(f, u, v, d, n);
    if (s != SCPHD_OK) return s;
    return f->update_staged(n, fixed_camera ? 1 : 0);
}

scphd_status scphd_update_device(scphd_filter* f, const double* u, const double* v, const double* d, int32_t n,
                                 int32_t fixed_camera) {
    HANDLE(f);
    if (n < 0) return fail(SCPHD_ERR_INVALID, "negative measurement count");
    if (n > f->prm.Mcap) return fail(SCPHD_ERR_CAPACITY, "more measurements than max_measurements");
    if (f->prm.K == 3 && n > 0 && !d) return fail(SCPHD_ERR_INVALID, "meas_dim 3 needs the disparity array");
    if (n > 0) {
        CUDA_TRY(cudaMemcpyAsync(f->d_stage, u, sizeof(double) * n, cudaMemcpyDeviceToDevice, f->stream));
        CUDA_TRY(cudaMemcpyAsync(f->d_stage + n, v, sizeof(double) * n, cudaMemcpyDeviceToDevice, f->stream));
        if (d) CUDA_TRY(cudaMemcpyAsync(f->d_stage + 2 * n, d, sizeof(double) * n, cudaMemcpyDeviceToDevice, f->stream));
    }
    return f->update_staged(n, fixed_camera ? 1 : 0);
}

scphd_status scphd_resample(scphd_filter* f, int32_t* resampled) {
    HANDLE(f);
    return f->resample(resampled, true);
}

scphd_status scphd_step(scphd_filter* f, double dt, const double* u, const double* v, const double* d, int32_t n,
                        int32_t fixed_camera) {
    HANDLE(f);
    if (!std::isfinite(dt)) return fail(SCPHD_ERR_INVALID, "dt must be finite");
    scphd_status s = stage_host(f, u, v, d, n);
    if (s != SCPHD_OK) return s;
    s = f->predict(dt);
    if (s != SCPHD_OK) return s;
    s = f->update_staged(n, fixed_camera ? 1 : 0);
    if (s != SCPHD_OK) return s;
    return f->resample(nullptr, false);
}

scphd_status scphd_step_device(scphd_filter* f, double dt, const double* u, const double* v, const double* d,
                               int32_t n, int32_t fixed_camera) {
    HANDLE(f);
    if (!std::isfinite(dt)) return fail(SCPHD_ERR_INVALID, "dt must be finite");
    if (n < 0) return fail(SCPHD_ERR_INVALID, "negative measurement count");
    if (n > f->prm.Mcap) return fail(SCPHD_ERR_CAPACITY, "more measurements than max_measurements");
    if (f->prm.K == 3 && n > 0 && !d) return fail(SCPHD_ERR_INVALID, "meas_dim 3 needs the disparity array");
    if (n > 0) {
        CUDA_TRY(cudaMemcpyAsync(f->d_stage, u, sizeof(double) * n, cudaMemcpyDeviceToDevice, f->stream));
        CUDA_TRY(cudaMemcpyAsync(f->d_stage + n, v, sizeof(double) * n, cudaMemcpyDeviceToDevice, f->stream));
        if (d) CUDA_TRY(cudaMemcpyAsync(f->d_stage + 2 * n, d, sizeof(double) * n, cudaMemcpyDeviceToDevice, f->stream));
    }
    scphd_status s = f->predict(dt);
    if (s != SCPHD_OK) return s;
    s = f->update_staged(n, fixed_camera ? 1 : 0);
    if (s != SCPHD_OK) return s;
    return f->resample(nullptr, false);
}

scphd_status scphd_check(scphd_filter* f) {
    HANDLE(f);
    return f->check();
}

scphd_status scphd_synchronize(scphd_filter* f) {
    HANDLE(f);
    CUDA_TRY(cudaStreamSynchronize(f->stream));
    return SCPHD_OK;
}

scphd_status scphd_get_particles(scphd_filter* f, double* states, double* log_weights) {
    HANDLE(f);
    return f->get_particles(states, log_weights);
}

scphd_status scphd_get_particles_async(scphd_filter* f, double* states, double* log_weights) {
    HANDLE(f);
    return f->get_particles_async(states, log_weights);
}

scphd_status scphd_get_map_sizes(scphd_filter* f, int32_t* sizes) {
    HANDLE(f);
    if (!sizes) return fail(SCPHD_ERR_INVALID, "null output");
    return f->get_map_sizes(sizes);
}

scphd_status scphd_get_map_weights(scphd_filter* f, int32_t p, double* weights) {
    HANDLE(f);
    if (p < 0 || p >= f->prm.N || !weights) return fail(SCPHD_ERR_INVALID, "bad parent index or output");
    return f->get_map_weights(p, weights);
}

scphd_status scphd_get_map_clouds(scphd_filter* f, int32_t p, double* xyz, double* omega) {
    HANDLE(f);
    if (p < 0 || p >= f->prm.N) return fail(SCPHD_ERR_INVALID, "bad parent index");
    return f->get_map_clouds(p, xyz, omega);
}

scphd_status scphd_get_mixture(scphd_filter* f, int32_t which, int32_t p, double* out, int32_t* count) {
    HANDLE(f);
    if (p < 0 || p >= f->prm.N) return fail(SCPHD_ERR_INVALID, "bad parent index");
    return f->get_mixture(which, p, out, count);
}

scphd_status scphd_get_normalizers(scphd_filter* f, double* ell, double* loglik) {
    HANDLE(f);
    return f->get_normalizers(ell, loglik);
}

scphd_status scphd_get_resample_indices(scphd_filter* f, int32_t* idx) {
    HANDLE(f);
    if (!idx) return fail(SCPHD_ERR_INVALID, "null output");
    return f->get_resample_indices(idx);
}

scphd_status scphd_set_state(scphd_filter* f, const double* states, const double* log_weights, const int32_t* sizes,
                             const double* weights, const double* clouds, const double* omega) {
    HANDLE(f);
    if (!states || !log_weights || !sizes) return fail(SCPHD_ERR_INVALID, "null state array");
    return f->set_state(states, log_weights, sizes, weights, clouds, omega);
}

scphd_status scphd_get_config(scphd_filter* f, scphd_config* out) {
    if (!f || !out) return fail(SCPHD_ERR_INVALID, "null argument");
    *out = f->cfg;
    return SCPHD_OK;
}

scphd_status scphd_set_autotune(scphd_filter* f, int32_t enable) {
    if (!f) return fail(SCPHD_ERR_INVALID, "null handle");
    if (!enable) {
        f->tuning = false;
        f->tune_pending = -1;
        f->chosen = 0;
        f->fit_tuning = false;
        f->fit_pending = -1;
        f->fit_chosen = 0;
    }
    return SCPHD_OK;
}

scphd_status scphd_set_fit_split(scphd_filter* f, int32_t blocks_per_parent) {
    if (!f) return fail(SCPHD_ERR_INVALID, "null handle");
    for (int k = 0; k < scphd_filter::kFitSplits; ++k)
        if (f->fit_splits[k] == blocks_per_parent) {
            f->fit_tuning = false;
            f->fit_pending = -1;
            f->fit_chosen = k;
            return SCPHD_OK;
        }
    return fail(SCPHD_ERR_INVALID, "blocks_per_parent must be 1, 2 or 4");
}

scphd_status scphd_get_fit_split(scphd_filter* f, int32_t* blocks_per_parent, int32_t* tuned) {
    if (!f) return fail(SCPHD_ERR_INVALID, "null handle");
    if (blocks_per_parent) *blocks_per_parent = f->fit_splits[f->fit_chosen];
    if (tuned) *tuned = f->fit_tuning ? 0 : 1;
    return SCPHD_OK;
}

scphd_status scphd_get_launch_shapes(scphd_filter* f, int32_t* merge_threads, int32_t* likelihood_full,
                                     int32_t* tuned) {
    if (!f) return fail(SCPHD_ERR_INVALID, "null handle");
    const scphd_filter::Shape& sh = f->shapes[f->chosen];
    if (merge_threads) *merge_threads = sh.merge_threads;
    if (likelihood_full) *likelihood_full = sh.lik_full;
    if (tuned) *tuned = f->tuning ? 0 : 1;
    return SCPHD_OK;
}

scphd_status scphd_set_fused(scphd_filter* f, int32_t mode) {
    HANDLE(f);
    if (mode < 0 || mode > 1) return fail(SCPHD_ERR_INVALID, "mode must be 0 or 1");
    if (mode == 1 && f->fused_grid <= 0)
        return fail(SCPHD_ERR_CAPACITY, "the fused kernel needs more shared memory than a block has");
    f->fused_mode = mode;
    return SCPHD_OK;
}

scphd_status scphd_get_fused(scphd_filter* f, int32_t* fused) {
    HANDLE(f);
    if (!fused) return fail(SCPHD_ERR_INVALID, "null output");
    *fused = f->fused_next() ? 1 : 0;
    return SCPHD_OK;
}

scphd_status scphd_get_counters(scphd_filter* f, int64_t counters[16]) {
    HANDLE(f);
    if (!counters) return fail(SCPHD_ERR_INVALID, "null output");
    return f->get_counters(counters);
}

scphd_status scphd_merge_components(const double* comps, const uint8_t* flags, int32_t n, double min_separation,
                                    int32_t precision, double* merged, int32_t* n_out, int32_t* member_of) {
    if (n < 0 || (n > 0 && (!comps || !flags || !merged || !n_out))) return fail(SCPHD_ERR_INVALID, "bad arguments");
    if (n > 2048) return fail(SCPHD_ERR_CAPACITY, "at most 2048 components");
    if (!(min_separation > 0)) return fail(SCPHD_ERR_INVALID, "min_separation must be > 0");
    if (precision != SCPHD_FP32 && precision != SCPHD_FP64)
        return fail(SCPHD_ERR_INVALID, "precision must be SCPHD_FP32 or SCPHD_FP64");
    if (n_out) *n_out = 0;
    if (n == 0) return SCPHD_OK;
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    auto run = [&](auto tag) -> scphd_status {
        using T = decltype(tag);
        std::vector<T> rows((size_t)n * kRow, T(0));
        for (int i = 0; i < n; ++i)
            for (int q = 0; q < 28; ++q) rows[(size_t)i * kRow + q] = (T)comps[(size_t)i * 28 + q];
        T *d_rows = nullptr, *d_out = nullptr;
        uint8_t* d_flags = nullptr;
        int* d_n = nullptr;
        int* d_mem = nullptr;
        size_t smem = merge_smem_bytes<T>(n + 1, 0, 4, false);
        T* d_sparse = nullptr;
        scphd_status st = SCPHD_OK;
        std::vector<T> out((size_t)n * kRow);
        int nout = 0;
        std::vector<int> mem(n, -1);
        do {
            if (cudaMalloc(&d_rows, sizeof(T) * rows.size()) != cudaSuccess ||
                cudaMalloc(&d_out, sizeof(T) * rows.size()) != cudaSuccess ||
                cudaMalloc(&d_flags, n) != cudaSuccess || cudaMalloc(&d_n, sizeof(int)) != cudaSuccess ||
                cudaMalloc(&d_mem, sizeof(int) * n) != cudaSuccess ||
                cudaMalloc(&d_sparse, sizeof(T) * rows.size()) != cudaSuccess) {
                st = fail(SCPHD_ERR_CUDA, "allocation for merge_components failed");
                break;
            }
            // every runtime call is checked: a failed copy or launch must not leave the
            // host reading uninitialised device memory as a result
            auto check = [&](cudaError_t e, const char* what) {
                if (e != cudaSuccess && st == SCPHD_OK)
                    st = fail(SCPHD_ERR_CUDA, std::string("merge_components ") + what + ": " + cudaGetErrorString(e));
                return st == SCPHD_OK;
            };
            if (!check(cudaMemcpy(d_rows, rows.data(), sizeof(T) * rows.size(), cudaMemcpyHostToDevice), "copy in") ||
                !check(cudaMemcpy(d_flags, flags, n, cudaMemcpyHostToDevice), "copy flags") ||
                !check(cudaMemset(d_mem, 0xff, sizeof(int) * n), "memset") ||
                !check(cudaMemset(d_n, 0, sizeof(int)), "memset") ||
                !check(allow_dynamic_smem((const void*)k_merge_list<T>), "shared memory attribute"))
                break;
            k_merge_list<T><<<1, 128, smem>>>(d_rows, d_flags, n, (T)min_separation, d_sparse, d_out, d_n, d_mem);
            g_launches.fetch_add(1, std::memory_order_relaxed);
            if (!check(cudaGetLastError(), "launch") || !check(cudaDeviceSynchronize(), "k_merge_list")) break;
            if (!check(cudaMemcpy(&nout, d_n, sizeof(int), cudaMemcpyDeviceToHost), "copy count") ||
                !check(cudaMemcpy(out.data(), d_out, sizeof(T) * out.size(), cudaMemcpyDeviceToHost), "copy out") ||
                !check(cudaMemcpy(mem.data(), d_mem, sizeof(int) * n, cudaMemcpyDeviceToHost), "copy membership"))
                break;
            if (nout < 0 || nout > n) st = fail(SCPHD_ERR_CUDA, "merge_components: output count out of range");
        } while (0);
        cudaFree(d_rows); cudaFree(d_out); cudaFree(d_flags); cudaFree(d_n); cudaFree(d_mem); cudaFree(d_sparse);
        if (st != SCPHD_OK) return st;
        *n_out = nout;
        for (int i = 0; i < nout; ++i)
            for (int q = 0; q < 28; ++q) merged[(size_t)i * 28 + q] = (double)out[(size_t)i * kRow + q];
        if (member_of)
            for (int i = 0; i < n; ++i) member_of[i] = mem[i];
        return SCPHD_OK;
    };
    (void)dev;
    return precision == SCPHD_FP64 ? run(double()) : run(float());
}

// ---------------------------------------------------------------------------
// Allocation-free merge: all device buffers of one call live in one static
// device array.  Layout (bytes, each part 256-aligned): host input rows as FP64
// (n x 28), prune flags (n), working rows in T (n x kRow), merge output indexed
// by centre (n x kRow), compact output (n x kRow), output converted to FP64
// (n x 28), membership (n int32), output count (int32).  Sized for T = double.
}  // extern "C"

namespace {

constexpr int kStaticMax = SCPHD_STATIC_MERGE_MAX;
constexpr size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffIn = 0;
constexpr size_t kOffFlags = kOffIn + al256((size_t)kStaticMax * 28 * 8);
constexpr size_t kOffRows = kOffFlags + al256(kStaticMax);
constexpr size_t kOffSparse = kOffRows + al256((size_t)kStaticMax * kRow * 8);
constexpr size_t kOffOut = kOffSparse + al256((size_t)kStaticMax * kRow * 8);
constexpr size_t kOffOut28 = kOffOut + al256((size_t)kStaticMax * kRow * 8);
constexpr size_t kOffMember = kOffOut28 + al256((size_t)kStaticMax * 28 * 8);
constexpr size_t kOffCount = kOffMember + al256((size_t)kStaticMax * 4);
constexpr size_t kStaticBytes = kOffCount + 256;

// Device-side scratch of scphd_merge_components_static.  In host code this name is
// only a stand-in for the symbol: the device address comes from
// cudaGetSymbolAddress (static_scratch_ptr below).
static __device__ __align__(256) unsigned char g_static_merge_scratch[kStaticBytes];

std::mutex g_static_mu;
void* g_static_ptr[256] = {nullptr};

// the array's device address on the current device, looked up once per device
scphd_status static_scratch_ptr(unsigned char** out) {
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return fail(SCPHD_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_merge_scratch);
        if (e != cudaSuccess || !p)
            return fail(SCPHD_ERR_CUDA, std::string("cudaGetSymbolAddress(static merge scratch): ") +
                                            cudaGetErrorString(e));
        g_static_ptr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_static_ptr[dev]);
    return SCPHD_OK;
}

template <typename T> __global__ void k_rows_from28(const double* in, int n, T* rows) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * kRow) return;
    int r = i / kRow, q = i - r * kRow;
    rows[i] = q < 28 ? (T)in[(size_t)r * 28 + q] : T(0);
}

template <typename T> __global__ void k_rows_to28(const T* rows, const int* count, double* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *count * 28) return;
    int r = i / 28, q = i - r * 28;
    out[i] = (double)rows[(size_t)r * kRow + q];
}

template <typename T>
scphd_status merge_static_impl(unsigned char* base, const double* comps, const uint8_t* flags, int n,
                               double min_separation, double* merged, int32_t* n_out, int32_t* member_of) {
    double* d_in = reinterpret_cast<double*>(base + kOffIn);
    uint8_t* d_flags = reinterpret_cast<uint8_t*>(base + kOffFlags);
    T* d_rows = reinterpret_cast<T*>(base + kOffRows);
    T* d_sparse = reinterpret_cast<T*>(base + kOffSparse);
    T* d_out = reinterpret_cast<T*>(base + kOffOut);
    double* d_out28 = reinterpret_cast<double*>(base + kOffOut28);
    int* d_mem = reinterpret_cast<int*>(base + kOffMember);
    int* d_cnt = reinterpret_cast<int*>(base + kOffCount);
    CUDA_TRY(cudaMemcpy(d_in, comps, sizeof(double) * 28 * (size_t)n, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d_flags, flags, (size_t)n, cudaMemcpyHostToDevice));
    // the array keeps the previous call's contents: membership must start at -1
    CUDA_TRY(cudaMemset(d_mem, 0xff, sizeof(int) * (size_t)n));
    k_rows_from28<T><<<(n * kRow + 255) / 256, 256>>>(d_in, n, d_rows);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    const size_t smem = merge_smem_bytes<T>(n + 1, 0, 4, false);
    CUDA_TRY(allow_dynamic_smem((const void*)k_merge_list<T>));
    k_merge_list<T><<<1, 128, smem>>>(d_rows, d_flags, n, (T)min_separation, d_sparse, d_out, d_cnt, d_mem);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    k_rows_to28<T><<<(n * 28 + 255) / 256, 256>>>(d_out, d_cnt, d_out28);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    CUDA_TRY(cudaGetLastError());
    int cnt = 0;
    CUDA_TRY(cudaMemcpy(&cnt, d_cnt, sizeof(int), cudaMemcpyDeviceToHost));
    if (cnt < 0 || cnt > n) return fail(SCPHD_ERR_CUDA, "static merge returned an invalid count");
    if (cnt) CUDA_TRY(cudaMemcpy(merged, d_out28, sizeof(double) * 28 * (size_t)cnt, cudaMemcpyDeviceToHost));
    if (member_of) CUDA_TRY(cudaMemcpy(member_of, d_mem, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost));
    *n_out = cnt;
    return SCPHD_OK;
}

}  // namespace

extern "C" {

scphd_status scphd_merge_components_static(const double* comps, const uint8_t* flags, int32_t n,
                                           double min_separation, int32_t precision, double* merged,
                                           int32_t* n_out, int32_t* member_of) {
    if (n < 0 || (n > 0 && (!comps || !flags || !merged || !n_out))) return fail(SCPHD_ERR_INVALID, "bad arguments");
    if (n > kStaticMax)
        return fail(SCPHD_ERR_CAPACITY, "scphd_merge_components_static takes at most " +
                                            std::to_string(kStaticMax) + " components, got " + std::to_string(n));
    if (!(min_separation > 0)) return fail(SCPHD_ERR_INVALID, "min_separation must be > 0");
    if (precision != SCPHD_FP32 && precision != SCPHD_FP64) return fail(SCPHD_ERR_INVALID, "bad precision");
    if (n_out) *n_out = 0;
    if (n == 0) return SCPHD_OK;
    unsigned char* base = nullptr;
    scphd_status s = static_scratch_ptr(&base);
    if (s != SCPHD_OK) return s;
    return precision == SCPHD_FP64 ? merge_static_impl<double>(base, comps, flags, n, min_separation, merged, n_out, member_of)
                                   : merge_static_impl<float>(base, comps, flags, n, min_separation, merged, n_out, member_of);
}

scphd_status scphd_systematic_resample(const double* weights, int32_t n, double u01v, int32_t* idx) {
    if (n < 1 || n > 16 * 1024 * 1024 || !weights || !idx) return fail(SCPHD_ERR_INVALID, "bad arguments");
    Params prm{};
    prm.N = n;
    prm.min_neff = 2.0;
    double *d_lw = nullptr, *d_ext = nullptr, *d_ext_tmp = nullptr, *d_cum = nullptr, *d_scal = nullptr;
    int *d_src = nullptr, *d_src_tmp = nullptr, *d_flags = nullptr, *d_idx = nullptr;
    std::vector<double> lw(n);
    for (int i = 0; i < n; ++i) lw[i] = std::log(weights[i]);
    scphd_status st = SCPHD_OK;
    do {
        if (cudaMalloc(&d_lw, 8 * n) || cudaMalloc(&d_ext, 96 * (size_t)n) || cudaMalloc(&d_ext_tmp, 96 * (size_t)n) ||
            cudaMalloc(&d_cum, 8 * n) || cudaMalloc(&d_scal, 32) || cudaMalloc(&d_src, 4 * n) ||
            cudaMalloc(&d_src_tmp, 4 * n) || cudaMalloc(&d_flags, 16) || cudaMalloc(&d_idx, 4 * n)) {
            st = fail(SCPHD_ERR_CUDA, "allocation for systematic_resample failed");
            break;
        }
        cudaMemcpy(d_lw, lw.data(), 8 * n, cudaMemcpyHostToDevice);
        cudaMemset(d_ext, 0, 96 * (size_t)n);
        cudaMemset(d_src, 0, 4 * n);
        k_resample<<<1, 1024>>>(prm, d_lw, d_ext, d_ext_tmp, d_src, d_src_tmp, d_cum, d_scal, d_flags, d_idx, 0, 1,
                                u01v, nullptr, 1);
        g_launches.fetch_add(1, std::memory_order_relaxed);
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            st = fail(SCPHD_ERR_CUDA, std::string("k_resample: ") + cudaGetErrorString(e));
            break;
        }
        cudaMemcpy(idx, d_idx, 4 * n, cudaMemcpyDeviceToHost);
    } while (0);
    cudaFree(d_lw); cudaFree(d_ext); cudaFree(d_ext_tmp); cudaFree(d_cum); cudaFree(d_scal);
    cudaFree(d_src); cudaFree(d_src_tmp); cudaFree(d_flags); cudaFree(d_idx);
    return st;
}

void* scphd_stream(scphd_filter* f) { return f ? (void*)f->stream : nullptr; }

scphd_status scphd_set_profiling(scphd_filter* f, int32_t enable) {
    HANDLE(f);
    if (!enable && f->profiling) f->flush_marks();
    f->profiling = enable != 0;
    return SCPHD_OK;
}

scphd_status scphd_get_stage_times(scphd_filter* f, double ms[8], int64_t launches[8]) {
    HANDLE(f);
    f->flush_marks();
    for (int i = 0; i < 8; ++i) {
        if (ms) ms[i] = f->stage_ms[i];
        if (launches) launches[i] = f->stage_n[i];
        f->stage_ms[i] = 0;
        f->stage_n[i] = 0;
    }
    return SCPHD_OK;
}

const char* scphd_last_error(void) { return g_err.c_str(); }

int64_t scphd_kernel_launches(void) { return g_launches.load(); }

}  // extern "C"

// ====================================================================== batches
struct scphd_batch {
    cudaStream_t stream = nullptr;
    std::vector<scphd_filter*> fs;
    virtual ~scphd_batch() {}
    virtual scphd_status step(double dt, const scphd_frame* frames, bool device_frames) = 0;
    virtual scphd_status set_fused(int mode) = 0;
    virtual int fused_path() const = 0;
    virtual scphd_status set_fit_split(int blocks_per_parent) = 0;
    virtual void get_fit_split(int32_t* blocks_per_parent, int32_t* tuned) const = 0;
};

namespace {

template <typename T> struct Batch final : scphd_batch {
    // Filters are launched in groups of up to kBatchSlots, each group with its own
    // parameter table and block maps; per group and frame seven launches (one kernel
    // per stage) or four (prediction, the fused update, weights, resampling).
    struct Group {
        int first = 0, count = 0;       // filters [first, first + count)
        SlotTable<T>* tab = nullptr;    // host copy, passed by value at each launch
        int2* map_parent = nullptr; int n_parent = 0;
        int2* map_pred = nullptr;   int n_pred = 0;
        int4* map_lik = nullptr;    int n_lik = 0;
        int* work = nullptr;            // the fused update's work counter
        bool fit_p = false;             // every member has kFitP samples per feature
    };
    int K = 3;
    bool use_graph = false;
    bool captured = false;
    cudaGraphExec_t exec = nullptr;
    // recorded after a step's copies out of the pinned buffers: the next step rewrites
    // them once these copies are done, while the previous step's kernels may still run
    cudaEvent_t copied = nullptr;
    std::vector<Group> groups;
    FrameArgs* h_fa = nullptr;    // pinned, one per filter
    FrameArgs* d_fa = nullptr;
    double* h_stage = nullptr;    // pinned, 3 x Mcap per filter
    double* d_stage = nullptr;
    std::vector<size_t> stage_off;
    size_t stage_total = 0;
    size_t merge_smem = 0;
    size_t fit_smem = 0;
    size_t lik_smem = 0;
    int lik_block = 32;
    // the update path: the stage kernels with 256 or 128 threads per merge block, tuned
    // on the first 4 steps before a graph is captured (twice each; results do not depend
    // on it), or the fused kernel when requested (scphd_batch_set_fused)
    static constexpr int kPaths = 2;
    int path = 0;              // 0, 1: stage kernels (merge 256 / 128 threads)
    int fused_mode = 0;        // 1: the fused kernel instead
    size_t fused_smem = 0;
    int fused_grid = 0;        // 0: the fused kernel is unavailable
    bool tuning = true;
    bool capturing = false;
    int tune_trials = 0, tune_pending = -1;
    double tune_ms[kPaths] = {0, 0};
    int path_now() const {     // the path of the step being enqueued (2: fused)
        if (fused_mode == 1 && fused_grid > 0) return 2;
        return (tuning && !capturing) ? tune_trials % kPaths : path;
    }
    cudaEvent_t tune_ev[2] = {nullptr, nullptr};
    // blocks per parent of the cloud fit, tuned on the first six steps (1, 2, 4, twice
    // each) by the cloud-fit launches' own time, before the graph is captured
    static constexpr int kFitSplits = 3;
    const int fit_splits[kFitSplits] = {1, 2, 4};
    bool fit_tuning = true;
    int fit_trials = 0, fit_pending = -1, fit_chosen = 0;
    double fit_ms[kFitSplits] = {0, 0, 0};
    cudaEvent_t fit_ev[2] = {nullptr, nullptr};
    void* dev_mem = nullptr;

    ~Batch() override {
        if (stream) cudaStreamSynchronize(stream);
        for (cudaEvent_t e : tune_ev)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : fit_ev)
            if (e) cudaEventDestroy(e);
        if (exec) cudaGraphExecDestroy(exec);
        if (copied) cudaEventDestroy(copied);
        if (h_fa) cudaFreeHost(h_fa);
        if (h_stage) cudaFreeHost(h_stage);
        if (dev_mem) cudaFree(dev_mem);
        for (Group& g : groups) delete g.tab;
        for (scphd_filter* f : fs) {   // give the filters their own streams back
            f->stream = f->own_stream;
            f->own_stream = nullptr;
            f->batch = nullptr;
        }
        if (stream) cudaStreamDestroy(stream);
    }

    Filter<T>* filt(size_t i) const { return static_cast<Filter<T>*>(fs[i]); }

    scphd_status init(bool graph) {
        use_graph = graph;
        const int F = (int)fs.size();
        K = fs[0]->prm.K;
        CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreate(&tune_ev[0]));
        CUDA_TRY(cudaEventCreate(&tune_ev[1]));
        CUDA_TRY(cudaEventCreate(&fit_ev[0]));
        CUDA_TRY(cudaEventCreate(&fit_ev[1]));
        std::vector<std::vector<int2>> mp, mpred;
        std::vector<std::vector<int4>> ml;
        stage_off.resize(F);
        for (int f = 0; f < F; ++f) lik_block = std::max(lik_block, likelihood_block(fs[f]->prm.Mcap));
        for (int first = 0; first < F; first += kBatchSlots) {
            Group g;
            g.first = first;
            g.count = std::min(kBatchSlots, F - first);
            g.tab = new SlotTable<T>();
            g.fit_p = true;
            mp.emplace_back();
            mpred.emplace_back();
            ml.emplace_back();
            for (int i = 0; i < g.count; ++i) {
                const Filter<T>* fl = filt(first + i);
                const Params& pr = fl->prm;
                g.tab->prm[i] = pr;
                g.fit_p = g.fit_p && fit_specialised<T>(pr);
                g.tab->b[i] = fl->b;
                for (int q = 0; q < pr.N; ++q) mp.back().push_back(make_int2(i, q));
                for (int q = 0; q < pr.N; q += 256) mpred.back().push_back(make_int2(i, q));
                const int mb = (pr.Mcap + lik_block - 1) / lik_block;
                for (int q = 0; q < pr.N; ++q)
                    for (int k = 0; k < mb; ++k) ml.back().push_back(make_int4(i, q, k, 0));
                stage_off[first + i] = stage_total;
                stage_total += 3 * (size_t)pr.Mcap;
                merge_smem = std::max(merge_smem, merge_smem_bytes<T>(pr.Scap, pr.Gcap, kMergeThreads / 32, true));
                fit_smem = std::max(fit_smem, cloud_fit_smem_bytes<T>(pr.P));
                fused_smem = std::max(fused_smem, fused_smem_bytes<T>(pr.P, pr.Gcap, pr.Scap));
                lik_smem = std::max(lik_smem, likelihood_smem_bytes<T>(pr.Gcap, lik_block));
            }
            g.n_parent = (int)mp.back().size();
            g.n_pred = (int)mpred.back().size();
            g.n_lik = (int)ml.back().size();
            groups.push_back(g);
        }
        Arena probe;
        probe.take<FrameArgs>(F);
        probe.take<double>(stage_total);
        for (size_t gi = 0; gi < groups.size(); ++gi) {
            probe.take<int2>(mp[gi].size());
            probe.take<int2>(mpred[gi].size());
            probe.take<int4>(ml[gi].size());
            probe.take<int>(1);
        }
        CUDA_TRY(cudaMalloc(&dev_mem, probe.used));
        Arena a;
        a.base = static_cast<char*>(dev_mem);
        d_fa = a.take<FrameArgs>(F);
        d_stage = a.take<double>(stage_total);
        for (size_t gi = 0; gi < groups.size(); ++gi) {
            Group& g = groups[gi];
            g.map_parent = a.take<int2>(mp[gi].size());
            g.map_pred = a.take<int2>(mpred[gi].size());
            g.map_lik = a.take<int4>(ml[gi].size());
            g.work = a.take<int>(1);
            CUDA_TRY(cudaMemset(g.work, 0, sizeof(int)));
            CUDA_TRY(cudaMemcpy(g.map_parent, mp[gi].data(), sizeof(int2) * mp[gi].size(), cudaMemcpyHostToDevice));
            CUDA_TRY(cudaMemcpy(g.map_pred, mpred[gi].data(), sizeof(int2) * mpred[gi].size(), cudaMemcpyHostToDevice));
            CUDA_TRY(cudaMemcpy(g.map_lik, ml[gi].data(), sizeof(int4) * ml[gi].size(), cudaMemcpyHostToDevice));
        }
        CUDA_TRY(cudaMallocHost(&h_fa, sizeof(FrameArgs) * F));
        CUDA_TRY(cudaMallocHost(&h_stage, sizeof(double) * std::max<size_t>(stage_total, 1)));
        if (merge_smem > 227 * 1024) return fail(SCPHD_ERR_CAPACITY, "batch merge needs more than 227 KB of shared memory");
        {
            const void* fn = K == 2 ? (const void*)k_fused_batch<T, 2> : (const void*)k_fused_batch<T, 3>;
            fused_grid = 0;
            if (fused_smem <= 220 * 1024) {
                CUDA_TRY(allow_dynamic_smem(fn));
                int dev = 0, nsm = 0, occ = 0;
                CUDA_TRY(cudaGetDevice(&dev));
                CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
                CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kFusedThreads, fused_smem));
                fused_grid = nsm * occ;
            }
        }
        if (K == 2) {
            CUDA_TRY(allow_dynamic_smem((const void*)k_merge_batch<T, 2>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_cloud_fit_batch<T, 2>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_cloud_fit_batch<T, 2, kFitP>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_likelihood_batch<T, 2>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_prep_batch<T, 2>));
        } else {
            CUDA_TRY(allow_dynamic_smem((const void*)k_merge_batch<T, 3>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_cloud_fit_batch<T, 3>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_cloud_fit_batch<T, 3, kFitP>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_likelihood_batch<T, 3>));
            CUDA_TRY(allow_dynamic_smem((const void*)k_prep_batch<T, 3>));
        }
        // members now issue on the batch stream
        for (scphd_filter* f : fs) {
            CUDA_TRY(cudaStreamSynchronize(f->stream));
            f->own_stream = f->stream;
            f->stream = stream;
            f->batch = this;
        }
        return SCPHD_OK;
    }

    // kernels of one frame, stage by stage over the groups
    template <int KK> scphd_status launch_all() {
        const int pth = path_now();
        const bool timed = tuning && !capturing && pth < kPaths;
        if (timed) CUDA_TRY(cudaEventRecord(tune_ev[0], stream));
        for (const Group& g : groups) {
            k_predict_parents_batch<T><<<g.n_pred, 256, 0, stream>>>(*g.tab, d_fa + g.first, g.map_pred,
                                                                     pth == 2 ? g.work : nullptr);
            LAUNCHED();
        }
        if (pth == 2) {
            for (const Group& g : groups) {
                k_fused_batch<T, KK><<<std::min(g.n_parent, fused_grid), kFusedThreads, fused_smem, stream>>>(
                    *g.tab, d_fa + g.first, g.map_parent, g.n_parent, g.work);
                LAUNCHED();
            }
        } else {
            const bool fit_timed = fit_tuning && !capturing;
            const int fsi = fit_timed ? fit_trials % kFitSplits : fit_chosen, split = fit_splits[fsi];
            if (fit_timed) CUDA_TRY(cudaEventRecord(fit_ev[0], stream));
            for (const Group& g : groups) {
                if (g.fit_p)
                    k_cloud_fit_batch<T, KK, kFitP><<<g.n_parent * split, 256, fit_smem, stream>>>(
                        *g.tab, d_fa + g.first, g.map_parent, split);
                else
                    k_cloud_fit_batch<T, KK><<<g.n_parent * split, 256, fit_smem, stream>>>(*g.tab, d_fa + g.first,
                                                                                            g.map_parent, split);
                LAUNCHED();
            }
            if (fit_timed) {
                CUDA_TRY(cudaEventRecord(fit_ev[1], stream));
                fit_pending = fsi;
            }
            for (const Group& g : groups) {
                k_prep_batch<T, KK><<<g.n_parent, kPrepThreads, prep_smem_bytes<T>(), stream>>>(*g.tab, d_fa + g.first,
                                                                                                   g.map_parent);
                LAUNCHED();
            }
            for (const Group& g : groups) {
                k_likelihood_batch<T, KK><<<g.n_lik, lik_block, lik_smem, stream>>>(*g.tab, d_fa + g.first, g.map_lik);
                LAUNCHED();
            }
            const int mt = pth == 1 ? 128 : kMergeThreads;
            for (const Group& g : groups) {
                k_merge_batch<T, KK><<<g.n_parent, mt, merge_smem, stream>>>(*g.tab, d_fa + g.first, g.map_parent);
                LAUNCHED();
            }
        }
        for (const Group& g : groups) {
            k_weights_batch<T><<<g.count, 1024, 0, stream>>>(*g.tab, d_fa + g.first);
            LAUNCHED();
        }
        for (const Group& g : groups) {
            k_resample_batch<T><<<g.count, 1024, 0, stream>>>(*g.tab, d_fa + g.first);
            LAUNCHED();
        }
        if (timed) {
            CUDA_TRY(cudaEventRecord(tune_ev[1], stream));
            tune_pending = tune_trials % kPaths;
        }
        return SCPHD_OK;
    }

    int launches_per_frame() const { return (path_now() == 2 ? 4 : 7) * (int)groups.size(); }

    scphd_status set_fused(int mode) override {
        if (mode < 0 || mode > 1) return fail(SCPHD_ERR_INVALID, "mode must be 0 or 1");
        if (mode == 1 && fused_grid <= 0)
            return fail(SCPHD_ERR_CAPACITY, "the fused kernel needs more shared memory than a block has");
        if (captured) return fail(SCPHD_ERR_INVALID, "the batch's step graph is already captured");
        fused_mode = mode;
        if (mode == 1) tuning = fit_tuning = false;   // the stage kernels' shapes are not needed
        return SCPHD_OK;
    }
    int fused_path() const override { return path_now() == 2 ? 1 : 0; }
    scphd_status set_fit_split(int blocks_per_parent) override {
        if (captured) return fail(SCPHD_ERR_INVALID, "the batch's step graph is already captured");
        for (int k = 0; k < kFitSplits; ++k)
            if (fit_splits[k] == blocks_per_parent) {
                fit_tuning = false;
                fit_pending = -1;
                fit_chosen = k;
                return SCPHD_OK;
            }
        return fail(SCPHD_ERR_INVALID, "blocks_per_parent must be 1, 2 or 4");
    }
    void get_fit_split(int32_t* blocks_per_parent, int32_t* tuned) const override {
        if (blocks_per_parent) *blocks_per_parent = fit_splits[fit_chosen];
        if (tuned) *tuned = fit_tuning ? 0 : 1;
    }

    scphd_status tune_collect() {
        if (fit_pending >= 0) {
            CUDA_TRY(cudaEventSynchronize(fit_ev[1]));
            float ms = 0;
            CUDA_TRY(cudaEventElapsedTime(&ms, fit_ev[0], fit_ev[1]));
            fit_ms[fit_pending] += ms;
            fit_pending = -1;
            if (++fit_trials >= 2 * kFitSplits) {
                fit_tuning = false;
                for (int k = 1; k < kFitSplits; ++k)
                    if (fit_ms[k] < fit_ms[fit_chosen]) fit_chosen = k;
            }
        }
        if (tune_pending < 0) return SCPHD_OK;
        CUDA_TRY(cudaEventSynchronize(tune_ev[1]));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, tune_ev[0], tune_ev[1]));
        tune_ms[tune_pending] += ms;
        tune_pending = -1;
        if (++tune_trials >= 2 * kPaths) {
            tuning = false;
            path = tune_ms[1] < tune_ms[0] ? 1 : 0;
        }
        return SCPHD_OK;
    }

    // the step's measurements and frame arguments to the device, ahead of its kernels on
    // the stream (outside the graph, which holds the kernels only)
    scphd_status copy_in() {
        CUDA_TRY(cudaMemcpyAsync(d_stage, h_stage, sizeof(double) * stage_total, cudaMemcpyHostToDevice, stream));
        CUDA_TRY(cudaMemcpyAsync(d_fa, h_fa, sizeof(FrameArgs) * fs.size(), cudaMemcpyHostToDevice, stream));
        CUDA_TRY(cudaEventRecord(copied, stream));
        return SCPHD_OK;
    }
    scphd_status enqueue() { return K == 2 ? launch_all<2>() : launch_all<3>(); }

    scphd_status step(double dt, const scphd_frame* frames, bool device_frames) override {
        const int F = (int)fs.size();
        for (int f = 0; f < F; ++f) {
            const scphd_frame& fr = frames[f];
            const Params& pr = fs[f]->prm;
            if (fr.n < 0 || fr.n > pr.Mcap)
                return fail(SCPHD_ERR_CAPACITY, "batch frame " + std::to_string(f) + ": bad measurement count");
            if (fr.n > 0 && (!fr.u || !fr.v || (K == 3 && !fr.d)))
                return fail(SCPHD_ERR_INVALID, "batch frame " + std::to_string(f) + ": null measurement array");
            if (!device_frames)
                for (int i = 0; i < fr.n; ++i)
                    if (!std::isfinite(fr.u[i]) || !std::isfinite(fr.v[i]) || (K == 3 && !std::isfinite(fr.d[i])))
                        return fail(SCPHD_ERR_INVALID, "non-finite measurement");
        }
        // the pinned buffers are rewritten: the previous step's copies out of them must be
        // done (its kernels may still run: this step's host work overlaps them)
        CUDA_TRY(cudaEventSynchronize(copied));
        for (int f = 0; f < F; ++f) {
            Filter<T>* fl = filt(f);
            if (fl->pending) {   // a predict() issued outside the batch: apply it first
                scphd_status s = fl->materialize_pending();
                if (s != SCPHD_OK) return s;
            }
            const scphd_frame& fr = frames[f];
            fl->frame++;
            if (fl->frame >= (1u << 20)) return fail(SCPHD_ERR_CAPACITY, "frame counter exhausted (2^20 frames)");
            FrameArgs& fa = h_fa[f];
            fa.cur = fl->cur;
            fa.M = fr.n;
            fa.fixed = fr.fixed_camera ? 1 : 0;
            fa.has_pred = 1;
            fa.dt = dt;
            fa.pred_frame = fl->frame;
            fa.sample_frame = fl->sample_frame[fl->cur];
            fa.frame = fl->frame;
            if (fr.n == 0) {
                fa.zu = fa.zv = fa.zd = nullptr;
            } else if (device_frames) {
                fa.zu = fr.u;
                fa.zv = fr.v;
                fa.zd = K == 3 ? fr.d : nullptr;
            } else {
                double* hs = h_stage + stage_off[f];
                std::memcpy(hs, fr.u, sizeof(double) * fr.n);
                std::memcpy(hs + fr.n, fr.v, sizeof(double) * fr.n);
                if (K == 3) std::memcpy(hs + 2 * fr.n, fr.d, sizeof(double) * fr.n);
                const double* ds = d_stage + stage_off[f];
                fa.zu = ds;
                fa.zv = ds + fr.n;
                fa.zd = K == 3 ? ds + 2 * fr.n : nullptr;
            }
        }
        {
            const scphd_status ts = tune_collect();
            if (ts != SCPHD_OK) return ts;
        }
        {
            const scphd_status cs = copy_in();
            if (cs != SCPHD_OK) return cs;
        }
        if (use_graph && !tuning && !fit_tuning) {
            if (!captured) {
                cudaGraph_t g = nullptr;
                CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
                capturing = true;
                scphd_status s = enqueue();
                capturing = false;
                cudaError_t e = cudaStreamEndCapture(stream, &g);
                if (s != SCPHD_OK) return s;
                if (e != cudaSuccess) return fail(SCPHD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
                e = cudaGraphInstantiate(&exec, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return fail(SCPHD_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
                captured = true;
                // captured, not run: counted at replay
                g_launches.fetch_sub(launches_per_frame(), std::memory_order_relaxed);
            }
            CUDA_TRY(cudaGraphLaunch(exec, stream));
            g_launches.fetch_add(launches_per_frame(), std::memory_order_relaxed);
        } else {
            scphd_status s = enqueue();
            if (s != SCPHD_OK) return s;
        }
        for (int f = 0; f < F; ++f) {
            Filter<T>* fl = filt(f);
            fl->cur ^= 1;
            fl->sample_frame[fl->cur] = fl->frame;
            fl->pending = false;
            fl->last_M = frames[f].n;
        }
        return SCPHD_OK;
    }
};

}  // namespace

extern "C" {

scphd_status scphd_batch_create(scphd_filter* const* filters, int32_t n, int32_t use_graph, scphd_batch** out) {
    if (!out || !filters || n < 1) return fail(SCPHD_ERR_INVALID, "bad batch arguments");
    *out = nullptr;
    const scphd_config& c0 = filters[0]->cfg;
    for (int i = 0; i < n; ++i) {
        if (!filters[i]) return fail(SCPHD_ERR_INVALID, "null filter in batch");
        const scphd_config& c = filters[i]->cfg;
        if (c.device != c0.device || c.precision != c0.precision || c.meas_dim != c0.meas_dim)
            return fail(SCPHD_ERR_INVALID, "batch members must share device, precision and meas_dim");
        if (filters[i]->batch) return fail(SCPHD_ERR_INVALID, "filter already in a batch");
        for (int j = 0; j < i; ++j)
            if (filters[j] == filters[i]) return fail(SCPHD_ERR_INVALID, "filter listed twice");
    }
    CUDA_TRY(cudaSetDevice(c0.device));
    scphd_batch* b = c0.precision == SCPHD_FP64 ? static_cast<scphd_batch*>(new Batch<double>())
                                                : static_cast<scphd_batch*>(new Batch<float>());
    b->fs.assign(filters, filters + n);
    scphd_status s = c0.precision == SCPHD_FP64 ? static_cast<Batch<double>*>(b)->init(use_graph != 0)
                                                : static_cast<Batch<float>*>(b)->init(use_graph != 0);
    if (s != SCPHD_OK) {
        delete b;
        return s;
    }
    *out = b;
    return SCPHD_OK;
}

scphd_status scphd_batch_set_fused(scphd_batch* b, int32_t mode) {
    if (!b) return fail(SCPHD_ERR_INVALID, "null batch");
    return b->set_fused(mode);
}

scphd_status scphd_batch_get_fused(scphd_batch* b, int32_t* fused) {
    if (!b || !fused) return fail(SCPHD_ERR_INVALID, "null batch or output");
    *fused = b->fused_path();
    return SCPHD_OK;
}

scphd_status scphd_batch_set_fit_split(scphd_batch* b, int32_t blocks_per_parent) {
    if (!b) return fail(SCPHD_ERR_INVALID, "null batch");
    return b->set_fit_split(blocks_per_parent);
}

scphd_status scphd_batch_get_fit_split(scphd_batch* b, int32_t* blocks_per_parent, int32_t* tuned) {
    if (!b) return fail(SCPHD_ERR_INVALID, "null batch");
    b->get_fit_split(blocks_per_parent, tuned);
    return SCPHD_OK;
}

scphd_status scphd_batch_destroy(scphd_batch* b) {
    if (!b) return fail(SCPHD_ERR_INVALID, "null batch");
    cudaSetDevice(b->fs[0]->cfg.device);
    delete b;
    return SCPHD_OK;
}

scphd_status scphd_batch_step(scphd_batch* b, double dt, const scphd_frame* frames) {
    if (!b || !frames) return fail(SCPHD_ERR_INVALID, "null batch or frames");
    if (!std::isfinite(dt)) return fail(SCPHD_ERR_INVALID, "dt must be finite");
    CUDA_TRY(cudaSetDevice(b->fs[0]->cfg.device));
    return b->step(dt, frames, false);
}

scphd_status scphd_batch_step_device(scphd_batch* b, double dt, const scphd_frame* frames) {
    if (!b || !frames) return fail(SCPHD_ERR_INVALID, "null batch or frames");
    if (!std::isfinite(dt)) return fail(SCPHD_ERR_INVALID, "dt must be finite");
    CUDA_TRY(cudaSetDevice(b->fs[0]->cfg.device));
    return b->step(dt, frames, true);
}

void* scphd_batch_stream(scphd_batch* b) { return b ? (void*)b->stream : nullptr; }

}  // extern "C"

// Serving loop over the batch API: first-come first-served admission by device
// memory budget, device-resident jobs, one batched step per iteration for every
// resident job, retirement of finished jobs with their results copied out.
// Host code only: it drives the filters through the library's own C ABI.
#include "scphd.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

__attribute__((visibility("hidden"))) scphd_status scphd_fail_internal(scphd_status st, const char* msg);

namespace {

scphd_status fail(scphd_status st, const std::string& m) { return scphd_fail_internal(st, m.c_str()); }

#define SRV_CUDA(expr)                                                                            \
    do {                                                                                          \
        cudaError_t e_ = (expr);                                                                  \
        if (e_ != cudaSuccess) return fail(SCPHD_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)
#define SRV_TRY(expr)                           \
    do {                                        \
        scphd_status s_ = (expr);               \
        if (s_ != SCPHD_OK) return s_;          \
    } while (0)

struct Job {
    int64_t id = 0;
    scphd_config cfg{};
    int n_frames = 0;
    double dt = 0;
    std::vector<int32_t> sizes, fixed;
    std::vector<int64_t> offs;
    std::vector<double> zu, zv, zd;   // host copy until admission
    int64_t bytes = 0;                // filter arena + frame sequence on the device
    int state = SCPHD_JOB_QUEUED;
    int next = 0;                     // frames queued so far
    scphd_filter* f = nullptr;
    double* dz = nullptr;             // device frames: u | v | d, each total long
    int64_t total = 0;
    std::vector<double> states, lw;   // result of a DONE job
    int64_t units = 0;
};

}  // namespace

struct scphd_server {
    int device = 0, precision = 0, meas_dim = 3;
    int64_t budget = 0, used = 0;
    bool use_graph = true;
    bool has_dt = false;
    double dt = 0;
    int64_t next_id = 1;
    std::map<int64_t, std::unique_ptr<Job>> jobs;
    std::deque<Job*> queue;
    std::vector<Job*> running;
    scphd_batch* batch = nullptr;
    bool dirty = true;
    bool in_flight = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int in_flight_jobs = 0;
    std::vector<double> step_ms;
    std::vector<int32_t> step_jobs;
    int64_t steps = 0, frames = 0, units_done = 0, rebuilds = 0;
    std::vector<scphd_frame> fr;

    ~scphd_server() {
        cudaSetDevice(device);
        if (batch) scphd_batch_destroy(batch);
        for (auto& kv : jobs) {
            Job* j = kv.second.get();
            if (j->f) scphd_destroy(j->f);
            if (j->dz) cudaFree(j->dz);
        }
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }

    scphd_status drop_batch() {
        if (batch) {
            SRV_TRY(scphd_batch_destroy(batch));
            batch = nullptr;
        }
        dirty = true;
        return SCPHD_OK;
    }

    // wait for the step in flight, record its time, retire the jobs it finished
    scphd_status complete() {
        if (!in_flight) return SCPHD_OK;
        SRV_CUDA(cudaEventSynchronize(ev1));
        float ms = 0;
        SRV_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        step_ms.push_back(ms);
        step_jobs.push_back(in_flight_jobs);
        in_flight = false;
        std::vector<Job*> keep;
        bool retired = false;
        for (Job* j : running) {
            if (j->next < j->n_frames) {
                keep.push_back(j);
                continue;
            }
            if (!retired) SRV_TRY(drop_batch());   // members leave the batch before they are destroyed
            retired = true;
            j->states.resize((size_t)12 * j->cfg.n_parents);
            j->lw.resize(j->cfg.n_parents);
            SRV_TRY(scphd_get_particles(j->f, j->states.data(), j->lw.data()));
            int64_t c[16];
            SRV_TRY(scphd_get_counters(j->f, c));
            j->units = c[6];
            units_done += c[6];
            SRV_TRY(scphd_destroy(j->f));
            j->f = nullptr;
            SRV_CUDA(cudaFree(j->dz));
            j->dz = nullptr;
            used -= j->bytes;
            j->state = SCPHD_JOB_DONE;
        }
        running.swap(keep);
        return SCPHD_OK;
    }

    scphd_status admit() {
        while (!queue.empty() && used + queue.front()->bytes <= budget) {
            Job* j = queue.front();
            SRV_TRY(scphd_create(&j->cfg, &j->f));
            const size_t nb = sizeof(double) * (size_t)std::max<int64_t>(1, 3 * j->total);
            cudaError_t e = cudaMalloc(&j->dz, nb);
            if (e != cudaSuccess) {
                scphd_destroy(j->f);
                j->f = nullptr;
                return fail(SCPHD_ERR_CUDA, std::string("job frames: ") + cudaGetErrorString(e));
            }
            if (j->total > 0) {
                SRV_CUDA(cudaMemcpy(j->dz, j->zu.data(), sizeof(double) * j->total, cudaMemcpyHostToDevice));
                SRV_CUDA(cudaMemcpy(j->dz + j->total, j->zv.data(), sizeof(double) * j->total, cudaMemcpyHostToDevice));
                if (meas_dim == 3)
                    SRV_CUDA(cudaMemcpy(j->dz + 2 * j->total, j->zd.data(), sizeof(double) * j->total,
                                        cudaMemcpyHostToDevice));
            }
            std::vector<double>().swap(j->zu);   // the device copy is the job's now
            std::vector<double>().swap(j->zv);
            std::vector<double>().swap(j->zd);
            used += j->bytes;
            j->state = SCPHD_JOB_RUNNING;
            running.push_back(j);
            queue.pop_front();
            SRV_TRY(drop_batch());
        }
        return SCPHD_OK;
    }

    scphd_status step(int32_t* stepped) {
        SRV_TRY(complete());
        SRV_TRY(admit());
        if (stepped) *stepped = 0;
        if (running.empty()) return SCPHD_OK;
        if (dirty || !batch) {
            std::vector<scphd_filter*> fs;
            for (Job* j : running) fs.push_back(j->f);
            SRV_TRY(scphd_batch_create(fs.data(), (int32_t)fs.size(), use_graph ? 1 : 0, &batch));
            dirty = false;
            rebuilds++;
        }
        fr.resize(running.size());
        for (size_t i = 0; i < running.size(); ++i) {
            Job* j = running[i];
            const int k = j->next;
            const int64_t o = j->offs[k];
            fr[i].u = j->dz + o;
            fr[i].v = j->dz + j->total + o;
            fr[i].d = meas_dim == 3 ? j->dz + 2 * j->total + o : nullptr;
            fr[i].n = j->sizes[k];
            fr[i].fixed_camera = j->fixed[k];
        }
        cudaStream_t st = (cudaStream_t)scphd_batch_stream(batch);
        SRV_CUDA(cudaEventRecord(ev0, st));
        SRV_TRY(scphd_batch_step_device(batch, dt, fr.data()));   // one dt per server (checked at submit)
        SRV_CUDA(cudaEventRecord(ev1, st));
        for (Job* j : running) j->next++;
        in_flight = true;
        in_flight_jobs = (int)running.size();
        steps++;
        frames += (int64_t)running.size();
        if (stepped) *stepped = (int32_t)running.size();
        return SCPHD_OK;
    }
};

extern "C" {

scphd_status scphd_server_create(int32_t device, int32_t precision, int32_t meas_dim, int64_t budget_bytes,
                                 int32_t use_graph, scphd_server** out) {
    if (!out) return fail(SCPHD_ERR_INVALID, "null output");
    *out = nullptr;
    if (budget_bytes <= 0) return fail(SCPHD_ERR_INVALID, "budget must be positive");
    if (meas_dim != 2 && meas_dim != 3) return fail(SCPHD_ERR_INVALID, "meas_dim must be 2 or 3");
    if (precision != SCPHD_FP32 && precision != SCPHD_FP64) return fail(SCPHD_ERR_INVALID, "bad precision");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SCPHD_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(SCPHD_ERR_INVALID, "device ordinal out of range");
    SRV_CUDA(cudaSetDevice(device));
    std::unique_ptr<scphd_server> s(new scphd_server());
    s->device = device;
    s->precision = precision;
    s->meas_dim = meas_dim;
    s->budget = budget_bytes;
    s->use_graph = use_graph != 0;
    SRV_CUDA(cudaEventCreate(&s->ev0));
    SRV_CUDA(cudaEventCreate(&s->ev1));
    *out = s.release();
    return SCPHD_OK;
}

scphd_status scphd_server_destroy(scphd_server* s) {
    if (!s) return fail(SCPHD_ERR_INVALID, "null server");
    delete s;
    return SCPHD_OK;
}

scphd_status scphd_server_submit(scphd_server* s, const scphd_config* cfg, int32_t n_frames, const int32_t* sizes,
                                 const double* u, const double* v, const double* d, const int32_t* fixed,
                                 double dt, int64_t* job_id) {
    if (!s || !cfg || !job_id) return fail(SCPHD_ERR_INVALID, "null argument");
    if (n_frames < 1 || !sizes || !fixed) return fail(SCPHD_ERR_INVALID, "a job needs at least one frame");
    if (cfg->device != s->device || cfg->precision != s->precision || cfg->meas_dim != s->meas_dim)
        return fail(SCPHD_ERR_INVALID, "job device, precision or meas_dim differs from the server's");
    if (!std::isfinite(dt)) return fail(SCPHD_ERR_INVALID, "dt must be finite");
    if (s->has_dt && dt != s->dt) return fail(SCPHD_ERR_INVALID, "the jobs of one server share one dt");
    int64_t fb = 0;
    SRV_TRY(scphd_device_bytes(cfg, &fb));
    std::unique_ptr<Job> j(new Job());
    j->cfg = *cfg;
    j->n_frames = n_frames;
    j->dt = dt;
    j->sizes.assign(sizes, sizes + n_frames);
    j->fixed.assign(fixed, fixed + n_frames);
    j->offs.resize(n_frames);
    int64_t tot = 0;
    for (int k = 0; k < n_frames; ++k) {
        if (sizes[k] < 0 || sizes[k] > cfg->max_measurements)
            return fail(SCPHD_ERR_CAPACITY, "frame " + std::to_string(k) + " exceeds max_measurements");
        j->offs[k] = tot;
        tot += sizes[k];
    }
    if (tot > 0 && (!u || !v || (s->meas_dim == 3 && !d))) return fail(SCPHD_ERR_INVALID, "null measurement array");
    for (int64_t i = 0; i < tot; ++i)
        if (!std::isfinite(u[i]) || !std::isfinite(v[i]) || (s->meas_dim == 3 && !std::isfinite(d[i])))
            return fail(SCPHD_ERR_INVALID, "non-finite measurement");
    j->total = tot;
    j->zu.assign(u, u + tot);
    j->zv.assign(v, v + tot);
    if (s->meas_dim == 3) j->zd.assign(d, d + tot);
    j->bytes = fb + (int64_t)sizeof(double) * 3 * std::max<int64_t>(1, tot) + 4096;
    if (j->bytes > s->budget) return fail(SCPHD_ERR_CAPACITY, "job needs more device memory than the whole budget");
    s->has_dt = true;
    s->dt = dt;
    j->id = s->next_id++;
    *job_id = j->id;
    s->queue.push_back(j.get());
    s->jobs[j->id] = std::move(j);
    return SCPHD_OK;
}

scphd_status scphd_server_step(scphd_server* s, int32_t* stepped) {
    if (!s) return fail(SCPHD_ERR_INVALID, "null server");
    SRV_CUDA(cudaSetDevice(s->device));
    return s->step(stepped);
}

scphd_status scphd_server_drain(scphd_server* s) {
    if (!s) return fail(SCPHD_ERR_INVALID, "null server");
    SRV_CUDA(cudaSetDevice(s->device));
    return s->complete();
}

scphd_status scphd_server_job_status(scphd_server* s, int64_t job, int32_t* state, int32_t* frames_done) {
    if (!s) return fail(SCPHD_ERR_INVALID, "null server");
    auto it = s->jobs.find(job);
    if (it == s->jobs.end()) return fail(SCPHD_ERR_INVALID, "unknown job");
    const Job* j = it->second.get();
    if (state) *state = j->state;
    if (frames_done) *frames_done = j->state == SCPHD_JOB_DONE ? j->n_frames : std::max(0, j->next - (s->in_flight ? 1 : 0));
    return SCPHD_OK;
}

scphd_status scphd_server_job_result(scphd_server* s, int64_t job, double* states, double* log_weights) {
    if (!s) return fail(SCPHD_ERR_INVALID, "null server");
    auto it = s->jobs.find(job);
    if (it == s->jobs.end()) return fail(SCPHD_ERR_INVALID, "unknown job");
    const Job* j = it->second.get();
    if (j->state != SCPHD_JOB_DONE) return fail(SCPHD_ERR_INVALID, "job not done");
    if (states) std::copy(j->states.begin(), j->states.end(), states);
    if (log_weights) std::copy(j->lw.begin(), j->lw.end(), log_weights);
    return SCPHD_OK;
}

scphd_status scphd_server_stats(scphd_server* s, int64_t out[8]) {
    if (!s || !out) return fail(SCPHD_ERR_INVALID, "null argument");
    int64_t done = 0;
    for (auto& kv : s->jobs) done += kv.second->state == SCPHD_JOB_DONE;
    out[0] = (int64_t)s->queue.size();
    out[1] = (int64_t)s->running.size();
    out[2] = done;
    out[3] = s->used;
    out[4] = s->steps;
    out[5] = s->frames;
    int64_t units = s->units_done;
    for (Job* j : s->running) {   // reads the running jobs' device counters (waits for their work)
        int64_t c[16];
        SRV_TRY(scphd_get_counters(j->f, c));
        units += c[6];
    }
    out[6] = units;
    out[7] = s->rebuilds;
    return SCPHD_OK;
}

scphd_status scphd_server_step_times(scphd_server* s, int64_t first, int32_t max, double* ms, int32_t* jobs,
                                     int32_t* n_out) {
    if (!s || !n_out || first < 0 || max < 0) return fail(SCPHD_ERR_INVALID, "bad argument");
    int32_t n = 0;
    for (int64_t i = first; i < (int64_t)s->step_ms.size() && n < max; ++i, ++n) {
        if (ms) ms[n] = s->step_ms[i];
        if (jobs) jobs[n] = s->step_jobs[i];
    }
    *n_out = n;
    return SCPHD_OK;
}

}  // extern "C"

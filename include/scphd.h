/*
 * scphd.h — C ABI of the B200 SC-PHD camera-calibration filter step.
 *
 * One handle = one filter: N parent particles (12-D camera extrinsics, FP64) each
 * owning a Gaussian-mixture map in 6-D disparity space (u, v, d, vu, vv, vd).
 * The entry points replace the step API of the reference class
 * SCPHDCameraCalibration (src/scphdcameracalibration.cuh:29-44):
 *
 *   reference                                   this ABI
 *   SCPHDCameraCalibration(cfg)  (.cu:823-1006) scphd_create
 *   predict(double dt)           (.cu:1034-1151) scphd_predict
 *   update(u, v, fixed_camera)   (.cu:1576-2094) scphd_update (d == NULL: (u,v) mode)
 *   resample()                   (.cu:2651-2817) scphd_resample
 *   checkStuff()                 (.cu:812-821)   scphd_check
 *   writeMat() particle dump     (.cu:2200-2373) scphd_get_particles / scphd_get_mixture
 *
 * Conventions: every call returns an scphd_status and never throws across the ABI.
 * Host arrays are copied during the call (the reference passes measurements by
 * value).  All device work of a handle runs on the handle's own CUDA stream; calls
 * on distinct handles may come from distinct threads, calls on one handle must be
 * serialised by the caller.  Memory is allocated once, in scphd_create, from the
 * capacities in scphd_config; no call allocates afterwards.
 */
#ifndef SCPHD_H
#define SCPHD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum scphd_status {
    SCPHD_OK = 0,
    SCPHD_ERR_INVALID = 1,      /* bad argument or configuration */
    SCPHD_ERR_CUDA = 2,         /* CUDA runtime error (message in scphd_last_error) */
    SCPHD_ERR_CAPACITY = 3,     /* a size exceeds the capacity fixed at create time */
    SCPHD_ERR_NAN = 4,          /* scphd_check found a NaN parent weight */
    SCPHD_ERR_NO_DEVICE = 5
} scphd_status;

/* Arithmetic of the Kalman update, merge and sample clouds.  Parent states,
 * parent log-weights, the log-likelihood accumulation and the resampling prefix
 * sum are FP64 in both modes. */
enum { SCPHD_FP32 = 0, SCPHD_FP64 = 1 };

/* Filter configuration.  Field names follow the keys the reference reads through
 * libconfig (src/scphdcameracalibration.cu:827-1005, 1145, 1343, 1744, 1920,
 * 2596-2610, 2655); the capacity fields, meas_dim, std_d, baseline, kappa,
 * precision and seed are additions of this implementation. */
typedef struct scphd_config {
    int32_t n_parents;              /* n_particles */
    int32_t particles_per_feature;  /* Monte-Carlo samples per daughter Gaussian, <= 256 */
    int32_t max_gaussians;          /* per-parent map capacity (G_max) */
    int32_t max_measurements;       /* per-frame measurement capacity (M_max) */
    int32_t meas_dim;               /* 2: (u,v) as the reference; 3: (u,v,d) */
    int32_t precision;              /* SCPHD_FP32 or SCPHD_FP64 */
    int32_t max_survivors;          /* per-parent merge scratch; 0 = 4*max_gaussians+max_measurements */
    int32_t device;                 /* CUDA device ordinal */
    uint64_t seed;                  /* key of the counter-based random streams */
    /* prior.{cartesian,angular}.{x,y,z,vx,vy,vz}.{a,b}: uniform prior box */
    double prior_a[12];
    double prior_b[12];
    /* camera_motion_model.{cartesian,angular}.{ax,ay,az} (acceleration std) */
    double cam_std[6];
    /* feature_motion_model.{ax,ay,az} */
    double feat_std[3];
    /* measurement_model.{fx,fy,u0,v0,std_u,std_v,pd}; std_d for meas_dim 3 */
    double fx, fy, u0, v0, std_u, std_v, std_d, pd;
    double kappa;                   /* clutter density; the reference uses lambda/(2 v0)^2 */
    double baseline;                /* stereo baseline B in d = -fx B / z; 1 reproduces the reference */
    double ps;                      /* survival probability */
    double min_weight;              /* prune threshold */
    double min_separation;          /* squared Mahalanobis merge threshold */
    double min_neff;                /* resample when N_eff/N < min_neff */
    /* birth.{w0,d0,vu0,vv0,vd0,var_d0,var_vu0,var_vv0,var_vd0} */
    double w0, d0, vu0, vv0, vd0, var_d0, var_vu0, var_vv0, var_vd0;
} scphd_config;

typedef struct scphd_filter scphd_filter;

/* Fill *cfg with the values of the reference's shipped config/calibration.cfg
 * (n_particles 100, particles_per_feature 100, min_weight 1e-4, ...), meas_dim 2,
 * baseline 1 and kappa = lambda/(2 v0)^2 with lambda 10.0001. */
void scphd_config_defaults(scphd_config* cfg);

/* SCPHDCameraCalibration(cfg): allocate device state, draw the uniform prior. */
scphd_status scphd_create(const scphd_config* cfg, scphd_filter** out);
scphd_status scphd_destroy(scphd_filter* f);

/* predict(dt): parent motion runs now; the feature-cloud motion is fused into the
 * next scphd_update. */
scphd_status scphd_predict(scphd_filter* f, double dt);

/* update(u, v, fixed_camera).  u, v (and d when meas_dim == 3) are HOST arrays of n
 * values.  fixed_camera != 0 transforms with the identity extrinsic and leaves the
 * parent weights unchanged, as the reference does. */
scphd_status scphd_update(scphd_filter* f, const double* u, const double* v,
                          const double* d, int32_t n, int32_t fixed_camera);

/* Same as scphd_update with DEVICE arrays (FP64, n values each; d may be NULL). */
scphd_status scphd_update_device(scphd_filter* f, const double* u_dev, const double* v_dev,
                                 const double* d_dev, int32_t n, int32_t fixed_camera);

/* resample(): systematic resampling when N_eff/N < min_neff.  *resampled (may be
 * NULL) receives 1 if it happened; the decision is read back from the device. */
scphd_status scphd_resample(scphd_filter* f, int32_t* resampled);

/* predict + update + resample in one call with no host synchronisation inside:
 * the resampling decision stays on the device.  Host measurement arrays. */
scphd_status scphd_step(scphd_filter* f, double dt, const double* u, const double* v,
                        const double* d, int32_t n, int32_t fixed_camera);

/* scphd_step with DEVICE measurement arrays (FP64; d may be NULL in (u,v) mode). */
scphd_status scphd_step_device(scphd_filter* f, double dt, const double* u_dev, const double* v_dev,
                               const double* d_dev, int32_t n, int32_t fixed_camera);

/* checkStuff(): SCPHD_ERR_NAN if any parent weight is NaN. */
scphd_status scphd_check(scphd_filter* f);

/* Wait for the handle's stream. */
scphd_status scphd_synchronize(scphd_filter* f);

/* Parent states (n_parents x 12 FP64: cartesian x,y,z,vx,vy,vz, angular x,y,z,vx,vy,vz)
 * and normalised log-weights (n_parents FP64).  Either pointer may be NULL. */
scphd_status scphd_get_particles(scphd_filter* f, double* states, double* log_weights);

/* The same copies, queued on the handle's stream (scphd_stream) after the work issued so
 * far, without waiting for them: the buffers hold the states and log-weights of that
 * point once scphd_synchronize(f) returns or an event recorded on the stream after this
 * call has completed.  With page-locked (pinned) buffers the copy overlaps the host's
 * next calls, so a caller can read step k's result while step k + 1 runs.  The buffers
 * must stay valid until then.  No reference counterpart (writeMat reads synchronously). */
scphd_status scphd_get_particles_async(scphd_filter* f, double* states, double* log_weights);

/* Map size of each parent (n_parents int32). */
scphd_status scphd_get_map_sizes(scphd_filter* f, int32_t* sizes);

/* Gaussian weights of parent p's map (sizes[p] FP64). */
scphd_status scphd_get_map_weights(scphd_filter* f, int32_t p, double* weights);

/* Euclidean sample cloud of parent p's map: sizes[p] x 6 x particles_per_feature
 * coordinates (x,y,z,vx,vy,vz) and sizes[p] x particles_per_feature sample
 * weights, FP64.  Merged components are regenerated from their stored parameters
 * with the same random streams the next update consumes. */
scphd_status scphd_get_map_clouds(scphd_filter* f, int32_t p, double* xyz, double* omega);

/* Inspection of the last update (the reference's save_all_maps dumps):
 * which = SCPHD_MIX_FITTED: the predicted mixture refitted in disparity space,
 *         per Gaussian 29 values: weight, mean pD, mean[6], packed lower cov[21];
 * which = SCPHD_MIX_MERGED: the merged mixture, per Gaussian 28 values: weight,
 *         mean[6], packed lower cov[21].  *count receives the number of rows;
 * out may be NULL to query the count. */
enum { SCPHD_MIX_FITTED = 0, SCPHD_MIX_MERGED = 1 };
scphd_status scphd_get_mixture(scphd_filter* f, int32_t which, int32_t p,
                               double* out, int32_t* count);

/* Per-(parent, measurement) log normalisers of the last update (n_parents x n FP64)
 * and per-parent log-likelihood increments (n_parents FP64). */
scphd_status scphd_get_normalizers(scphd_filter* f, double* ell, double* loglik);

/* Resampling indices of the last resample that happened (n_parents int32). */
scphd_status scphd_get_resample_indices(scphd_filter* f, int32_t* idx);

/* Replace the filter state: parent states (N x 12), log-weights (N), and per parent
 * a map given as Euclidean clouds: sizes (N), weights (sum sizes), clouds
 * (sum sizes x 6 x P_f) and sample weights (sum sizes x P_f).  Clears any
 * pending prediction.  Used to start device and reference from one state. */
scphd_status scphd_set_state(scphd_filter* f, const double* states, const double* log_weights,
                             const int32_t* sizes, const double* weights,
                             const double* clouds, const double* omega);

/* Counters since create: [0] map truncations at max_gaussians, [1] merge-scratch
 * overflows at max_survivors, [2] frames updated, [3] resamplings,
 * [4] Gaussian-measurement units of the last update (sum_p G_p * n),
 * [5] survivors of the last update (sum over parents), [6] units since create,
 * [7] survivors since create, [8] sample clouds read from memory, [9] sample
 * clouds written, [10] Gaussians fitted, [11] merged components produced,
 * [12] full Mahalanobis evaluations in the merge, [13] largest survivor count of
 * one parent (before the max_survivors cut), [14] Gaussians fitted with unit sample
 * weights (in view, but every in-view sample of zero weight: only with pd = 1);
 * [15] reserved. */
scphd_status scphd_get_counters(scphd_filter* f, int64_t counters[16]);

/* Launch shapes tuned on the filter's first updates that have measurements: threads
 * per merge block (256 or 128) and the likelihood's blocks (1: one block over all of a
 * parent's measurements, 0: 128-thread blocks).  Each of the four combinations runs
 * twice, timed with events (those updates wait for the previous one), and the fastest is
 * kept.  Results do not depend on the shape.  enable = 0 stops tuning and keeps
 * (256, 1); *tuned = 1 once a choice is made.  No reference counterpart. */
scphd_status scphd_set_autotune(scphd_filter* f, int32_t enable);
scphd_status scphd_get_launch_shapes(scphd_filter* f, int32_t* merge_threads, int32_t* likelihood_full,
                                     int32_t* tuned);

/* Update path: 0 (the default) = one kernel per stage; 1 = the fused kernel (one
 * launch runs the cloud fit, Kalman terms, likelihood and merge of every parent, each
 * parent's stages in one block, blocks taking parents from a work counter).  The fused
 * kernel was measured slower than the stage kernels on every workload of this project
 * (it runs the cloud fit at lower occupancy and each block's Kalman terms as a serial
 * tail), so it runs only on request.  Per-stage profiling (scphd_set_profiling) always
 * runs the stage kernels.  Results equal the stage kernels' (FP64: bit for bit; FP32:
 * to FP32 rounding, as the two builds may contract multiply-adds differently).
 * scphd_get_fused reports the path the next update takes.  No reference counterpart
 * (the reference runs its stages as separate kernels and host loops,
 * src/scphdcameracalibration.cu:1576-2094). */
scphd_status scphd_set_fused(scphd_filter* f, int32_t mode);
scphd_status scphd_get_fused(scphd_filter* f, int32_t* fused);

/* Cloud-fit tiling: blocks per parent (1, 2 or 4).  Each block has 8 warps and the
 * parent's daughter Gaussians are dealt out over the warps of all its blocks (a warp
 * per Gaussian), so 2 or 4 blocks per parent fill the GPU when a filter has few
 * parents (256 blocks leave most of 148 SMs x 4 block slots idle).  By default the
 * updates with measurements after the first 16 (when the maps have grown) time the
 * cloud-fit launch at each split (twice) and keep the fastest; until then the split is
 * 1.  scphd_set_fit_split fixes one (and ends that tuning),
 * scphd_set_autotune(f, 0) fixes 1.  Results do not depend on the split.  *tuned = 1
 * once a choice is made.  No reference counterpart (fitGaussiansKernel runs a block
 * per Gaussian, src/kernels.cu:102-438). */
scphd_status scphd_set_fit_split(scphd_filter* f, int32_t blocks_per_parent);
scphd_status scphd_get_fit_split(scphd_filter* f, int32_t* blocks_per_parent, int32_t* tuned);

/* The configuration the filter was created with. */
scphd_status scphd_get_config(scphd_filter* f, scphd_config* out);

/* The CUDA stream (a cudaStream_t) all of the handle's work is issued on, so a
 * caller can order its own work or timing events after the filter's. */
void* scphd_stream(scphd_filter* f);

/* Per-stage device timing with CUDA events recorded on the handle's stream around
 * each stage's kernel (off by default).  Stages: 0 parent prediction, 1 cloud
 * fit, 2 likelihood/survivors, 3 merge, 4 parent weights, 5 resampling, 6 Kalman
 * terms of the fitted Gaussians.
 * scphd_get_stage_times synchronises the stream, returns the summed milliseconds
 * and launch counts per stage since the last call, and clears them. */
scphd_status scphd_set_profiling(scphd_filter* f, int32_t enable);
scphd_status scphd_get_stage_times(scphd_filter* f, double ms[8], int64_t launches[8]);

/* Stand-alone stages on caller-provided HOST data, for parity checks of the
 * device code paths the step uses.
 *
 * scphd_merge_components: the greedy GM reduction of phdUpdateMergeKernel
 * (src/kernels.cu:662-874) on one list of n components (28 FP64 each: weight,
 * mean[6], packed lower cov[21]) with prune flags (1 = excluded).  Outputs the
 * merged list (up to n rows of 28) in *n_out and, per input, the output row it was
 * absorbed into (-1 if none).  precision selects the FP32 or FP64 device code. */
scphd_status scphd_merge_components(const double* comps, const uint8_t* flags, int32_t n,
                                    double min_separation, int32_t precision,
                                    double* merged, int32_t* n_out, int32_t* member_of);

/* scphd_merge_components_static: the same greedy merge as scphd_merge_components,
 * for callers that must not allocate device memory — a host that runs inside
 * another framework's memory pool (which owns all free device memory, so a
 * cudaMalloc can fail), or a latency-bounded loop (cudaMalloc and cudaFree can
 * synchronise the device and stall behind unrelated work).  It calls no
 * cudaMalloc, cudaFree or other allocating routine: its device scratch (inputs,
 * outputs and working rows, about 0.6 MB) is one static array that every GPU
 * loading this library holds until the process exits.  Limits and sharing:
 * n <= SCPHD_STATIC_MERGE_MAX components (larger n returns SCPHD_ERR_CAPACITY);
 * every call on a device uses the same array, so calls that overlap on the GPU
 * (from several host threads) race and must be serialised by the caller; the
 * array keeps the previous call's contents, and the call re-initialises what it
 * reads.  The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call before
 * any stream capture.  Arguments, outputs and errors as scphd_merge_components.
 * This entry point has no counterpart in the reference. */
#define SCPHD_STATIC_MERGE_MAX 512
scphd_status scphd_merge_components_static(const double* comps, const uint8_t* flags, int32_t n,
                                           double min_separation, int32_t precision,
                                           double* merged, int32_t* n_out, int32_t* member_of);

/* scphd_systematic_resample: the systematic resampling of resample()
 * (src/scphdcameracalibration.cu:2660-2702) on n linear weights with the offset
 * u01 * (1/n); writes n indices. */
scphd_status scphd_systematic_resample(const double* weights, int32_t n, double u01,
                                       int32_t* idx);

/* Device memory, in bytes, that scphd_create would allocate for this configuration
 * (the filter's arena).  Pure arithmetic: needs no device.  For admission by memory
 * budget; no reference counterpart. */
scphd_status scphd_device_bytes(const scphd_config* cfg, int64_t* bytes);

/* ------------------------------------------------------------------ batches
 * Many filters advanced together: every batched step runs predict(dt) + update +
 * resample for all member filters with one kernel launch per stage (seven per frame,
 * or four with the fused update, whatever the number of filters), each launch covering
 * every filter's parents
 * through a block -> (filter, parent) map.  Member filters must share device,
 * precision and meas_dim; they may differ in size.  While in a batch, the filters
 * issue all their work on the batch's stream (their own stream is restored by
 * scphd_batch_destroy), so single-filter calls stay ordered with batched steps.  With
 * use_graph != 0 the first step captures the step into a CUDA graph and later steps
 * replay it.  A batched step gives each filter the same result as predict + update +
 * resample on that filter alone.  This batching has no counterpart in the reference
 * (which runs one filter per process). */
typedef struct scphd_frame {
    const double* u;        /* n measurements */
    const double* v;
    const double* d;        /* NULL in (u,v) mode */
    int32_t n;
    int32_t fixed_camera;
} scphd_frame;

typedef struct scphd_batch scphd_batch;

scphd_status scphd_batch_create(scphd_filter* const* filters, int32_t n_filters, int32_t use_graph,
                                scphd_batch** out);
scphd_status scphd_batch_destroy(scphd_batch* b);
/* frames[i] is filter i's frame; arrays in HOST memory (copied during the call).  The
 * step is queued on the batch's stream and the call returns; the next call waits only
 * until this step's frame copies have run (not its kernels), so consecutive steps
 * overlap their host work with the previous step's kernels. */
scphd_status scphd_batch_step(scphd_batch* b, double dt, const scphd_frame* frames);
/* As scphd_batch_step with the frames' arrays in DEVICE memory (read by the kernels;
 * keep them unchanged until the step has run on the batch's stream). */
scphd_status scphd_batch_step_device(scphd_batch* b, double dt, const scphd_frame* frames);
/* The batch's CUDA stream (a cudaStream_t). */
void* scphd_batch_stream(scphd_batch* b);
/* The batch's update path, as scphd_set_fused / scphd_get_fused: 0 (default) the
 * stage kernels, 1 the fused kernel (set before the first graph capture).  A fused
 * batch step is four launches per group of up to 32 filters: prediction (with the
 * frame's measurement conversion), the fused update, parent weights, resampling. */
scphd_status scphd_batch_set_fused(scphd_batch* b, int32_t mode);
scphd_status scphd_batch_get_fused(scphd_batch* b, int32_t* fused);
/* The batch's cloud-fit tiling, as scphd_set_fit_split / scphd_get_fit_split (one
 * split for all member filters, tuned on the batch's first six steps before its graph
 * is captured; set it before the capture). */
scphd_status scphd_batch_set_fit_split(scphd_batch* b, int32_t blocks_per_parent);
scphd_status scphd_batch_get_fit_split(scphd_batch* b, int32_t* blocks_per_parent, int32_t* tuned);

/* ------------------------------------------------------------------ serving
 * A resident request loop over batches.  A job is a filter configuration plus its
 * whole frame sequence.  Jobs may be submitted at any time; they are admitted first
 * come, first served while their device memory (filter arena + frame sequence) fits
 * the server's budget, kept resident between frames, and advanced together: each
 * scphd_server_step steps every resident job by one frame in one batched step.  A
 * job that has processed its last frame is retired at the next call: its parent
 * states and log-weights are copied out, its memory returns to the budget, and
 * queued jobs that now fit are admitted.  Each job's result equals that of the same
 * filter stepped alone.  All jobs of a server share device, precision, meas_dim and dt.
 * Calls on one server must be serialised by the caller.  No reference counterpart
 * (the reference runs one filter per process). */
typedef struct scphd_server scphd_server;
enum { SCPHD_JOB_QUEUED = 0, SCPHD_JOB_RUNNING = 1, SCPHD_JOB_DONE = 2 };

scphd_status scphd_server_create(int32_t device, int32_t precision, int32_t meas_dim, int64_t budget_bytes,
                                 int32_t use_graph, scphd_server** out);
scphd_status scphd_server_destroy(scphd_server* s);
/* Frame k has sizes[k] measurements at offset sizes[0] + ... + sizes[k-1] of u, v and
 * d (d NULL when meas_dim == 2); fixed[k] != 0 marks a fixed-camera frame; every
 * frame is preceded by predict(dt).  Host arrays, copied during the call.  A job
 * larger than the whole budget is refused with SCPHD_ERR_CAPACITY. */
scphd_status scphd_server_submit(scphd_server* s, const scphd_config* cfg, int32_t n_frames, const int32_t* sizes,
                                 const double* u, const double* v, const double* d, const int32_t* fixed,
                                 double dt, int64_t* job_id);
/* One serving iteration: wait for the previous step, retire the jobs it finished,
 * admit queued jobs that fit, then queue one batched step of every resident job and
 * return without waiting for it.  *stepped = jobs in that step (0: nothing resident). */
scphd_status scphd_server_step(scphd_server* s, int32_t* stepped);
/* Wait for the last step and retire the jobs it finished. */
scphd_status scphd_server_drain(scphd_server* s);
scphd_status scphd_server_job_status(scphd_server* s, int64_t job, int32_t* state, int32_t* frames_done);
/* Result of a DONE job: states (n_parents x 12, row-major) and log-weights (n_parents). */
scphd_status scphd_server_job_result(scphd_server* s, int64_t job, double* states, double* log_weights);
/* out[0] queued jobs, [1] running, [2] done, [3] device bytes in use, [4] steps,
 * [5] job-frames stepped, [6] Gaussian-measurement updates of all admitted jobs
 * (reading the running jobs' counters waits for their queued work), [7] batch
 * rebuilds. */
scphd_status scphd_server_stats(scphd_server* s, int64_t out[8]);
/* Device time in ms of completed steps first .. first+max-1 (oldest first) and the
 * number of jobs each advanced; *n_out = entries written. */
scphd_status scphd_server_step_times(scphd_server* s, int64_t first, int32_t max, double* ms, int32_t* jobs,
                                     int32_t* n_out);

/* Text of the last error on this thread. */
const char* scphd_last_error(void);

/* Number of CUDA kernels this library launched since load (all handles). */
int64_t scphd_kernel_launches(void);

#ifdef __cplusplus
}
#endif

#endif /* SCPHD_H */
